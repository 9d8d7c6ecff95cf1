/*
 * ifc_oracle.h -- CPU oracle for the SIMPLE hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a serial C restatement of the reference solver's kernels
 * (WanZijun271/IncompFlow-CUDA, include/kernels.cuh:10-1005) driven in the step
 * order of Solver::solve (src/Solver.cu:153-299).  It exists to check the CUDA
 * library; nothing in the product links or calls it.  Only tests/, the smoke
 * check in __graft_entry__.py and the cpu_baseline leg of bench.py use it.
 *
 * Differences from the reference, all deliberate and documented:
 *   - runtime configuration instead of compile-time constexpr (include/config.h);
 *   - 3D indexing is corrected (reference defects D2-D5: coefficient planes,
 *     wf layout, top/bottom index typos, missing `top` branch);
 *   - Gauss-Seidel is deterministic: lexicographic or red-black ordering instead
 *     of the reference's unordered in-place update (defect D8);
 *   - norms are accumulated in FP64 without the partial-block garbage of D7;
 *   - the convergence test offers the reference's rule (D6 reproduced) or a
 *     per-field rule.
 * Arithmetic otherwise follows the reference operation by operation, including
 * the places where a double literal promotes a float expression to FP64 (D13).
 *
 * Parity pinning: the reference ships no tests or golden vectors.  The oracle is
 * pinned against the reference's own kernels and Solver built from its sources
 * and run on a B200 (oracle/Makefile builds them into oracle/_ref/;
 * tests/golden/make_golden.py records their outputs).
 *
 * Two builds of every function exist: suffix _f (float) and _d (double).
 */
#ifndef IFC_ORACLE_H
#define IFC_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary face order and types, as in include/constants.h:7-12,32-34. */
enum { ORC_EAST = 0, ORC_WEST = 1, ORC_NORTH = 2, ORC_SOUTH = 3, ORC_TOP = 4, ORC_BOTTOM = 5 };
enum { ORC_WALL = 0, ORC_INLET = 1, ORC_OUTLET = 2 };
/* Coefficient slots, include/constants.h:14-20. */
enum { ORC_AC = 0, ORC_AE = 1, ORC_AW = 2, ORC_AN = 3, ORC_AS = 4, ORC_AT = 5, ORC_AB = 6 };
/* Linear sweep orderings. */
enum { ORC_GS_LEX = 0, ORC_GS_REDBLACK = 1, ORC_JACOBI = 2 };
/* Convergence rules. */
enum { ORC_CRIT_REFERENCE = 0, ORC_CRIT_PER_FIELD = 1, ORC_CRIT_RESIDUAL = 2 };
/* Equation ids for the linear solves. */
enum { ORC_EQ_U = 0, ORC_EQ_V = 1, ORC_EQ_W = 2, ORC_EQ_P = 3 };
/* Convection schemes; every scheme but upwind is applied by deferred correction. */
enum { ORC_CONV_UPWIND = 0, ORC_CONV_CENTRAL = 1, ORC_CONV_SOU = 2, ORC_CONV_QUICK = 3, ORC_CONV_MINMOD = 4,
       ORC_CONV_VAN_LEER = 5 };

typedef struct orc_config {
    int dim, nx, ny, nz;
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double density, viscosity;
    int bc_type[6];
    double bc_val[6][3];
    int num_outer_iter;
    int n_iter[4];          /* u v w p' sweeps per outer iteration */
    double relax[4];        /* u v w p */
    double tol[4];          /* u v w p */
    double tol_mass;
    int sweep_mode;         /* ORC_GS_LEX / ORC_GS_REDBLACK / ORC_JACOBI */
    int check_every;        /* sweeps between inner early-exit checks (1 = reference) */
    int criterion;          /* ORC_CRIT_REFERENCE / ORC_CRIT_PER_FIELD / ORC_CRIT_RESIDUAL */
    int pin_pressure;       /* subtract the FP64 mean of p' (closed domains) */
    const double *inlet_profile; /* optional: west-face normal velocity per boundary cell (ny*nz) */
    int convection;         /* ORC_CONV_*; 0 = first-order upwind, the reference's only scheme */
    int slab_axis_cells;    /* > 0: this state holds a slab of a grid with that many cells along
                               y (2D) or z (3D); the axis spacing is the whole grid's (the
                               library's ifc_config field of the same name) */
} orc_config;

/* Per-outer-iteration norms (RMS, FP64), src/Solver.cu:226-235. */
typedef struct orc_norms {
    double p, u, v, w, uf, vf, wf, mass;
    double rel_p, rel_u, rel_v, rel_w, rel_uf, rel_vf, rel_wf;
    double res_u, res_v, res_w;  /* RMS momentum residuals at the start of the iteration (FP64) */
    int sweeps[4];          /* sweeps actually done in this outer iteration */
    int converged;
} orc_norms;

typedef struct orc_state_f orc_state_f;
typedef struct orc_state_d orc_state_d;

/* Field ids for orc_field_*. */
enum {
    ORC_F_U = 0, ORC_F_V, ORC_F_W, ORC_F_P, ORC_F_PC, ORC_F_UF, ORC_F_VF, ORC_F_WF,
    ORC_F_MCOEF, ORC_F_PCOEF, ORC_F_SRC_U, ORC_F_SRC_V, ORC_F_SRC_W, ORC_F_SRC_P, ORC_F_COUNT
};

#define ORC_DECLARE(T, S)                                                                  \
    orc_state_##S *orc_create_##S(const orc_config *cfg);                                  \
    void orc_destroy_##S(orc_state_##S *s);                                                \
    T *orc_field_##S(orc_state_##S *s, int field);                                         \
    size_t orc_field_len_##S(const orc_state_##S *s, int field);                           \
    void orc_init_face_vel_##S(orc_state_##S *s);                                          \
    void orc_bc_face_vel_##S(orc_state_##S *s);                                            \
    void orc_mom_link_coef_##S(orc_state_##S *s);                                          \
    void orc_mom_src_##S(orc_state_##S *s);                                                \
    void orc_bc_mom_##S(orc_state_##S *s);                                                 \
    void orc_dc_source_##S(orc_state_##S *s);                                              \
    double orc_sweep_##S(orc_state_##S *s, int eq, int mode);                              \
    int orc_linear_solve_##S(orc_state_##S *s, int eq, double *sweep_norms);               \
    void orc_rhie_chow_##S(orc_state_##S *s);                                              \
    void orc_pcorr_link_coef_##S(orc_state_##S *s);                                        \
    double orc_pcorr_src_##S(orc_state_##S *s);                                            \
    void orc_pin_pcorr_##S(orc_state_##S *s);                                              \
    void orc_update_field_##S(orc_state_##S *s, orc_norms *out);                           \
    int orc_outer_iteration_##S(orc_state_##S *s, orc_norms *out);                         \
    int orc_solve_##S(orc_state_##S *s, int max_outer, orc_norms *last);                   \
    int orc_iteration_count_##S(const orc_state_##S *s);

ORC_DECLARE(float, f)
ORC_DECLARE(double, d)

/* Reverse pass of one SIMPLE outer iteration at a fixed point (2D, FP64):
 * given a seed on the outputs (u, v, p, uf, vf; boundary-face entries ignored)
 * returns G_x^T seed (same layout, boundary faces 0), G_theta^T seed (west
 * inlet rows, ny values; needs an inlet profile) and G_mu^T seed. */
int orc_adjoint_apply_d(orc_state_d *s, const double *lu_in, const double *lv_in, const double *lp_in,
                        const double *luf_in, const double *lvf_in, double *lu_out, double *lv_out, double *lp_out,
                        double *luf_out, double *lvf_out, double *ltheta, double *lmu);
void orc_set_iteration_count_f(orc_state_f *s, int it);
void orc_set_iteration_count_d(orc_state_d *s, int it);

#ifdef __cplusplus
}
#endif

#endif
