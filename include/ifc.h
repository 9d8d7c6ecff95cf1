/*
 * ifc.h -- C ABI of the B200 SIMPLE solver (libifc.so).
 *
 * The reference (WanZijun271/IncompFlow-CUDA) exposes one C++ class, Solver
 * (include/Solver.h:8-72), configured at compile time by include/config.h.
 * This header is the plain-C boundary underneath a drop-in replacement of that
 * class (incompflow-cuda_b200/host/Solver.h): opaque handles, int status codes,
 * host pointers and sizes only, no exceptions and no C++ or torch types.
 *
 * Ownership: the library owns all device memory of a handle; the caller owns
 * every host buffer it passes.  Threading: one handle per host thread; calls on
 * one handle must not overlap.  All work of a handle runs on one CUDA stream
 * (its own, or ifc_config.stream).  Every call that returns data is
 * host-synchronous on return, as the reference's Solver methods are.
 */
#ifndef IFC_H
#define IFC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IFC_ABI_VERSION 1

/* Status codes returned by every entry point (the reference reports none, D11). */
typedef enum ifc_status {
    IFC_OK = 0,
    IFC_NOT_CONVERGED = 1,   /* num_outer_iter reached without convergence */
    IFC_DIVERGED = 2,        /* NaN/Inf in a norm, or a norm grew 1e6x over its running max */
    IFC_TIMEOUT = 3,         /* a bounded device wait gave up */
    IFC_CUDA_ERROR = 4,
    IFC_BAD_CONFIG = 5,
    IFC_BAD_ARGUMENT = 6,
    IFC_IO_ERROR = 7,
    IFC_UNSUPPORTED = 8
} ifc_status;

/* Boundary faces and types: include/constants.h:7-12 and :32-34. */
enum { IFC_EAST = 0, IFC_WEST = 1, IFC_NORTH = 2, IFC_SOUTH = 3, IFC_TOP = 4, IFC_BOTTOM = 5 };
enum { IFC_WALL = 0, IFC_INLET = 1, IFC_OUTLET = 2 };

enum { IFC_FP32 = 0, IFC_FP64 = 1 };
/* Linear sweeps (reference: src/Solver.cu:868-966).  Gauss-Seidel runs in
 * red-black order (deterministic); Jacobi ping-pongs two buffers. */
enum { IFC_GAUSS_SEIDEL = 0, IFC_JACOBI = 1 };
/* Convergence rule.  REFERENCE reproduces src/Solver.cu:237-268 exactly,
 * including the division of every norm by the running max of the pressure norm;
 * PER_FIELD divides each norm by its own running max (FP64).  RESIDUAL (an
 * addition; not in the batched form) applies the per-field rule to FP64
 * residuals instead of corrections: u, v, w by the RMS of their assembled
 * momentum equation's residual b - aC phi - sum a_nb phi_nb at the start of
 * the outer iteration (tolerances tol_u, tol_v, tol_w), p by the RMS mass
 * imbalance (tol_p); in FP32 the correction norms level off at the rounding
 * noise of the corrected fields, these residuals do not. */
enum { IFC_CRIT_REFERENCE = 0, IFC_CRIT_PER_FIELD = 1, IFC_CRIT_RESIDUAL = 2 };

/* Convection schemes of the momentum equations.  IFC_CONV_UPWIND is the
 * reference's first-order upwind (include/kernels.cuh:97-134) and the default;
 * the others are applied by deferred correction: the links stay upwind and
 * F_f (phi_f,HO - phi_f,upwind) of every interior face whose far-upwind cell
 * is inside the domain enters the source, lagged by one outer iteration.
 * The reference lists such schemes as planned (README.md:412). */
enum {
    IFC_CONV_UPWIND = 0,
    IFC_CONV_CENTRAL = 1,
    IFC_CONV_SOU = 2,        /* second-order upwind (linear upwind) */
    IFC_CONV_QUICK = 3,
    IFC_CONV_MINMOD = 4,     /* TVD, minmod limiter */
    IFC_CONV_VAN_LEER = 5    /* TVD, van Leer limiter */
};

/* Field ids for ifc_get_field / ifc_set_field / ifc_device_ptr.  Layouts follow
 * the reference: cells i + nx*(j + ny*k); uf i + (nx+1)*(j + ny*k);
 * vf i + nx*(j + (ny+1)*k); wf i + nx*(j + ny*k) with k in [0, nz].
 * IFC_FIELD_MOM_COEF / PCORR_COEF hold 2*dim+1 planes coef[cell + N*slot], slot
 * order aC,aE,aW,aN,aS,aT,aB (include/constants.h:14-20); they are filled by
 * ifc_run_stage(IFC_STAGE_MOM_ASSEMBLE / IFC_STAGE_PCORR_COEF), the fused
 * solver never stores them. */
enum {
    IFC_FIELD_U = 0, IFC_FIELD_V, IFC_FIELD_W, IFC_FIELD_P, IFC_FIELD_T, IFC_FIELD_PCORR,
    IFC_FIELD_UF, IFC_FIELD_VF, IFC_FIELD_WF, IFC_FIELD_MOM_AC,
    IFC_FIELD_MOM_COEF, IFC_FIELD_PCORR_COEF,
    IFC_FIELD_SRC_U, IFC_FIELD_SRC_V, IFC_FIELD_SRC_W, IFC_FIELD_SRC_P,
    IFC_FIELD_COUNT
};

/* Every parameter of include/config.h:6-81 under the same meaning, plus the
 * new-build additions at the end.  Values are doubles and are rounded to the
 * solver's scalar type exactly as the reference's `constexpr scalar` are. */
typedef struct ifc_config {
    int dim;                          /* 2 or 3 */
    int nx, ny, nz;                   /* nz is forced to 1 when dim == 2 */
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double thermal_conductivity;      /* energy equation (ifc_solve_energy): Gamma = */
    double specific_heat_capacity;    /* thermal_conductivity / specific_heat_capacity */
    double density;
    double dynamic_viscosity;
    int vel_bc_type[6];               /* velBCs::type, face order E W N S T B */
    double vel_bc_val[6][3];          /* velBCs::val[face][u,v,w] */
    int temp_bc_type[6];              /* TempBCs: 0 Dirichlet (temp_bc_val), 1 Neumann (zero gradient) */
    double temp_bc_val[6];
    int num_outer_iter;
    int n_iter_u, n_iter_v, n_iter_w, n_iter_p;
    double relax_u, relax_v, relax_w, relax_p;
    double tol_u, tol_v, tol_w, tol_p, tol_mass;
    /* ---- additions ---- */
    int precision;                    /* IFC_FP32 (default) or IFC_FP64 */
    int linear_solver;                /* IFC_GAUSS_SEIDEL (default) or IFC_JACOBI */
    int criterion;                    /* IFC_CRIT_PER_FIELD (default), _REFERENCE or _RESIDUAL */
    int pin_pressure;                 /* -1 auto (closed domains), 0 off, 1 on */
    int sweeps_per_pass;              /* sweeps fused per device pass; 0 = tuned default */
    int log_level;                    /* 0 silent, 1 reference log cadence on stdout */
    const double *inlet_profile;      /* optional west-face inlet velocity per boundary cell (ny*nz) */
    void *stream;                     /* cudaStream_t to run on, or NULL for a private stream */
    int convection_scheme;            /* IFC_CONV_* (default IFC_CONV_UPWIND); ifc_adjoint takes
                                         IFC_CONV_UPWIND only */
    int slab_axis_cells;              /* 0 (default): the handle holds the whole grid.  > 0: it
                                         holds a slab of whole rows (2D) or planes (3D) of a grid
                                         with this many cells along y (2D) or z (3D), whose
                                         extents are ymin..ymax (zmin..zmax); that axis's spacing
                                         is (max - min) / slab_axis_cells, bit for bit the whole
                                         grid's.  Used by the slab decomposition; batches take 0 */
} ifc_config;

typedef struct ifc_stats {
    int status;                       /* ifc_status of the call */
    int outer_iterations;             /* total outer iterations done by the handle */
    int converged;
    int sweeps[4];                    /* u v w p' sweeps in the last outer iteration */
    long long cell_updates;           /* relaxed point updates done by the call */
    double norm_p, norm_u, norm_v, norm_w, norm_uf, norm_vf, norm_wf, norm_mass;   /* RMS, FP64 */
    double rel_p, rel_u, rel_v, rel_w, rel_uf, rel_vf, rel_wf;
    double device_ms;                 /* device time of the call (CUDA events) */
    long long kernel_launches;        /* device kernels launched by the call */
} ifc_stats;

typedef struct ifc_solver ifc_solver;

/* Fill *cfg with the values of the reference's shipped include/config.h. */
int ifc_config_default(ifc_config *cfg);

/* Validate a config without touching the GPU. */
int ifc_config_check(const ifc_config *cfg);

/* Replaces Solver::Solver (src/Solver.cu:13-104): allocates every device
 * buffer and sets uniform initial fields u=v=w=p=0, T=273 (the reference's
 * default arguments, include/Solver.h:50). */
int ifc_create(const ifc_config *cfg, ifc_solver **out);

/* Replaces Solver::~Solver (src/Solver.cu:106-151). NULL is accepted. */
int ifc_destroy(ifc_solver *h);

/* The constructor's uniform initial values (src/Solver.cu:15-21); also resets
 * face velocities, the iteration counter and the running norm maxima. */
int ifc_set_uniform(ifc_solver *h, double u, double v, double w, double p, double temp);

/* Copy a field between host and device.  bytes must equal the field's size in
 * the handle's precision (ifc_field_size). */
int ifc_set_field(ifc_solver *h, int field, const void *host, size_t bytes);
int ifc_get_field(ifc_solver *h, int field, void *host, size_t bytes);
size_t ifc_field_size(const ifc_solver *h, int field);

/* Device address of a field (valid until ifc_destroy). */
int ifc_device_ptr(ifc_solver *h, int field, void **dptr);

/* Replaces Solver::solve (src/Solver.cu:153-299): SIMPLE outer iterations from
 * the current state until convergence or num_outer_iter further iterations.
 * The whole loop runs on the device (CUDA graph with a device-side convergence
 * test); returns IFC_OK, IFC_NOT_CONVERGED or an error. */
int ifc_solve(ifc_solver *h, ifc_stats *stats);

/* Exactly n_outer outer iterations with the convergence test evaluated but not
 * acted on (fixed work, for throughput measurement). */
int ifc_iterate(ifc_solver *h, int n_outer, ifc_stats *stats);

/* Replaces Solver::writeVTK (src/Solver.cu:301-367): ASCII RECTILINEAR_GRID,
 * same header, coordinates and FIELD blocks, 6-significant-digit values.
 * The path is used as given (the Solver wrapper prepends output/). */
int ifc_write_vtk(ifc_solver *h, const char *path);

/* The same writer on host arrays (no GPU needed); arrays are float for
 * IFC_FP32 and double for IFC_FP64, nx*ny*nz each. */
int ifc_write_vtk_host(const ifc_config *cfg, const void *u, const void *v, const void *w,
                       const void *p, const void *temp, const char *path);

/* The same file in legacy VTK BINARY encoding: the header says BINARY and
 * every data block (coordinates, temperature, velocity, pressure) holds
 * big-endian values of the handle's scalar type, "float" or "double", so FP64
 * fields are written without rounding.  No counterpart in the reference, which
 * writes ASCII only (src/Solver.cu:301-367). */
int ifc_write_vtk_binary(ifc_solver *h, const char *path);
int ifc_write_vtk_binary_host(const ifc_config *cfg, const void *u, const void *v, const void *w,
                              const void *p, const void *temp, const char *path);

/* ---- batched form: many independent 2D cases in one persistent launch ---- */
typedef struct ifc_batch_result {
    int status;                       /* IFC_OK (converged), IFC_NOT_CONVERGED, IFC_DIVERGED */
    int outer_iterations;
    int converged;
    int sweeps[4];                    /* u v w p' sweeps of the last outer iteration */
    double rel_p, rel_u, rel_v, rel_uf, rel_vf, norm_mass;
    int tile_x, tile_y;               /* tile shape the case ran with (0 0: whole-row sweeps) */
    int sweeps_per_pass;              /* sweeps between the inner early-exit checks */
} ifc_batch_result;

/* Solves n independent 2D cases (each a full ifc_config: its own grid, fluid,
 * boundary conditions and iteration counts; all 2D, Gauss-Seidel, one
 * precision, criterion other than IFC_CRIT_RESIDUAL, slab_axis_cells 0:
 * IFC_UNSUPPORTED otherwise) to convergence or num_outer_iter, in persistent kernels of
 * thread-block clusters that take cases from a device queue, relaunched by a
 * CUDA graph until every case has finished.  Each case runs the same SIMPLE
 * iteration as ifc_solve.  A case's size class (up to 64^2, 160^2, larger
 * cells) selects how its sweeps run: whole-row sweeps, or temporally blocked
 * passes of a tile shape and sweeps per pass; the first batch of a process
 * that meets a class times every variant on copies of the class's median case
 * and keeps the fastest for the rest of the process (IFC_BATCH_VARIANT=<k> in
 * the environment forces variant k).  results: n
 * entries.  fields_out (optional): n host pointers, each receiving u, v, p of
 * its case (3*nx*ny values of the case's precision), or NULL entries.
 * device_ms (optional): device time of the whole batch.  Device memory is
 * allocated for the call and freed before it returns.  No counterpart in the
 * reference (which solves one compiled-in case per executable). */
int ifc_batch_solve(const ifc_config *cases, int n, ifc_batch_result *results, void *const *fields_out,
                    double *device_ms);

/* Replaces the west-inlet velocity profile of a handle created with an
 * inlet_profile (ny*nz host doubles, stored in the handle's precision); the
 * next solve, iteration or adjoint uses it.  IFC_BAD_ARGUMENT when the handle
 * has no profile.  No counterpart in the reference (its inlet is a compiled-in
 * constant); it lets a design loop update theta without rebuilding a handle. */
int ifc_set_inlet_profile(ifc_solver *h, const double *profile);

/* ---- energy equation on the converged flow ---- */
typedef struct ifc_energy_result {
    int status;
    int sweeps;                       /* red-black sweeps done */
    int converged;
    double residual;                  /* last sweep's RMS change over the largest of this solve */
    double device_ms;
} ifc_energy_result;

/* Steady temperature on the handle's current face mass fluxes (solve the
 * flow first): div(rho u T) = div(Gamma grad T) with Gamma =
 * thermal_conductivity / specific_heat_capacity, discretised like the
 * momentum equations (upwind convection, central diffusion, the same
 * boundary fold-in: wall form for Dirichlet faces, zero-gradient form for
 * Neumann faces, temp_bc_type/temp_bc_val), solved by unrelaxed red-black
 * Gauss-Seidel sweeps from the current temperature until the RMS change of
 * a sweep falls below tol times the largest of this solve (FP64 norms), or
 * max_sweeps (tol 0: exactly max_sweeps).  With a convection_scheme other
 * than IFC_CONV_UPWIND the sweeps run in cycles of 25, each starting from the
 * source plus the deferred correction of the current temperature, and the
 * solve ends when a cycle meets tol in its first sweep.  The result is the T field
 * (IFC_FIELD_T, written by ifc_write_vtk).  Returns IFC_NOT_CONVERGED when
 * max_sweeps ran out first.  The reference carries TempBCs and writes T but
 * never solves the energy equation. */
int ifc_solve_energy(ifc_solver *h, int max_sweeps, double tol, ifc_energy_result *result);

/* ---- differentiation form: discrete adjoint of the converged 2D solve ---- */
/* Objectives of ifc_adjoint. */
enum {
    IFC_OBJ_PRESSURE_DROP = 0,        /* J = mean p of the first cell column - mean of the last */
    IFC_OBJ_CUSTOM = 1                /* dJ/du, dJ/dv, dJ/dp given by the caller */
};

typedef struct ifc_adjoint_result {
    int status;
    int iterations;                   /* adjoint fixed-point iterations (reverse passes) */
    int converged;
    double residual;                  /* last max|lambda_new - lambda| / max|lambda_new| */
    double objective;                 /* J at the current state (IFC_OBJ_PRESSURE_DROP), else NaN */
    double dJ_dmu;                    /* gradient with respect to the dynamic viscosity */
    double device_ms;                 /* device time of the whole call (CUDA events) */
    long long kernel_launches;
} ifc_adjoint_result;

/* Gradient of an objective J(u, v, p) of the converged state with respect to
 * the west-inlet velocity of every boundary row (theta, ny values: the
 * inlet_profile entries, or the uniform inlet value per row) and the dynamic
 * viscosity, by the discrete adjoint of the SIMPLE outer iteration: the
 * adjoint lambda = G_x^T lambda + dJ/dx is iterated from lambda = dJ/dx to
 * relative change `tol` (at most max_iter reverse passes), and
 * dJ/dtheta = G_theta^T lambda, dJ/dmu = G_mu^T lambda.  The linearisation is
 * taken at the handle's current fields (solve first); all adjoint arithmetic
 * is FP64 for either precision of the handle.  dJ_du/dJ_dv/dJ_dp: host arrays
 * of nx*ny doubles (NULL = 0), read with IFC_OBJ_CUSTOM only.  dJ_dtheta:
 * host array of ny doubles (zeros unless the west face is an inlet).  2D,
 * red-black Gauss-Seidel and upwind convection only (IFC_UNSUPPORTED
 * otherwise).  Returns
 * IFC_NOT_CONVERGED when max_iter passes did not reach tol (the gradient of
 * the last iterate is still returned).  No counterpart in the reference. */
int ifc_adjoint(ifc_solver *h, int objective, const double *dJ_du, const double *dJ_dv, const double *dJ_dp,
                int max_iter, double tol, double *dJ_dtheta, ifc_adjoint_result *result);

/* One reverse pass at the current fields: out = G_x^T lambda (u, v, p: nx*ny;
 * uf: (nx+1)*ny; vf: nx*(ny+1); boundary-face entries of lambda are ignored
 * and those of out are 0), dJ_dtheta = G_theta^T lambda (ny), *dJ_dmu =
 * G_mu^T lambda.  All host arrays of doubles.  For testing the adjoint
 * operator against a transposition of the forward iteration. */
int ifc_adjoint_apply(ifc_solver *h, const double *lam_u, const double *lam_v, const double *lam_p,
                      const double *lam_uf, const double *lam_vf, double *out_u, double *out_v, double *out_p,
                      double *out_uf, double *out_vf, double *dJ_dtheta, double *dJ_dmu);

/* ---- single steps, for testing one application of each device kernel ---- */
enum {
    IFC_STAGE_FACE_BC = 0,       /* first iteration: face init; then face BCs (kernels.cuh:10-95) */
    IFC_STAGE_MOM_ASSEMBLE = 1,  /* materialise coefficients + sources (kernels.cuh:97-334), with the
                                    deferred-correction sources when convection_scheme != UPWIND */
    IFC_STAGE_MOM_SOLVE = 2,     /* assembly fused with the u,v,w sweeps (kernels.cuh:926-1005) */
    IFC_STAGE_RHIE_CHOW = 3,     /* faces + face BCs + p' source + mass norm (kernels.cuh:336-500,542-581) */
    IFC_STAGE_PCORR_COEF = 4,    /* materialise p' link coefficients (kernels.cuh:502-540) */
    IFC_STAGE_PCORR_SOLVE = 5,   /* p' = 0, then the p' sweeps (src/Solver.cu:193-196) */
    IFC_STAGE_UPDATE = 6,        /* corrections, norms, convergence test (kernels.cuh:583-843) */
    IFC_STAGE_COUNT = 7
};
int ifc_run_stage(ifc_solver *h, int stage);

/* The same launches on the handle's stream without waiting for them (for a
 * caller that orders its own work after them on that stream, such as halo
 * copies or NCCL transfers between slabs); their outcome -- a bounded wait
 * that ran out (IFC_TIMEOUT), an index out of range in the bounds-checked
 * build -- is reported by the next ifc_sync. */
int ifc_run_stage_async(ifc_solver *h, int stage);

/* ifc_sweep without norms (n sweeps as one cooperative launch where the
 * handle has one), enqueued without waiting; outcome at the next ifc_sync. */
int ifc_sweep_async(ifc_solver *h, int eq, int n);

/* Wait for the handle's stream and report what its launches left in the
 * control block (IFC_OK, IFC_TIMEOUT, IFC_BAD_ARGUMENT). */
int ifc_sync(ifc_solver *h);

/* n sweeps of one equation (0=u 1=v 2=w 3=p') with the coefficients and
 * sources currently materialised by IFC_STAGE_MOM_ASSEMBLE / PCORR_COEF;
 * sq_norms (optional, n entries) receives sum (d phi)^2 of each sweep.  With
 * sq_norms NULL the n Gauss-Seidel sweeps run as one cooperative launch on
 * the stored planes where the handle has one (2D; 3D when its p' solve is
 * cooperative), else back to back, and the call waits for the device once. */
int ifc_sweep(ifc_solver *h, int eq, int n, double *sq_norms);

/* Average device time (ms, CUDA events on the handle's stream) of one launch
 * sequence of a stage, over reps back-to-back repetitions on the current state;
 * *launches receives the kernels one repetition launches.  For profiling. */
int ifc_time_stage(ifc_solver *h, int stage, int reps, double *ms, int *launches);

/* Norms of the last outer iteration and the running maxima (see ifc_stats). */
int ifc_get_stats(ifc_solver *h, ifc_stats *stats);

/* Red-black Gauss-Seidel sweeps on caller-owned device buffers, allocating
 * nothing.  No counterpart in the reference: it exists for callers that cannot
 * call cudaMalloc -- a program that reserved the whole device for its own pool,
 * or a time-critical loop that cannot afford cudaFree (it synchronises the
 * device).  Runs the same sweep kernel as ifc_sweep: coef holds 2*dim+1
 * planes coef[cell + N*slot] (slots aC,aE,aW,aN,aS[,aT,aB]), src and phi N
 * cells, all device pointers in the precision given (IFC_FP32 or IFC_FP64);
 * phi is updated in place by n_sweeps sweeps relaxed by `relax`, with no inner
 * early exit; sq_norms (optional host array, n_sweeps entries) receives the
 * FP64 sum of squared changes of each sweep.  stream: cudaStream_t or NULL.
 * Scratch comes from a fixed 152 KB array inside the library, held on every
 * GPU that loads it until the process exits.  Grids above 2^26 cells are
 * rejected with IFC_BAD_ARGUMENT and a message on stderr.  Every call looks
 * the array's address up on the current device (cudaGetSymbolAddress), so a
 * device reset between calls is safe; make the first call on a device before
 * any stream capture, since it may load the module.  All calls share the
 * array, so calls that
 * overlap on the GPU (from several streams or threads) race.  Returns when
 * the sweeps are done. */
int ifc_rb_sweeps_noalloc(int dim, int nx, int ny, int nz, int precision, const void *coef, const void *src,
                          void *phi, double relax, int n_sweeps, double *sq_norms, void *stream);

const char *ifc_status_string(int status);
const char *ifc_last_error(const ifc_solver *h);
int ifc_abi_version(void);
/* Build options of the loaded library (an addition; the reference has one
 * build): IFC_BUILD_BOUNDS_CHECK when it was compiled with IFC_BOUNDS_CHECK,
 * whose kernels check every field-array index and report an out-of-range
 * one as IFC_BAD_ARGUMENT instead of touching the memory. */
enum { IFC_BUILD_BOUNDS_CHECK = 1 };
int ifc_build_flags(void);

#ifdef __cplusplus
}
#endif

#endif
