// ifc_solver.cu -- C ABI of the solver (include/ifc.h).  Every entry point
// validates its arguments, catches C++ exceptions and returns a status code;
// the reference has no error reporting at all (its defect D11).
#include <cstring>
#include <new>

#include <nvtx3/nvToolsExt.h>

#include "ifc.h"
#include "ifc_engine.cuh"

using ifc::EngineBase;

// NVTX range around a C ABI call, so timeline profilers show the library's
// stages (solve, iterate, adjoint, VTK output) by name.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

struct ifc_solver {
    ifc_config cfg;
    EngineBase *eng;
    std::string err;
};

#include "ifc_fused2d_impl.cuh"

extern "C" {

int ifc_abi_version(void) { return IFC_ABI_VERSION; }

int ifc_build_flags(void)
{
#ifdef IFC_BOUNDS_CHECK
    return IFC_BUILD_BOUNDS_CHECK;
#else
    return 0;
#endif
}

const char *ifc_status_string(int s)
{
    switch (s) {
    case IFC_OK: return "ok";
    case IFC_NOT_CONVERGED: return "not converged";
    case IFC_DIVERGED: return "diverged";
    case IFC_TIMEOUT: return "timeout";
    case IFC_CUDA_ERROR: return "CUDA error";
    case IFC_BAD_CONFIG: return "bad configuration";
    case IFC_BAD_ARGUMENT: return "bad argument";
    case IFC_IO_ERROR: return "I/O error";
    case IFC_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
    }
}

// include/config.h:6-81 as shipped by the reference.
int ifc_config_default(ifc_config *c)
{
    if (!c) return IFC_BAD_ARGUMENT;
    std::memset(c, 0, sizeof(*c));
    c->dim = 2;
    c->nx = 1024;
    c->ny = 256;
    c->nz = 1;
    c->xmin = -2; c->xmax = 2; c->ymin = -0.5; c->ymax = 0.5; c->zmin = 0.0; c->zmax = 1.0;
    c->thermal_conductivity = 1;
    c->specific_heat_capacity = 1;
    c->density = 50;
    c->dynamic_viscosity = 1;
    const int vt[6] = {IFC_OUTLET, IFC_INLET, IFC_WALL, IFC_WALL, IFC_WALL, IFC_WALL};
    for (int f = 0; f < 6; ++f) c->vel_bc_type[f] = vt[f];
    c->vel_bc_val[IFC_WEST][0] = 1;
    const int tt[6] = {1, 1, 0, 0, 1, 1};
    const double tv[6] = {0.0, 0.0, 293.0, 373.0, 0.0, 0.0};
    for (int f = 0; f < 6; ++f) { c->temp_bc_type[f] = tt[f]; c->temp_bc_val[f] = tv[f]; }
    c->num_outer_iter = 20000;
    c->n_iter_u = 10; c->n_iter_v = 10; c->n_iter_w = 10; c->n_iter_p = 20;
    c->relax_u = 0.75; c->relax_v = 0.75; c->relax_w = 0.75; c->relax_p = 0.25;
    c->tol_u = 1e-5; c->tol_v = 1e-5; c->tol_w = 1e-5; c->tol_p = 1e-3; c->tol_mass = 1e-9;
    c->precision = IFC_FP32;
    c->linear_solver = IFC_GAUSS_SEIDEL;
    c->criterion = IFC_CRIT_PER_FIELD;
    c->pin_pressure = -1;
    c->sweeps_per_pass = 0;
    c->log_level = 0;
    c->inlet_profile = nullptr;
    c->stream = nullptr;
    c->convection_scheme = IFC_CONV_UPWIND;
    return IFC_OK;
}

int ifc_config_check(const ifc_config *c)
{
    if (!c) return IFC_BAD_ARGUMENT;
    if (c->dim != 2 && c->dim != 3) return IFC_BAD_CONFIG;
    const int nz = c->dim == 2 ? 1 : c->nz;
    if (c->nx < 3 || c->ny < 3 || (c->dim == 3 && nz < 3)) return IFC_BAD_CONFIG;
    if ((double)c->nx * c->ny * nz > (double)(1 << 28)) return IFC_BAD_CONFIG;
    if (!(c->xmax > c->xmin) || !(c->ymax > c->ymin) || !(c->zmax > c->zmin)) return IFC_BAD_CONFIG;
    for (int f = 0; f < 6; ++f)
        if (c->vel_bc_type[f] < IFC_WALL || c->vel_bc_type[f] > IFC_OUTLET) return IFC_BAD_CONFIG;
    if (c->num_outer_iter < 0 || c->n_iter_u < 0 || c->n_iter_v < 0 || c->n_iter_w < 0 || c->n_iter_p < 0)
        return IFC_BAD_CONFIG;
    if (c->n_iter_u > 100000 || c->n_iter_v > 100000 || c->n_iter_w > 100000 || c->n_iter_p > 100000)
        return IFC_BAD_CONFIG;
    if (c->precision != IFC_FP32 && c->precision != IFC_FP64) return IFC_BAD_CONFIG;
    if (c->linear_solver != IFC_GAUSS_SEIDEL && c->linear_solver != IFC_JACOBI) return IFC_BAD_CONFIG;
    if (c->criterion != IFC_CRIT_REFERENCE && c->criterion != IFC_CRIT_PER_FIELD && c->criterion != IFC_CRIT_RESIDUAL)
        return IFC_BAD_CONFIG;
    if (c->pin_pressure < -1 || c->pin_pressure > 1) return IFC_BAD_CONFIG;
    if (c->sweeps_per_pass < 0 || c->sweeps_per_pass > 16) return IFC_BAD_CONFIG;
    if (c->convection_scheme < IFC_CONV_UPWIND || c->convection_scheme > IFC_CONV_VAN_LEER) return IFC_BAD_CONFIG;
    if (c->slab_axis_cells != 0 && c->slab_axis_cells < (c->dim == 2 ? c->ny : nz)) return IFC_BAD_CONFIG;
    return IFC_OK;
}

int ifc_create(const ifc_config *cfg, ifc_solver **out)
{
    if (!cfg || !out) return IFC_BAD_ARGUMENT;
    *out = nullptr;
    int rc = ifc_config_check(cfg);
    if (rc != IFC_OK) return rc;
    ifc_solver *h = new (std::nothrow) ifc_solver;
    if (!h) return IFC_CUDA_ERROR;
    h->cfg = *cfg;
    if (h->cfg.dim == 2) h->cfg.nz = 1;
    h->eng = nullptr;
    try {
        if (cfg->precision == IFC_FP64) {
            auto *e = new ifc::Engine<double>();
            h->eng = e;
            rc = e->init(h->cfg);
        } else {
            auto *e = new ifc::Engine<float>();
            h->eng = e;
            rc = e->init(h->cfg);
        }
    } catch (const std::exception &ex) {
        h->err = ex.what();
        rc = IFC_CUDA_ERROR;
    }
    if (rc != IFC_OK) {
        delete h->eng;
        delete h;
        return rc;
    }
    *out = h;
    return IFC_OK;
}

int ifc_destroy(ifc_solver *h)
{
    if (!h) return IFC_OK;
    delete h->eng;
    delete h;
    return IFC_OK;
}

#define IFC_GUARD(h)                             \
    if (!(h) || !(h)->eng) return IFC_BAD_ARGUMENT; \
    try {
#define IFC_END(h)                               \
    }                                            \
    catch (const std::exception &ex) {           \
        (h)->eng->err = ex.what();               \
        return IFC_CUDA_ERROR;                   \
    }

int ifc_set_uniform(ifc_solver *h, double u, double v, double w, double p, double temp)
{
    IFC_GUARD(h)
    return h->eng->set_uniform(u, v, w, p, temp);
    IFC_END(h)
}

int ifc_set_field(ifc_solver *h, int field, const void *host, size_t bytes)
{
    IFC_GUARD(h)
    return h->eng->set_field(field, host, bytes);
    IFC_END(h)
}

int ifc_get_field(ifc_solver *h, int field, void *host, size_t bytes)
{
    IFC_GUARD(h)
    return h->eng->get_field(field, host, bytes);
    IFC_END(h)
}

size_t ifc_field_size(const ifc_solver *h, int field)
{
    if (!h || !h->eng) return 0;
    return h->eng->field_size(field);
}

int ifc_device_ptr(ifc_solver *h, int field, void **dptr)
{
    if (!dptr) return IFC_BAD_ARGUMENT;
    IFC_GUARD(h)
    *dptr = h->eng->device_ptr(field);
    return *dptr ? IFC_OK : IFC_BAD_ARGUMENT;
    IFC_END(h)
}

int ifc_solve(ifc_solver *h, ifc_stats *stats)
{
    NvtxRange r("ifc_solve");
    IFC_GUARD(h)
    return h->eng->run(h->cfg.num_outer_iter, 1, stats);
    IFC_END(h)
}

int ifc_iterate(ifc_solver *h, int n_outer, ifc_stats *stats)
{
    NvtxRange r("ifc_iterate");
    IFC_GUARD(h)
    return h->eng->run(n_outer, 0, stats);
    IFC_END(h)
}

int ifc_run_stage(ifc_solver *h, int stage)
{
    IFC_GUARD(h)
    return h->eng->run_stage(stage);
    IFC_END(h)
}

int ifc_run_stage_async(ifc_solver *h, int stage)
{
    IFC_GUARD(h)
    return h->eng->run_stage_async(stage);
    IFC_END(h)
}

int ifc_sweep_async(ifc_solver *h, int eq, int n)
{
    IFC_GUARD(h)
    return h->eng->sweep_async(eq, n);
    IFC_END(h)
}

int ifc_sync(ifc_solver *h)
{
    IFC_GUARD(h)
    return h->eng->sync();
    IFC_END(h)
}

int ifc_sweep(ifc_solver *h, int eq, int n, double *sq_norms)
{
    IFC_GUARD(h)
    return h->eng->sweep(eq, n, sq_norms);
    IFC_END(h)
}

int ifc_time_stage(ifc_solver *h, int stage, int reps, double *ms, int *launches)
{
    IFC_GUARD(h)
    return h->eng->time_stage(stage, reps, ms, launches);
    IFC_END(h)
}

int ifc_solve_energy(ifc_solver *h, int max_sweeps, double tol, ifc_energy_result *result)
{
    NvtxRange r("ifc_solve_energy");
    IFC_GUARD(h)
    ifc_energy_result tmp;
    const int rc = h->eng->solve_energy(max_sweeps, tol, result ? result : &tmp);
    if (result) result->status = rc;
    return rc;
    IFC_END(h)
}

int ifc_set_inlet_profile(ifc_solver *h, const double *profile)
{
    IFC_GUARD(h)
    return h->eng->set_inlet(profile);
    IFC_END(h)
}

int ifc_adjoint(ifc_solver *h, int objective, const double *dJ_du, const double *dJ_dv, const double *dJ_dp,
                int max_iter, double tol, double *dJ_dtheta, ifc_adjoint_result *result)
{
    NvtxRange nr("ifc_adjoint");
    if (objective != IFC_OBJ_PRESSURE_DROP && objective != IFC_OBJ_CUSTOM) return IFC_BAD_ARGUMENT;
    if (max_iter < 1 || !(tol >= 0.0)) return IFC_BAD_ARGUMENT;
    IFC_GUARD(h)
    ifc::AdjointReq rq;
    std::memset(&rq, 0, sizeof(rq));
    rq.mode = 0;
    rq.objective = objective;
    rq.seed[0] = dJ_du;
    rq.seed[1] = dJ_dv;
    rq.seed[2] = dJ_dp;
    rq.max_iter = max_iter;
    rq.tol = tol;
    rq.dtheta = dJ_dtheta;
    ifc_adjoint_result r;
    std::memset(&r, 0, sizeof(r));
    const int rc = h->eng->adjoint(rq, &r);
    r.status = rc;
    if (result) *result = r;
    return rc;
    IFC_END(h)
}

int ifc_adjoint_apply(ifc_solver *h, const double *lam_u, const double *lam_v, const double *lam_p,
                      const double *lam_uf, const double *lam_vf, double *out_u, double *out_v, double *out_p,
                      double *out_uf, double *out_vf, double *dJ_dtheta, double *dJ_dmu)
{
    IFC_GUARD(h)
    ifc::AdjointReq rq;
    std::memset(&rq, 0, sizeof(rq));
    rq.mode = 1;
    const double *in[5] = {lam_u, lam_v, lam_p, lam_uf, lam_vf};
    double *out[5] = {out_u, out_v, out_p, out_uf, out_vf};
    for (int q = 0; q < 5; ++q) {
        rq.seed[q] = in[q];
        rq.out[q] = out[q];
    }
    rq.max_iter = 1;
    rq.dtheta = dJ_dtheta;
    rq.dmu = dJ_dmu;
    return h->eng->adjoint(rq, nullptr);
    IFC_END(h)
}

int ifc_get_stats(ifc_solver *h, ifc_stats *stats)
{
    IFC_GUARD(h)
    return h->eng->stats(stats);
    IFC_END(h)
}

static int write_vtk_any(ifc_solver *h, const char *path, bool binary)
{
    IFC_GUARD(h)
    const size_t bytes = h->eng->field_size(IFC_FIELD_U);
    std::vector<char> u(bytes), v(bytes), w(bytes), p(bytes), t(bytes);
    int rc;
    if ((rc = h->eng->get_field(IFC_FIELD_U, u.data(), bytes)) != IFC_OK) return rc;
    if ((rc = h->eng->get_field(IFC_FIELD_V, v.data(), bytes)) != IFC_OK) return rc;
    if ((rc = h->eng->get_field(IFC_FIELD_W, w.data(), bytes)) != IFC_OK) return rc;
    if ((rc = h->eng->get_field(IFC_FIELD_P, p.data(), bytes)) != IFC_OK) return rc;
    if ((rc = h->eng->get_field(IFC_FIELD_T, t.data(), bytes)) != IFC_OK) return rc;
    return binary ? ifc_write_vtk_binary_host(&h->cfg, u.data(), v.data(), w.data(), p.data(), t.data(), path)
                  : ifc_write_vtk_host(&h->cfg, u.data(), v.data(), w.data(), p.data(), t.data(), path);
    IFC_END(h)
}

int ifc_write_vtk(ifc_solver *h, const char *path)
{
    NvtxRange r("ifc_write_vtk");
    if (!path) return IFC_BAD_ARGUMENT;
    return write_vtk_any(h, path, false);
}

int ifc_write_vtk_binary(ifc_solver *h, const char *path)
{
    NvtxRange r("ifc_write_vtk_binary");
    if (!path) return IFC_BAD_ARGUMENT;
    return write_vtk_any(h, path, true);
}

const char *ifc_last_error(const ifc_solver *h)
{
    if (!h) return "null handle";
    if (h->eng && !h->eng->err.empty()) return h->eng->err.c_str();
    return h->err.c_str();
}

}  // extern "C"
