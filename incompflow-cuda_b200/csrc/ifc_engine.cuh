// ifc_engine.cuh -- host-side engine of one solver handle: device buffers, the
// SIMPLE outer iteration as a CUDA graph with a device-side loop condition
// (conditional WHILE node), single-step launches for testing, and host
// transfers.  Replaces the reference's Solver members (src/Solver.cu:13-966).
#pragma once

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "ifc.h"
#include "ifc_adjoint.h"
#include "ifc_kernels.cuh"
#include "ifc_persist2d.cuh"
#include "ifc_fused3d.cuh"
#include "ifc_coop3d.cuh"
#include "ifc_energy.cuh"

namespace ifc {

struct EngineBase {
    virtual ~EngineBase() {}
    virtual int set_uniform(double u, double v, double w, double p, double t) = 0;
    virtual int set_field(int field, const void *host, size_t bytes) = 0;
    virtual int get_field(int field, void *host, size_t bytes) = 0;
    virtual size_t field_size(int field) const = 0;
    virtual void *device_ptr(int field) = 0;
    virtual int run(int n_outer, int act, ifc_stats *st) = 0;
    virtual int run_stage(int stage) = 0;
    virtual int run_stage_async(int stage) = 0;
    virtual int sync() = 0;
    virtual int sweep(int eq, int n, double *sq) = 0;
    virtual int sweep_async(int eq, int n) = 0;
    virtual int stats(ifc_stats *st) = 0;
    virtual int time_stage(int stage, int reps, double *ms, int *launches) = 0;
    virtual int adjoint(const AdjointReq &rq, ifc_adjoint_result *res) = 0;
    virtual int set_inlet(const double *profile) = 0;
    virtual int solve_energy(int max_sweeps, double tol, ifc_energy_result *res) = 0;
    std::string err;
};

#define IFC_CK(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            return IFC_CUDA_ERROR;                                                        \
        }                                                                                 \
    } while (0)

// Geometry and constants in the scalar type, evaluated like the reference's
// constexpr expressions (include/constants.h:22-28, include/config.h).
template <typename T>
Params<T> make_params(const ifc_config &c)
{
    Params<T> P;
    std::memset(&P, 0, sizeof(P));
    Geo<T> &g = P.g;
    g.dim = c.dim;
    g.nx = c.nx;
    g.ny = c.ny;
    g.nz = c.dim == 2 ? 1 : c.nz;
    g.N = g.nx * g.ny * g.nz;
    const T xmax = (T)c.xmax, xmin = (T)c.xmin, ymax = (T)c.ymax, ymin = (T)c.ymin;
    const T zmax = (T)c.zmax, zmin = (T)c.zmin;
    g.dx = (xmax - xmin) / (T)g.nx;
    // A slab handle takes the whole grid's spacing along its cut axis.
    const int sy = (c.slab_axis_cells > 0 && c.dim == 2) ? c.slab_axis_cells : g.ny;
    const int sz = (c.slab_axis_cells > 0 && c.dim == 3) ? c.slab_axis_cells : g.nz;
    g.dy = (ymax - ymin) / (T)sy;
    g.dz = (zmax - zmin) / (T)sz;
    g.Ax = g.dy * g.dz;
    g.Ay = g.dz * g.dx;
    g.Az = g.dx * g.dy;
    g.rho = (T)c.density;
    g.mu = (T)c.dynamic_viscosity;
    const double rl[4] = {c.relax_u, c.relax_v, c.relax_w, c.relax_p};
    const double tl[4] = {c.tol_u, c.tol_v, c.tol_w, c.tol_p};
    for (int q = 0; q < 4; ++q) {
        g.relax[q] = (T)rl[q];
        g.tol[q] = (double)(T)tl[q];
    }
    g.tol_mass = (double)(T)c.tol_mass;
    for (int f = 0; f < 6; ++f) {
        g.bc[f] = c.vel_bc_type[f];
        g.closed[f] = c.vel_bc_type[f] != IFC_OUTLET;
        for (int q = 0; q < 3; ++q) g.bcv[f][q] = (T)c.vel_bc_val[f][q];
    }
    g.inlet = nullptr;
    g.criterion = c.criterion == IFC_CRIT_REFERENCE ? 0 : c.criterion == IFC_CRIT_RESIDUAL ? 2 : 1;
    g.conv = c.convection_scheme;
    Derived<T> &d = P.d;
    d.Dx = g.mu * g.Ax / g.dx;
    d.Dy = g.mu * g.Ay / g.dy;
    d.Dz = g.mu * g.Az / g.dz;
    const double rho = (double)g.rho;
    d.Kx = -0.5 * rho * (double)g.Ax * (double)g.Ax;
    d.Ky = -0.5 * rho * (double)g.Ay * (double)g.Ay;
    d.Kz = -0.5 * rho * (double)g.Az * (double)g.Az;
    for (int q = 0; q < 3; ++q) d.ru[q] = (double)g.relax[q] * 0.5;
    d.c83 = (T)8 / (T)3;
    return P;
}

template <typename T>
struct Engine : EngineBase {
    ifc_config cfg;
    Params<T> P;
    Fields<T> f;
    Ctl *ctl = nullptr;
    double *partials = nullptr;
    T *inlet_d = nullptr;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nsm = 148;
    int max_grid = 148 * 8;
    int dim = 2;
    bool pin = false;
    bool fused = false;               // 2D temporally blocked kernels
    int spp_mom = 5, spp_p = 5;       // sweeps per pass of the fused kernels
    int spp_persist = 5;              // sweeps per pass of the single-launch solve
    bool persist = false;             // the whole loop runs as one cooperative launch
    bool persist_mt = false;          // ... with several tiles per CTA
    int persist_grid = 0;             // CTAs of that launch
    GridBarrier *barrier = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t body_graph = nullptr;
    cudaGraphExec_t body_exec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<void *> allocs;
    Ctl ctl_h;
    double last_ms = 0.0;
    long long launches = 0;           // kernels enqueued (counted by the enq_* helpers)
    long long launches_per_iter = 0;  // kernels in one captured outer iteration
    long long last_launches = 0;
    AdjointCtx *adj = nullptr;        // discrete-adjoint buffers and graphs (first ifc_adjoint call)
    // The 3D p' solve as one cooperative launch (ifc_coop3d.cuh): row blocks,
    // shared memory per CTA, and the packed links and sources
    static constexpr int kPcNT = 1024;
    bool pc3d = false;
    PcBlocks pcb = {0, 0, 0, 0};
    size_t pc3d_smem = 0;
    T *packed = nullptr;
    // The 3D momentum coefficients and sources of one solve, packed by the
    // first sweep (k_mom_half3d<T, true>): 10 values per slot
    T *mpk = nullptr;
    long long mpk_slots = 0;

    ~Engine() override
    {
        adjoint_free(adj);
        destroy_graphs();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamSynchronize(stream);
        for (void *p : allocs) cudaFree(p);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    // Blocks of 256 threads for the row-segment kernels (one warp per unit).
    int row_grid() const { return grid(32LL * row_units(P.g.nx, P.g.ny * P.g.nz)); }

    // At most one resident wave of kernel `kern` (256 threads, no dynamic
    // shared memory): the grid-stride kernels then run without a partial
    // second wave, and their last-block reduction sums fewer partials.
    // IFC_WAVE_GRID=0 keeps the plain sizing (A/B timing).
    std::vector<std::pair<const void *, int>> wave_cap;
    int wave_off = -1;  // IFC_WAVE_GRID, read at the handle's first launch
    int wave_grid(const void *kern, int blocks)
    {
        if (wave_off < 0) {
            const char *e = std::getenv("IFC_WAVE_GRID");
            wave_off = (e && e[0] == '0') ? 1 : 0;
        }
        if (wave_off) return blocks;
        int cap = -1;
        for (auto &kv : wave_cap)
            if (kv.first == kern) cap = kv.second;
        if (cap < 0) {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0) != cudaSuccess) {
                cudaGetLastError();
                per_sm = 0;
            }
            cap = per_sm * nsm;
            wave_cap.push_back({kern, cap});
        }
        return cap > 0 && cap < blocks ? cap : blocks;
    }

    int grid(long long work) const
    {
        long long b = (work + 255) / 256;
        if (b < 1) b = 1;
        if (b > max_grid) b = max_grid;
        return (int)b;
    }

#ifdef IFC_BOUNDS_CHECK
    template <typename U>
    int alloc(Checked<U> *p, size_t n)
    {
        U *q = nullptr;
        int rc = alloc(&q, n);
        p->p = q;
        p->n = (long long)n;
        return rc;
    }

    // IFC_BAD_ARGUMENT when a kernel of the last launch sequence indexed a
    // field array out of range (the flag is then cleared).
    int bounds_status()
    {
        int e = 0;
        unsigned long long idx = 0;
        IFC_CK(cudaMemcpyFromSymbol(&e, g_ifc_bounds_err, sizeof(int)));
        if (!e) return IFC_OK;
        IFC_CK(cudaMemcpyFromSymbol(&idx, g_ifc_bounds_idx, sizeof(idx)));
        const int zero = 0;
        IFC_CK(cudaMemcpyToSymbol(g_ifc_bounds_err, &zero, sizeof(int)));
        err = "bounds check: a kernel indexed a field array out of range (index " +
              std::to_string((long long)idx) + ")";
        return IFC_BAD_ARGUMENT;
    }
#else
    int bounds_status() { return IFC_OK; }
#endif

    template <typename U>
    int alloc(U **p, size_t n)
    {
        void *q = nullptr;
        IFC_CK(cudaMalloc(&q, n * sizeof(U) > 0 ? n * sizeof(U) : 16));
        allocs.push_back(q);
        *p = (U *)q;
        return IFC_OK;
    }

    size_t nface(int which) const
    {
        const Geo<T> &g = P.g;
        if (which == 0) return (size_t)(g.nx + 1) * g.ny * g.nz;
        if (which == 1) return (size_t)g.nx * (g.ny + 1) * g.nz;
        return (size_t)g.nx * g.ny * (g.nz + 1);
    }

    int init(const ifc_config &c)
    {
        cfg = c;
        P = make_params<T>(c);
        dim = P.g.dim;
        const size_t N = (size_t)P.g.N, nc = (size_t)(2 * dim + 1);
        int dev = 0;
        IFC_CK(cudaGetDevice(&dev));
        IFC_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        max_grid = nsm * 8;
        if (c.stream) {
            stream = (cudaStream_t)c.stream;
        } else {
            IFC_CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
            own_stream = true;
        }
        IFC_CK(cudaEventCreate(&ev0));
        IFC_CK(cudaEventCreate(&ev1));
        std::memset(&f, 0, sizeof(f));
        int rc;
#define A_(ptr, n) if ((rc = alloc(&(ptr), (n))) != IFC_OK) return rc
        A_(f.u, N); A_(f.v, N); A_(f.w, N); A_(f.p, N); A_(f.temp, N); A_(f.pc, N);
        A_(f.uf, nface(0)); A_(f.vf, nface(1)); A_(f.wf, nface(2));
        A_(f.ac, N); A_(f.mc, N * nc); A_(f.pcoef, N * nc);
        A_(f.su, N); A_(f.sv, N); A_(f.sw, N); A_(f.sp, N); A_(f.tmp, 3 * N); A_(f.rac, N);
        if (c.convection_scheme != IFC_CONV_UPWIND) A_(f.sdc, (size_t)dim * N);
        if (dim == 3 && c.linear_solver == IFC_GAUSS_SEIDEL) {
            mpk_slots = (long long)P.g.ny * P.g.nz * 2 * ((P.g.nx + 1) / 2);
            A_(mpk, (size_t)mpk_slots * 10);
        }
        // One FP64 partial per value and block: the grid-stride kernels use at
        // most max_grid blocks, the tiled 2D kernels one block per 32x8 tile.
        const size_t tiles = (size_t)((P.g.nx + 31) / 32) * (size_t)((P.g.ny + 7) / 8) * (size_t)P.g.nz;
        const size_t max_blocks = tiles > (size_t)max_grid ? tiles : (size_t)max_grid;
        A_(partials, max_blocks * kMaxReduce);
        A_(ctl, 1);
        A_(barrier, 1);
#undef A_
        if (c.inlet_profile) {
            const size_t n = (size_t)P.g.ny * P.g.nz;
            std::vector<T> h(n);
            for (size_t q = 0; q < n; ++q) h[q] = (T)c.inlet_profile[q];
            if ((rc = alloc(&inlet_d, n)) != IFC_OK) return rc;
            IFC_CK(cudaMemcpy(inlet_d, h.data(), n * sizeof(T), cudaMemcpyHostToDevice));
            P.g.inlet = inlet_d;
        }
        bool closed = true;
        for (int q = 0; q < 2 * dim; ++q) closed = closed && c.vel_bc_type[q] != IFC_OUTLET;
        pin = c.pin_pressure == 1 || (c.pin_pressure < 0 && closed);
        fused = (dim == 2) && fused2d_supported<T>(P.g);
        if (c.sweeps_per_pass > 0) spp_mom = spp_p = spp_persist = c.sweeps_per_pass;
        if (fused && (rc = prepare_fused()) != IFC_OK) return rc;
        if ((rc = prepare_persist()) != IFC_OK) return rc;
        if (dim == 3 && c.linear_solver == IFC_GAUSS_SEIDEL && (rc = prepare_pc3d()) != IFC_OK) return rc;
        if ((rc = set_uniform(0.0, 0.0, 0.0, 0.0, 273.0)) != IFC_OK) return rc;
        if ((rc = build_graph()) != IFC_OK && pc3d) {
            // the cooperative p' launch could not be captured: per-half-sweep kernels
            cudaGetLastError();
            destroy_graphs();
            pc3d = false;
            rc = build_graph();
        }
        return rc;
    }

    void destroy_graphs()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (body_exec) cudaGraphExecDestroy(body_exec);
        if (body_graph) cudaGraphDestroy(body_graph);
        exec = nullptr;
        graph = nullptr;
        body_exec = nullptr;
        body_graph = nullptr;
        cond = 0;
    }

    // Row blocks of the cooperative 3D p' solve: the smallest blocks (fewest
    // rows, then the shortest perimeter) whose count fits one CTA per SM and
    // whose p' fits the CTA's shared memory.  IFC_PC3D_OFF=1 keeps the
    // per-half-sweep kernel (A/B timing, tests).
    int prepare_pc3d()
    {
        pc3d = false;
        const char *off = std::getenv("IFC_PC3D_OFF");
        if (off && off[0] == '1') return IFC_OK;
        int dev = 0, optin = 0, coop = 0;
        IFC_CK(cudaGetDevice(&dev));
        IFC_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        IFC_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        if (!coop) return IFC_OK;
        const int nx = P.g.nx, ny = P.g.ny, nz = P.g.nz;
        const size_t per_row = sizeof(T) * (size_t)(2 * ((nx + 1) / 2)) + 20;  // p' and the row table
        const long long max_rows = ((long long)optin - 4096) / (long long)per_row;
        if (max_rows < 1) return IFC_OK;
        long long best = -1, best_per = 0;
        PcBlocks b = {0, 0, 0, 0};
        for (int bj = 1; bj <= ny; ++bj)
            for (int bk = 1; bk <= nz && (long long)bj * bk <= max_rows; ++bk) {
                const int nbj = (ny + bj - 1) / bj, nbk = (nz + bk - 1) / bk;
                if ((long long)nbj * nbk > nsm) continue;
                const long long rows = (long long)bj * bk, per = bj + bk;
                if (best < 0 || rows < best || (rows == best && per < best_per)) {
                    best = rows;
                    best_per = per;
                    b = {bj, bk, nbj, nbk};
                }
            }
        if (best < 0) return IFC_OK;
        const size_t smem = coop3d_smem_bytes<T>(b.bj * b.bk, nx);
        auto kern = k_csolve3d<T, kPcNT>;
        // The limit is one setting of the kernel shared by every handle of
        // the process, whose blocks need different amounts: set it to the
        // device's maximum (less the kernel's static shared memory), so no
        // handle lowers it below another's launch.
        cudaFuncAttributes fa;
        IFC_CK(cudaFuncGetAttributes(&fa, kern));
        const int dyn_max = optin - (int)fa.sharedSizeBytes;
        if ((long long)smem > dyn_max) return IFC_OK;
        IFC_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max));
        int per_sm = 0;
        IFC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPcNT, smem));
        if (per_sm < 1 || (long long)per_sm * nsm < (long long)b.nbj * b.nbk) return IFC_OK;
        int rc = alloc(&packed, (size_t)coop3d_slots(b, nx) * 8);
        if (rc != IFC_OK) return rc;
        pcb = b;
        pc3d_smem = smem;
        pc3d = true;
        return IFC_OK;
    }

    // The p' solve (sys.coef null) or a stored-coefficient system as one
    // cooperative launch of n sweeps (k_csolve3d).
    void enq_csolve3d(const Params<T> &PP, CSys<T> sys, int n)
    {
        cudaMemsetAsync(barrier, 0, sizeof(GridBarrier), stream);
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(pcb.nbj * pcb.nbk);
        lc.blockDim = dim3(kPcNT);
        lc.dynamicSmemBytes = pc3d_smem;
        lc.stream = stream;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        lc.attrs = at;
        lc.numAttrs = 1;
        const char *stall_env = std::getenv("IFC_TEST_STALL_BARRIER");  // failure-detection test, per launch
        const int stall = (stall_env && stall_env[0] == '1') ? 1 : 0;
        cudaLaunchKernelEx(&lc, k_csolve3d<T, kPcNT>, PP, f, ctl, partials, barrier, pcb, n, packed, sys, stall);
        ++launches;
    }

    void enq_pc_solve3d()
    {
        CSys<T> sys = {nullptr, f.sp, f.pc, EQ_P};
        enq_csolve3d(P, sys, cfg.n_iter_p);
    }

    int set_uniform(double u, double v, double w, double p, double t) override
    {
        const long long N = P.g.N;
        const int G = grid(N);
        k_fill<T><<<G, 256, 0, stream>>>(f.u, N, (T)u);
        k_fill<T><<<G, 256, 0, stream>>>(f.v, N, (T)v);
        k_fill<T><<<G, 256, 0, stream>>>(f.w, N, (T)w);
        k_fill<T><<<G, 256, 0, stream>>>(f.p, N, (T)p);
        k_fill<T><<<G, 256, 0, stream>>>(f.temp, N, (T)t);
        const size_t nc = (size_t)(2 * dim + 1);
        IFC_CK(cudaMemsetAsync(f.pc, 0, N * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.uf, 0, nface(0) * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.vf, 0, nface(1) * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.wf, 0, nface(2) * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.ac, 0, N * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.mc, 0, N * nc * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.pcoef, 0, N * nc * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.su, 0, N * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.sv, 0, N * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.sw, 0, N * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(f.sp, 0, N * sizeof(T), stream));
        IFC_CK(cudaMemsetAsync(ctl, 0, sizeof(Ctl), stream));
        IFC_CK(cudaGetLastError());
        IFC_CK(cudaStreamSynchronize(stream));
        return IFC_OK;
    }

    T *field_ptr(int field) const
    {
        switch (field) {
        case IFC_FIELD_U: return f.u;
        case IFC_FIELD_V: return f.v;
        case IFC_FIELD_W: return f.w;
        case IFC_FIELD_P: return f.p;
        case IFC_FIELD_T: return f.temp;
        case IFC_FIELD_PCORR: return f.pc;
        case IFC_FIELD_UF: return f.uf;
        case IFC_FIELD_VF: return f.vf;
        case IFC_FIELD_WF: return f.wf;
        case IFC_FIELD_MOM_AC: return f.ac;
        case IFC_FIELD_MOM_COEF: return f.mc;
        case IFC_FIELD_PCORR_COEF: return f.pcoef;
        case IFC_FIELD_SRC_U: return f.su;
        case IFC_FIELD_SRC_V: return f.sv;
        case IFC_FIELD_SRC_W: return f.sw;
        case IFC_FIELD_SRC_P: return f.sp;
        default: return nullptr;
        }
    }

    size_t field_size(int field) const override
    {
        const size_t N = (size_t)P.g.N;
        switch (field) {
        case IFC_FIELD_UF: return nface(0) * sizeof(T);
        case IFC_FIELD_VF: return nface(1) * sizeof(T);
        case IFC_FIELD_WF: return nface(2) * sizeof(T);
        case IFC_FIELD_MOM_COEF:
        case IFC_FIELD_PCORR_COEF: return N * (size_t)(2 * dim + 1) * sizeof(T);
        default: return field_ptr(field) ? N * sizeof(T) : 0;
        }
    }

    void *device_ptr(int field) override { return field_ptr(field); }

    int set_field(int field, const void *host, size_t bytes) override
    {
        T *d = field_ptr(field);
        if (!d || !host || bytes != field_size(field)) {
            err = "set_field: bad field id, pointer or size";
            return IFC_BAD_ARGUMENT;
        }
        IFC_CK(cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        return IFC_OK;
    }

    int get_field(int field, void *host, size_t bytes) override
    {
        T *d = field_ptr(field);
        if (!d || !host || bytes != field_size(field)) {
            err = "get_field: bad field id, pointer or size";
            return IFC_BAD_ARGUMENT;
        }
        IFC_CK(cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        return IFC_OK;
    }

    // ---- enqueue helpers (no synchronisation; usable under stream capture) ----
    template <int DIM>
    void enq_face_bc()
    {
        const long long nf = (long long)nface(0) + nface(1) + (DIM == 3 ? (long long)nface(2) : 0);
        k_face_bc<T, DIM><<<grid(nf), 256, 0, stream>>>(P, f, ctl);
        ++launches;
    }

    template <int DIM, int NC>
    void enq_sweeps(const T *coef, T *const *phi, T *const *src, const int *eqs, const int *niter)
    {
        int nmax = 0;
        for (int c = 0; c < NC; ++c) nmax = niter[c] > nmax ? niter[c] : nmax;
        const bool jac = cfg.linear_solver == IFC_JACOBI;
        const long long N = P.g.N;
        const long long half = (long long)((P.g.nx + 1) / 2) * P.g.ny * P.g.nz;
        for (int s = 0; s < nmax; ++s) {
            SweepArgs<T, NC> A;
            A.coef = coef;
            for (int c = 0; c < NC; ++c) {
                A.phi[c] = phi[c];
                A.src[c] = src[c];
                A.eq[c] = eqs[c];
                A.active[c] = s < niter[c];
                A.old[c] = jac ? f.tmp + (size_t)c * N : phi[c];
            }
            if (jac) {
                A.color = -1;
                k_copy_active<T, NC><<<grid(N), 256, 0, stream>>>(A, ctl, (int)N);
                k_sweep<T, DIM, NC><<<grid(N), 256, 0, stream>>>(P, A, ctl, partials);
                launches += 2;
            } else {
                A.color = 0;
                k_sweep<T, DIM, NC><<<grid(half), 256, 0, stream>>>(P, A, ctl, partials);
                A.color = 1;
                k_sweep<T, DIM, NC><<<grid(half), 256, 0, stream>>>(P, A, ctl, partials);
                launches += 2;
            }
        }
    }

    // Deferred-correction sources of the momentum equations (higher-order
    // convection), from the fields at the start of the outer iteration.
    template <int DIM>
    void enq_dc_source()
    {
        if (P.g.conv == CONV_UPWIND) return;
        k_dc_source<T, DIM><<<wave_grid((const void *)k_dc_source<T, DIM>, row_grid()), 256, 0, stream>>>(P, f);
        ++launches;
    }

    template <int DIM>
    void enq_mom_assemble()
    {
        k_mom_assemble<T, DIM><<<grid(P.g.N), 256, 0, stream>>>(P, f, ctl);
        ++launches;
    }

    template <int DIM>
    void enq_mom_solve()
    {
        if (DIM == 2 && fused && cfg.linear_solver == IFC_GAUSS_SEIDEL) {
            enq_fused_mom();
            return;
        }
        if (DIM == 3 && cfg.linear_solver == IFC_GAUSS_SEIDEL) {
            const int ni[3] = {cfg.n_iter_u, cfg.n_iter_v, cfg.n_iter_w};
            const int nmax = ni[0] > ni[1] ? (ni[0] > ni[2] ? ni[0] : ni[2]) : (ni[1] > ni[2] ? ni[1] : ni[2]);
            const long long half = (long long)((P.g.nx + 1) / 2) * P.g.ny * P.g.nz;
            for (int s = 0; s < (nmax > 0 ? nmax : 1); ++s) {
                Half3D h;
                for (int c = 0; c < 3; ++c) h.active[c] = s < ni[c];
                h.first = s == 0;
                for (int color = 0; color < 2; ++color) {
                    h.color = color;
                    if (s == 0)
                        k_mom_half3d<T, true><<<wave_grid((const void *)k_mom_half3d<T, true>, grid(half)), 256, 0, stream>>>(
                            P, f, ctl, partials, h, mpk, mpk_slots);
                    else
                        k_mom_half3d<T, false><<<wave_grid((const void *)k_mom_half3d<T, false>, grid(half)), 256, 0, stream>>>(
                            P, f, ctl, partials, h, mpk, mpk_slots);
                    ++launches;
                }
            }
            return;
        }
        enq_mom_assemble<DIM>();
        T *phi[3] = {f.u, f.v, f.w};
        T *src[3] = {f.su, f.sv, f.sw};
        const int eqs[3] = {EQ_U, EQ_V, EQ_W};
        const int ni[3] = {cfg.n_iter_u, cfg.n_iter_v, cfg.n_iter_w};
        enq_sweeps<DIM, DIM>(f.mc, phi, src, eqs, ni);
    }

    template <int DIM>
    void enq_rhie_chow()
    {
        if (DIM == 2 && fused && cfg.linear_solver == IFC_GAUSS_SEIDEL) {
            enq_fused_rc();
            return;
        }
        k_rhie_chow<T, DIM><<<wave_grid((const void *)k_rhie_chow<T, DIM>, row_grid()), 256, 0, stream>>>(P, f);
        k_pcorr_src<T, DIM><<<wave_grid((const void *)k_pcorr_src<T, DIM>, row_grid()), 256, 0, stream>>>(P, f, ctl, partials);
        launches += 2;
    }

    template <int DIM>
    void enq_pcorr_coef()
    {
        k_pcorr_coef<T, DIM><<<grid(P.g.N), 256, 0, stream>>>(P, f, ctl);
        ++launches;
    }

    template <int DIM>
    void enq_pcorr_solve()
    {
        if (DIM == 2 && fused && cfg.linear_solver == IFC_GAUSS_SEIDEL) {
            enq_fused_pcorr();
        } else if (DIM == 3 && cfg.linear_solver == IFC_GAUSS_SEIDEL && pc3d) {
            k_reset_inner_p<<<1, 1, 0, stream>>>(ctl);
            k_recip_ac<T><<<grid(P.g.N), 256, 0, stream>>>(f.ac, f.rac, P.g.N);
            launches += 2;
            enq_pc_solve3d();
        } else if (DIM == 3 && cfg.linear_solver == IFC_GAUSS_SEIDEL) {
            k_reset_inner_p<<<1, 1, 0, stream>>>(ctl);
            k_recip_ac<T><<<grid(P.g.N), 256, 0, stream>>>(f.ac, f.rac, P.g.N);
            launches += 2;
            if (cfg.n_iter_p == 0) cudaMemsetAsync(f.pc, 0, (size_t)P.g.N * sizeof(T), stream);
            const long long half = (long long)((P.g.nx + 1) / 2) * P.g.ny * P.g.nz;
            for (int s = 0; s < cfg.n_iter_p; ++s)
                for (int color = 0; color < 2; ++color) {
                    const int zm = s == 0 ? (color == 0 ? 1 : 2) : 0;
                    k_pc_half3d<T><<<wave_grid((const void *)k_pc_half3d<T>, grid(half)), 256, 0, stream>>>(P, f, f.rac, ctl, partials, color, zm);
                    ++launches;
                }
        } else {
            enq_pcorr_coef<DIM>();
            cudaMemsetAsync(f.pc, 0, (size_t)P.g.N * sizeof(T), stream);
            T *phi[1] = {f.pc};
            T *src[1] = {f.sp};
            const int eqs[1] = {EQ_P};
            const int ni[1] = {cfg.n_iter_p};
            enq_sweeps<DIM, 1>(f.pcoef, phi, src, eqs, ni);
        }
        if (pin) {
            k_pc_sum<T><<<grid(P.g.N), 256, 0, stream>>>(f.pc, P.g.N, ctl, partials);
            k_pc_shift<T><<<grid(P.g.N), 256, 0, stream>>>(f.pc, P.g.N, ctl);
            launches += 2;
        }
    }

    template <int DIM>
    void enq_update(int use_cond)
    {
        k_update<T, DIM><<<wave_grid((const void *)k_update<T, DIM>, row_grid()), 256, 0, stream>>>(P, f, ctl, partials, cond, use_cond);
        ++launches;
    }

    template <int DIM>
    void enq_iteration(int use_cond)
    {
        // The boundary faces of each iteration are written by the previous
        // iteration's update kernel; run() applies them before the first.
        enq_dc_source<DIM>();
        if (P.g.criterion == 2) {
            k_mom_residual<T, DIM><<<wave_grid((const void *)k_mom_residual<T, DIM>, row_grid()), 256, 0, stream>>>(P, f, ctl, partials);
            ++launches;
        }
        enq_mom_solve<DIM>();
        enq_rhie_chow<DIM>();
        enq_pcorr_solve<DIM>();
        enq_update<DIM>(use_cond);
    }

    void enq_iteration_any(int use_cond)
    {
        if (dim == 2) enq_iteration<2>(use_cond);
        else enq_iteration<3>(use_cond);
    }

    // Fused 2D path (ifc_fused2d.cuh).
    void enq_fused_mom();
    void enq_fused_pcorr();
    void enq_fused_rc();
    int prepare_fused();
    int prepare_persist();
    int launch_persist();

    int build_graph()
    {
        // Preferred form: one graph whose WHILE node repeats the outer
        // iteration until the update kernel clears the condition.
        bool ok = cudaGraphCreate(&graph, 0) == cudaSuccess &&
                  cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            ok = cudaGraphAddNode(&node, graph, nullptr, 0, &cp) == cudaSuccess;
            if (ok) {
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                ok = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    const long long l0 = launches;
                    enq_iteration_any(1);
                    launches_per_iter = launches - l0;
                    ok = cudaStreamEndCapture(stream, &body) == cudaSuccess;
                }
            }
            ok = ok && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
        }
        if (!ok) {
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            exec = nullptr;
            graph = nullptr;
            cond = 0;
            // Fallback: one captured outer iteration, relaunched from the host.
            IFC_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            const long long l0 = launches;
            enq_iteration_any(0);
            launches_per_iter = launches - l0;
            IFC_CK(cudaStreamEndCapture(stream, &body_graph));
            IFC_CK(cudaGraphInstantiate(&body_exec, body_graph, 0));
        }
        IFC_CK(cudaGetLastError());
        return IFC_OK;
    }

    int read_ctl()
    {
        IFC_CK(cudaMemcpyAsync(&ctl_h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        return IFC_OK;
    }

    void print_log()
    {
        for (int q = 0; q < ctl_h.log_n && q < kLogCap; ++q) {
            const LogRec &L = ctl_h.log[q];
            std::printf("iter: %d\n", L.it);
            std::printf("pRelNorm : %.3E\n", L.rel[0]);
            std::printf("uRelNorm : %.3E\n", L.rel[1]);
            std::printf("vRelNorm : %.3E\n", L.rel[2]);
            if (dim == 3) std::printf("wRelNorm : %.3E\n", L.rel[3]);
            std::printf("ufRelNorm: %.3E\n", L.rel[4]);
            std::printf("vfRelNorm: %.3E\n", L.rel[5]);
            if (dim == 3) std::printf("wfRelNorm: %.3E\n", L.rel[6]);
            std::printf("massNorm : %.3E\n", L.mass);
            std::printf("------------------------------------------------------------\n");
        }
        std::fflush(stdout);
    }

    void fill_stats(ifc_stats *st)
    {
        if (!st) return;
        std::memset(st, 0, sizeof(*st));
        st->outer_iterations = ctl_h.it;
        st->converged = ctl_h.converged;
        for (int q = 0; q < 4; ++q) st->sweeps[q] = ctl_h.it_sweeps[q];
        st->cell_updates = ctl_h.cell_updates;
        const double *n = ctl_h.norm, *r = ctl_h.rel;
        st->norm_p = n[0]; st->norm_u = n[1]; st->norm_v = n[2]; st->norm_w = n[3];
        st->norm_uf = n[4]; st->norm_vf = n[5]; st->norm_wf = n[6]; st->norm_mass = n[7];
        st->rel_p = r[0]; st->rel_u = r[1]; st->rel_v = r[2]; st->rel_w = r[3];
        st->rel_uf = r[4]; st->rel_vf = r[5]; st->rel_wf = r[6];
        st->device_ms = last_ms;
        st->kernel_launches = last_launches;
    }

    int run(int n_outer, int act, ifc_stats *st) override
    {
        if (n_outer < 0) {
            err = "negative iteration count";
            return IFC_BAD_ARGUMENT;
        }
        int rc;
        if (n_outer == 0) {
            if ((rc = read_ctl()) != IFC_OK) return rc;
            last_ms = 0.0;
            fill_stats(st);
            if (st) st->status = IFC_OK;
            return IFC_OK;
        }
        k_begin<<<1, 1, 0, stream>>>(ctl, n_outer, act, cfg.log_level);
        IFC_CK(cudaEventRecord(ev0, stream));
        if (dim == 2) enq_face_bc<2>();
        else enq_face_bc<3>();
        if (persist) {
            if ((rc = launch_persist()) != IFC_OK) {
                err = std::string("cooperative launch failed: ") + cudaGetErrorString(cudaGetLastError());
                return rc;
            }
        } else if (exec) {
            IFC_CK(cudaGraphLaunch(exec, stream));
        } else {
            for (int q = 0; q < n_outer; ++q) {
                IFC_CK(cudaGraphLaunch(body_exec, stream));
                if ((rc = read_ctl()) != IFC_OK) return rc;
                if (ctl_h.status || (act && ctl_h.converged)) break;
            }
        }
        IFC_CK(cudaEventRecord(ev1, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        IFC_CK(cudaGetLastError());
        float ms = 0.f;
        IFC_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        last_ms = ms;
        if ((rc = read_ctl()) != IFC_OK) return rc;
        if ((rc = bounds_status()) != IFC_OK) return rc;
        if (cfg.log_level > 0) print_log();
        last_launches = persist ? 3 : 2 + (long long)(ctl_h.it - ctl_h.it_begin) * launches_per_iter;
        fill_stats(st);
        int status = IFC_OK;
        if (ctl_h.status == 3) {
            status = IFC_TIMEOUT;
            err = "a grid barrier of the single-launch solve timed out";
        } else if (ctl_h.status == 2) status = IFC_DIVERGED;
        else if (act && !ctl_h.converged) status = IFC_NOT_CONVERGED;
        if (st) st->status = status;
        return status;
    }

    int run_stage(int stage) override
    {
        if (stage < 0 || stage >= IFC_STAGE_COUNT) {
            err = "unknown stage";
            return IFC_BAD_ARGUMENT;
        }
        if (dim == 2) run_stage_t<2>(stage);
        else run_stage_t<3>(stage);
        IFC_CK(cudaGetLastError());
        return sync();
    }

    // The stage's launches on the handle's stream, without waiting: a caller
    // that orders its own work after them on the same stream (the slab halo
    // copies, NCCL transfers) reads their outcome at the next sync().
    int run_stage_async(int stage) override
    {
        if (stage < 0 || stage >= IFC_STAGE_COUNT) {
            err = "unknown stage";
            return IFC_BAD_ARGUMENT;
        }
        if (dim == 2) run_stage_t<2>(stage);
        else run_stage_t<3>(stage);
        IFC_CK(cudaGetLastError());
        return IFC_OK;
    }

    // Wait for the handle's stream; report a bounded wait that ran out
    // (control-block status 3) and, in the bounds-checked build, an index out
    // of range.
    int sync() override
    {
        IFC_CK(cudaStreamSynchronize(stream));
        const int rc = read_ctl();
        if (rc != IFC_OK) return rc;
        if (ctl_h.status == 3) {  // reported once: cleared for the handle's next launches
            IFC_CK(cudaMemsetAsync(&ctl->status, 0, sizeof(int), stream));
            IFC_CK(cudaStreamSynchronize(stream));
            err = "a grid barrier of a cooperative launch timed out";
            return IFC_TIMEOUT;
        }
        return bounds_status();
    }

    template <int DIM>
    void run_stage_t(int stage)
    {
        switch (stage) {
        case IFC_STAGE_FACE_BC: enq_face_bc<DIM>(); break;
        case IFC_STAGE_MOM_ASSEMBLE:
            enq_dc_source<DIM>();
            enq_mom_assemble<DIM>();
            break;
        case IFC_STAGE_MOM_SOLVE:
            k_reset_inner<<<1, 1, 0, stream>>>(ctl, 7);
            enq_dc_source<DIM>();
            enq_mom_solve<DIM>();
            break;
        case IFC_STAGE_RHIE_CHOW: enq_rhie_chow<DIM>(); break;
        case IFC_STAGE_PCORR_COEF: enq_pcorr_coef<DIM>(); break;
        case IFC_STAGE_PCORR_SOLVE:
            k_reset_inner<<<1, 1, 0, stream>>>(ctl, 8);
            enq_pcorr_solve<DIM>();
            break;
        case IFC_STAGE_UPDATE:
            k_begin<<<1, 1, 0, stream>>>(ctl, 1, 0, 0);
            enq_update<DIM>(0);
            break;
        }
    }

    int time_stage(int stage, int reps, double *ms, int *nl) override
    {
        if (stage < 0 || stage >= IFC_STAGE_COUNT || reps < 1 || !ms) {
            err = "time_stage: bad stage or count";
            return IFC_BAD_ARGUMENT;
        }
        IFC_CK(cudaStreamSynchronize(stream));
        const long long l0 = launches;
        IFC_CK(cudaEventRecord(ev0, stream));
        for (int r = 0; r < reps; ++r) {
            if (dim == 2) run_stage_t<2>(stage);
            else run_stage_t<3>(stage);
        }
        IFC_CK(cudaEventRecord(ev1, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        IFC_CK(cudaGetLastError());
        float t = 0.f;
        IFC_CK(cudaEventElapsedTime(&t, ev0, ev1));
        *ms = (double)t / reps;
        if (nl) *nl = (int)((launches - l0) / reps);
        return bounds_status();
    }

    int sweep(int eq, int n, double *sq) override
    {
        if (eq < 0 || eq > 3 || (eq == 2 && dim == 2) || n < 0) {
            err = "sweep: bad equation or count";
            return IFC_BAD_ARGUMENT;
        }
        if (!sq) {
            const int rc = enq_sweeps_stored(eq, n);
            return rc != IFC_OK ? rc : sync();
        }
        // With sq the host reads each sweep's sum.
        T *phi[1] = {eq == 0 ? f.u : eq == 1 ? f.v : eq == 2 ? f.w : f.pc};
        T *src[1] = {eq == 0 ? f.su : eq == 1 ? f.sv : eq == 2 ? f.sw : f.sp};
        const int eqs[1] = {eq};
        const int one[1] = {1};
        for (int s = 0; s < n; ++s) {
            k_reset_inner<<<1, 1, 0, stream>>>(ctl, 1 << eq);
            if (dim == 2) enq_sweeps<2, 1>(eq == 3 ? f.pcoef : f.mc, phi, src, eqs, one);
            else enq_sweeps<3, 1>(eq == 3 ? f.pcoef : f.mc, phi, src, eqs, one);
            IFC_CK(cudaGetLastError());
            int rc = read_ctl();
            if (rc != IFC_OK) return rc;
            sq[s] = ctl_h.last_sweep_sq[eq];
        }
        return bounds_status();
    }

    int sweep_async(int eq, int n) override
    {
        if (eq < 0 || eq > 3 || (eq == 2 && dim == 2) || n < 0) {
            err = "sweep: bad equation or count";
            return IFC_BAD_ARGUMENT;
        }
        return enq_sweeps_stored(eq, n);
    }

    // Exactly n red-black sweeps of equation eq on the stored planes, enqueued:
    // one cooperative launch where the handle has one (k_coef_solve2d in 2D,
    // k_csolve3d in 3D; the same point updates in the same colour order,
    // tolerance 0 so no early exit), else a launch pair per sweep.
    int enq_sweeps_stored(int eq, int n)
    {
        T *phi[1] = {eq == 0 ? f.u : eq == 1 ? f.v : eq == 2 ? f.w : f.pc};
        T *src[1] = {eq == 0 ? f.su : eq == 1 ? f.sv : eq == 2 ? f.sw : f.sp};
        const T *coef = eq == 3 ? f.pcoef : f.mc;
        if (n > 0 && cfg.linear_solver == IFC_GAUSS_SEIDEL) {
            Params<T> PT = P;
            PT.g.tol[eq] = 0.0;
            using S = TileShape2D<T>;
            using R = Region<S::TX, S::TY, 10>;
            const int tiles = ((P.g.nx + S::TX - 1) / S::TX) * ((P.g.ny + S::TY - 1) / S::TY);
            const bool c2 = dim == 2 && fused && energy_coop(tiles);
            const bool c3 = dim == 3 && pc3d;
            if (c2 || c3) {
                k_reset_inner<<<1, 1, 0, stream>>>(ctl, 1 << eq);
                if (c3) {
                    CSys<T> sys = {coef, src[0], phi[0], eq};
                    enq_csolve3d(PT, sys, n);
                } else {
                    IFC_CK(cudaMemsetAsync(barrier, 0, sizeof(GridBarrier), stream));
                    int e = eq, ns = n, stall = 0;
                    T *x0 = phi[0], *x1 = f.tmp + 2 * (size_t)P.g.N;
                    const T *srcp = src[0];
                    void *args[] = {&PT, &coef, &srcp, &ctl, &partials, &barrier, &e, &ns, &x0, &x1, &stall};
                    IFC_CK(cudaLaunchCooperativeKernel((const void *)k_coef_solve2d<T, S::TX, S::TY, 5, S::NT>,
                                                       dim3(tiles), dim3(S::NT), args, R::NR * sizeof(T), stream));
                    ++launches;
                }
                IFC_CK(cudaGetLastError());
                return IFC_OK;
            }
        }
        const int eqs[1] = {eq};
        const int one[1] = {1};
        for (int s = 0; s < n; ++s) {
            k_reset_inner<<<1, 1, 0, stream>>>(ctl, 1 << eq);
            if (dim == 2) enq_sweeps<2, 1>(coef, phi, src, eqs, one);
            else enq_sweeps<3, 1>(coef, phi, src, eqs, one);
        }
        IFC_CK(cudaGetLastError());
        return IFC_OK;
    }

    // Steady temperature on the current flow (ifc_energy.cuh): assemble the
    // energy equation once, then red-black sweeps of the temperature in chunks
    // until the inner rule (RMS change of a sweep over the largest RMS change
    // of this solve < tol) or max_sweeps.  The sweep bookkeeping uses the w
    // slots of the control block, which the next outer iteration resets.
    int solve_energy(int max_sweeps, double tol, ifc_energy_result *res) override
    {
        if (max_sweeps < 0 || !(tol >= 0.0)) {
            err = "solve_energy: bad sweep count or tolerance";
            return IFC_BAD_ARGUMENT;
        }
        const Geo<T> &g = P.g;
        TempArgs<T> ta;
        const T gam = (T)cfg.thermal_conductivity / (T)cfg.specific_heat_capacity;
        ta.Dx = gam * g.Ax / g.dx;
        ta.Dy = gam * g.Ay / g.dy;
        ta.Dz = gam * g.Az / g.dz;
        for (int q = 0; q < 6; ++q) {
            ta.type[q] = cfg.temp_bc_type[q];
            ta.val[q] = (T)cfg.temp_bc_val[q];
        }
        Params<T> PT = P;
        PT.g.relax[EQ_W] = (T)1;
        PT.g.tol[EQ_W] = tol;
        const long long N = g.N;
        T *src = f.tmp;
        IFC_CK(cudaStreamSynchronize(stream));
        // A timeout of an earlier call leaves status 3 in the control block.
        IFC_CK(cudaMemsetAsync(&ctl->status, 0, sizeof(int), stream));
        const char *stall_env = std::getenv("IFC_TEST_STALL_BARRIER");
        int stall_test = (stall_env && stall_env[0] == '1') ? 1 : 0;
        IFC_CK(cudaEventRecord(ev0, stream));
        if (dim == 2) k_temp_assemble<T, 2><<<grid(N), 256, 0, stream>>>(P, f, ta, f.mc, src);
        else k_temp_assemble<T, 3><<<grid(N), 256, 0, stream>>>(P, f, ta, f.mc, src);
        k_reset_inner<<<1, 1, 0, stream>>>(ctl, 1 << EQ_W);
        // Higher-order convection: every cycle of up to 25 sweeps starts from
        // src + the deferred correction of the current temperature; the solve
        // has converged when a cycle meets the tolerance in its first sweep.
        const bool dc = g.conv != CONV_UPWIND;
        T *src_eff = dc ? f.tmp + N : src;
        SweepArgs<T, 1> A;
        A.coef = f.mc;
        A.phi[0] = f.temp;
        A.old[0] = f.temp;
        A.src[0] = src_eff;
        A.eq[0] = EQ_W;
        A.active[0] = 1;
        const long long half = (long long)((g.nx + 1) / 2) * g.ny * g.nz;
        // 2D: temporally blocked passes of kEnergyKS sweeps on the stored
        // coefficients (k_coef_pass2d), ping-ponging T with scratch; the
        // early-exit rule is then applied after each pass, as in the fused
        // p' passes.  3D: one cooperative launch per cycle when the p'
        // solve has one (k_csolve3d), else one launch per colour and sweep.
        const bool blocked = dim == 2 && fused && cfg.linear_solver == IFC_GAUSS_SEIDEL;
        constexpr int kEnergyKS = 5;
        const int gran = blocked ? kEnergyKS : 1;  // sweeps counted per early-exit check
        T *tbuf[2] = {f.temp, f.tmp + 2 * N};
        // Cycles of 25 sweeps with a host check between them; without the
        // deferred correction the cooperative kernel applies the early-exit
        // rule on the device, so the whole solve is one cycle there.
        int cycle_len = 25;
        {
            using S = TileShape2D<T>;
            const int tiles = ((g.nx + S::TX - 1) / S::TX) * ((g.ny + S::TY - 1) / S::TY);
            if (blocked && !dc && energy_coop(tiles) && max_sweeps > 0) cycle_len = max_sweeps;
        }
        // 3D: one cooperative launch per cycle on the stored planes
        // (k_csolve3d), the early-exit rule applied after every sweep on the
        // device, as the per-sweep launches apply it.
        const bool coop3 = dim == 3 && pc3d && cfg.linear_solver == IFC_GAUSS_SEIDEL;
        if (coop3 && !dc && max_sweeps > 0) cycle_len = max_sweeps;
        int done = 0, cycle_start = 0;
        while (done < max_sweeps) {
            const int chunk = max_sweeps - done < cycle_len ? max_sweeps - done : cycle_len;
            if (dc) {
                if (dim == 2) k_temp_dc<T, 2><<<row_grid(), 256, 0, stream>>>(P, f, src, src_eff);
                else k_temp_dc<T, 3><<<row_grid(), 256, 0, stream>>>(P, f, src, src_eff);
                k_clear_stop<<<1, 1, 0, stream>>>(ctl, EQ_W);
                cycle_start = done == 0 ? 0 : ctl_h.sweeps[EQ_W];  // host copy read after the last cycle
            }
            using S = TileShape2D<T>;
            using R = Region<S::TX, S::TY, 2 * kEnergyKS>;
            const int tiles = ((g.nx + S::TX - 1) / S::TX) * ((g.ny + S::TY - 1) / S::TY);
            if (blocked && energy_coop(tiles)) {
                // the whole cycle in one cooperative launch (k_coef_solve2d)
                IFC_CK(cudaMemsetAsync(barrier, 0, sizeof(GridBarrier), stream));
                int ns_cycle = chunk, eq = EQ_W;
                T *x1 = tbuf[1];
                const T *coef = f.mc, *srcp = src_eff;
                void *args[] = {&PT, &coef, &srcp, &ctl, &partials, &barrier, &eq, &ns_cycle, &f.temp, &x1, &stall_test};
                IFC_CK(cudaLaunchCooperativeKernel((const void *)k_coef_solve2d<T, S::TX, S::TY, kEnergyKS, S::NT>,
                                                   dim3(tiles), dim3(S::NT), args, R::NR * sizeof(T), stream));
                ++launches;
            } else if (blocked) {
                int cur = 0;
                for (int pass = 0; pass * kEnergyKS < chunk; ++pass) {
                    k_coef_pass2d<T, S::TX, S::TY, kEnergyKS, S::NT><<<tiles, S::NT, R::NR * sizeof(T), stream>>>(
                        PT, f.mc, src_eff, ctl, partials, EQ_W, clamp_sweeps(chunk, pass, kEnergyKS), tbuf[cur],
                        tbuf[cur ^ 1]);
                    cur ^= 1;
                }
                if (cur) IFC_CK(cudaMemcpyAsync(f.temp, tbuf[1], (size_t)N * sizeof(T), cudaMemcpyDeviceToDevice, stream));
            } else if (coop3) {
                CSys<T> sys = {f.mc, src_eff, f.temp, EQ_W};
                enq_csolve3d(PT, sys, chunk);
            } else {
                for (int q = 0; q < chunk; ++q)
                    for (int color = 0; color < 2; ++color) {
                        A.color = color;
                        if (dim == 2) k_sweep<T, 2, 1><<<grid(half), 256, 0, stream>>>(PT, A, ctl, partials);
                        else k_sweep<T, 3, 1><<<grid(half), 256, 0, stream>>>(PT, A, ctl, partials);
                    }
            }
            done += chunk;
            IFC_CK(cudaGetLastError());
            int rc = read_ctl();
            if (rc != IFC_OK) return rc;
            if (ctl_h.status == 3) {
                // A grid barrier of the cooperative sweep launch gave up: the
                // temperature may hold tiles of different passes.
                err = "a grid barrier of the cooperative energy solve timed out";
                if (res) {
                    std::memset(res, 0, sizeof(*res));
                    res->status = IFC_TIMEOUT;
                }
                k_reset_inner<<<1, 1, 0, stream>>>(ctl, 1 << EQ_W);
                IFC_CK(cudaMemsetAsync(&ctl->status, 0, sizeof(int), stream));
                IFC_CK(cudaStreamSynchronize(stream));
                return IFC_TIMEOUT;
            }
            if (ctl_h.stop[EQ_W] && (!dc || ctl_h.sweeps[EQ_W] - cycle_start <= gran)) break;
        }
        IFC_CK(cudaEventRecord(ev1, stream));
        int rc = read_ctl();
        if (rc != IFC_OK) return rc;
        float ms = 0.f;
        IFC_CK(cudaEventElapsedTime(&ms, ev0, ev1));
        if (res) {
            std::memset(res, 0, sizeof(*res));
            res->sweeps = ctl_h.sweeps[EQ_W];
            res->converged = ctl_h.stop[EQ_W];
            const double last = std::sqrt(ctl_h.last_sweep_sq[EQ_W] / (double)N);
            res->residual = ctl_h.inner_max[EQ_W] > 0.0 ? last / ctl_h.inner_max[EQ_W] : 0.0;
            res->device_ms = ms;
            res->status = ctl_h.stop[EQ_W] || tol == 0.0 ? IFC_OK : IFC_NOT_CONVERGED;
        }
        k_reset_inner<<<1, 1, 0, stream>>>(ctl, 1 << EQ_W);
        IFC_CK(cudaStreamSynchronize(stream));
        if ((rc = bounds_status()) != IFC_OK) return rc;
        return ctl_h.stop[EQ_W] || tol == 0.0 ? IFC_OK : IFC_NOT_CONVERGED;
    }

    // Whether the energy cycle fits one cooperative launch (one tile per CTA).
    int energy_coop_state = -1;
    bool energy_coop(int tiles)
    {
        if (energy_coop_state < 0) {
            using S = TileShape2D<T>;
            using R = Region<S::TX, S::TY, 10>;
            int per_sm = 0, dev = 0, coop = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
            if (coop && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coef_solve2d<T, S::TX, S::TY, 5, S::NT>,
                                                                      S::NT, R::NR * sizeof(T)) != cudaSuccess) {
                cudaGetLastError();
                per_sm = 0;
            }
            const char *off = std::getenv("IFC_PERSIST_OFF");
            energy_coop_state = coop && per_sm > 0 && !(off && off[0] == '1') && tiles <= per_sm * nsm ? 1 : 0;
        }
        return energy_coop_state == 1;
    }

    int set_inlet(const double *profile) override
    {
        if (!inlet_d || !profile) {
            err = "set_inlet_profile: the handle was created without an inlet profile";
            return IFC_BAD_ARGUMENT;
        }
        const size_t n = (size_t)P.g.ny * P.g.nz;
        std::vector<T> h(n);
        for (size_t q = 0; q < n; ++q) h[q] = (T)profile[q];
        IFC_CK(cudaMemcpyAsync(inlet_d, h.data(), n * sizeof(T), cudaMemcpyHostToDevice, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        return IFC_OK;
    }

    int adjoint(const AdjointReq &rq0, ifc_adjoint_result *res) override
    {
        AdjointReq rq = rq0;
        rq.pin = pin ? 1 : 0;
        IFC_CK(cudaStreamSynchronize(stream));
        return adjoint_run<T>(adj, cfg, make_params<double>(cfg), f, inlet_d, stream, rq, res, err);
    }

    int stats(ifc_stats *st) override
    {
        int rc = read_ctl();
        if (rc != IFC_OK) return rc;
        fill_stats(st);
        if (st) st->status = IFC_OK;
        return IFC_OK;
    }
};

}  // namespace ifc
