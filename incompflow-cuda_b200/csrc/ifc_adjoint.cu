// ifc_adjoint.cu -- driver of the discrete adjoint.  Preferred form: the
// whole fixed-point solve in one cooperative launch (ifc_adjoint_persist.cuh),
// when every tile's CTA fits on the GPU at once.  Otherwise one reverse pass
// (ifc_adjoint2d.cuh) is captured into a CUDA graph whose conditional WHILE
// node repeats it until the adjoint iterate stops changing (the finish kernel
// sets the condition on the device); a second graph holds one pass without
// the iterate update, used for the final gradient and for single applications
// of G_x^T.  IFC_ADJOINT_GRAPH=1 in the environment selects the graph form
// (for testing both).  FP64 buffers are allocated on the first call of a
// handle and kept with it.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ifc_adjoint.h"
#include "ifc_adjoint2d.cuh"
#include "ifc_adjoint_persist.cuh"

namespace ifc {

#define IFC_CK(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                     \
            return IFC_CUDA_ERROR;                                                        \
        }                                                                                 \
    } while (0)

struct AdjointCtx {
    int nx = 0, ny = 0, N = 0, NU = 0, NV = 0;
    int grid = 1;
    AdjBufs b;
    Ctl *ctl = nullptr;
    double *partials = nullptr;
    double *inlet = nullptr;
    std::vector<void *> allocs;
    cudaStream_t stream = nullptr;
    Params<double> P;
    AdjArgs A;
    int n_u = 0, n_v = 0, n_p = 0, pin = 0;
    cudaGraph_t g_loop = nullptr, g_tail = nullptr, g_body = nullptr;
    cudaGraphExec_t x_loop = nullptr, x_tail = nullptr, x_body = nullptr;
    cudaGraphConditionalHandle cond = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    long long per_pass = 0;  // kernels in one reverse pass
    std::string err;
    // single-launch form
    static constexpr int kTX = 32, kTY = 8, kKS = 5, kNT = 512;
    bool persist = false;
    int tiles = 0;
    size_t smem = 0;
    GridBarrier *bar = nullptr;

    ~AdjointCtx()
    {
        if (stream) cudaStreamSynchronize(stream);
        if (x_loop) cudaGraphExecDestroy(x_loop);
        if (g_loop) cudaGraphDestroy(g_loop);
        if (x_tail) cudaGraphExecDestroy(x_tail);
        if (g_tail) cudaGraphDestroy(g_tail);
        if (x_body) cudaGraphExecDestroy(x_body);
        if (g_body) cudaGraphDestroy(g_body);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        for (void *p : allocs) cudaFree(p);
    }

    template <typename U>
    int alloc(U **p, size_t n)
    {
        void *q = nullptr;
        IFC_CK(cudaMalloc(&q, n * sizeof(U) > 0 ? n * sizeof(U) : 16));
        allocs.push_back(q);
        *p = (U *)q;
        return IFC_OK;
    }

    // Transposed red-black sweeps: n sweeps, colour 1 then colour 0 in each
    // (the forward sweep does colour 0 first).  Ends in buffer 0.
    void enq_halves(int n, int ncomp, double *const *bufs0, double *const *bufs1, double *const *lb,
                    const double *const *phi, const double *alpha, const double *a, double *la)
    {
        int cur = 0;
        for (int s = 0; s < n; ++s)
            for (int color = 1; color >= 0; --color) {
                HalfT H;
                std::memset(&H, 0, sizeof(H));
                H.a = a;
                H.ncomp = ncomp;
                H.color = color;
                H.la = la;
                for (int m = 0; m < ncomp; ++m) {
                    H.in[m] = cur == 0 ? bufs0[m] : bufs1[m];
                    H.out[m] = cur == 0 ? bufs1[m] : bufs0[m];
                    H.lb[m] = lb[m];
                    H.phi[m] = phi ? phi[m] : nullptr;
                    H.alpha[m] = alpha[m];
                }
                k_adj_half<<<grid, 256, 0, stream>>>(P, H);
                ++per_pass;
                cur ^= 1;
            }
    }

    // One reverse pass.  finish_mode: bit 0 sets the loop condition, bit 1
    // counts the pass; copy: make the new iterate current.
    void enq_pass(int finish_mode, bool copy)
    {
        per_pass = 0;
        k_adj_corr<<<grid, 256, 0, stream>>>(P, b, A);
        ++per_pass;
        if (pin) {
            k_adj_sum<<<grid, 256, 0, stream>>>(b.lpc[0], N, ctl, partials);
            k_adj_shift<<<grid, 256, 0, stream>>>(b.lpc[0], N, ctl);
            per_pass += 2;
        }
        {
            double *b0[1] = {b.lpc[0]}, *b1[1] = {b.lpc[1]}, *lb[1] = {b.lbp};
            const double al[1] = {A.alpha_p};
            enq_halves(n_p, 1, b0, b1, lb, nullptr, al, b.ap, nullptr);
        }
        k_adj_src_faces<<<grid, 256, 0, stream>>>(P, b);
        k_adj_rc<<<grid, 256, 0, stream>>>(P, b, 0);
        per_pass += 2;
        if (n_u == n_v) {
            double *b0[2] = {b.lus[0], b.lvs[0]}, *b1[2] = {b.lus[1], b.lvs[1]}, *lb[2] = {b.lbu, b.lbv};
            const double *phi[2] = {b.u, b.v};
            const double al[2] = {A.alpha_u, A.alpha_v};
            enq_halves(n_u, 2, b0, b1, lb, phi, al, b.afold, b.la);
        } else {
            double *b0u[1] = {b.lus[0]}, *b1u[1] = {b.lus[1]}, *lbu[1] = {b.lbu};
            const double *phu[1] = {b.u};
            const double alu[1] = {A.alpha_u};
            enq_halves(n_u, 1, b0u, b1u, lbu, phu, alu, b.afold, b.la);
            double *b0v[1] = {b.lvs[0]}, *b1v[1] = {b.lvs[1]}, *lbv[1] = {b.lbv};
            const double *phv[1] = {b.v};
            const double alv[1] = {A.alpha_v};
            enq_halves(n_v, 1, b0v, b1v, lbv, phv, alv, b.afold, b.la);
        }
        k_adj_fold<<<grid, 256, 0, stream>>>(P, b);
        k_adj_links<<<grid, 256, 0, stream>>>(P, b);
        k_adj_finish<<<grid, 256, 0, stream>>>(P, b, 0, ctl, partials, cond, finish_mode);
        per_pass += 3;
        if (copy) {
            k_adj_copy<<<grid, 256, 0, stream>>>(P, b);
            ++per_pass;
        }
    }

    int build_graphs()
    {
        bool ok = cudaGraphCreate(&g_loop, 0) == cudaSuccess &&
                  cudaGraphConditionalHandleCreate(&cond, g_loop, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        if (ok) {
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            ok = cudaGraphAddNode(&node, g_loop, nullptr, 0, &cp) == cudaSuccess;
            if (ok) {
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                ok = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0,
                                                   cudaStreamCaptureModeThreadLocal) == cudaSuccess;
                if (ok) {
                    enq_pass(3, true);
                    ok = cudaStreamEndCapture(stream, &body) == cudaSuccess;
                }
            }
            ok = ok && cudaGraphInstantiate(&x_loop, g_loop, 0) == cudaSuccess;
        }
        if (!ok) {
            // Without conditional nodes: one pass per graph launch, the host
            // checks the convergence flag between chunks of launches.
            cudaGetLastError();
            if (x_loop) cudaGraphExecDestroy(x_loop);
            if (g_loop) cudaGraphDestroy(g_loop);
            x_loop = nullptr;
            g_loop = nullptr;
            cond = 0;
            IFC_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            enq_pass(2, true);
            IFC_CK(cudaStreamEndCapture(stream, &g_body));
            IFC_CK(cudaGraphInstantiate(&x_body, g_body, 0));
        }
        IFC_CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        enq_pass(0, false);
        IFC_CK(cudaStreamEndCapture(stream, &g_tail));
        IFC_CK(cudaGraphInstantiate(&x_tail, g_tail, 0));
        IFC_CK(cudaGetLastError());
        return IFC_OK;
    }

    int init(const ifc_config &cfg, const Params<double> &Pd, cudaStream_t s, int pin_, bool has_inlet)
    {
        stream = s;
        P = Pd;
        nx = P.g.nx;
        ny = P.g.ny;
        N = P.g.N;
        NU = (nx + 1) * ny;
        NV = nx * (ny + 1);
        n_u = cfg.n_iter_u;
        n_v = cfg.n_iter_v;
        n_p = cfg.n_iter_p;
        pin = pin_;
        A.alpha_u = cfg.relax_u;
        A.alpha_v = cfg.relax_v;
        A.alpha_p = cfg.relax_p;
        A.ru = cfg.relax_u * 0.5;
        A.rv = cfg.relax_v * 0.5;
        int dev = 0, nsm = 148;
        IFC_CK(cudaGetDevice(&dev));
        IFC_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const long long work = (long long)(N > NU + NV ? N : NU + NV);
        long long G = (work + 255) / 256;
        if (G > 8LL * nsm) G = 8LL * nsm;
        grid = (int)(G < 1 ? 1 : G);
        std::memset(&b, 0, sizeof(b));
        int rc;
#define A_(ptr, n) if ((rc = alloc(&(ptr), (size_t)(n))) != IFC_OK) return rc
        A_(b.u, N); A_(b.v, N); A_(b.p, N); A_(b.uf, NU); A_(b.vf, NV);
        A_(b.araw, 5 * (size_t)N); A_(b.afold, 5 * (size_t)N); A_(b.ap, 5 * (size_t)N);
        A_(b.lu, N); A_(b.lv, N); A_(b.lp, N); A_(b.luf, NU); A_(b.lvf, NV);
        A_(b.ou, N); A_(b.ov, N); A_(b.op, N); A_(b.ouf, NU); A_(b.ovf, NV);
        A_(b.ju, N); A_(b.jv, N); A_(b.jp, N);
        A_(b.lpc[0], N); A_(b.lpc[1], N); A_(b.lus[0], N); A_(b.lus[1], N); A_(b.lvs[0], N); A_(b.lvs[1], N);
        A_(b.lbp, N); A_(b.lbu, N); A_(b.lbv, N); A_(b.la, 5 * (size_t)N);
        A_(b.lufs, NU); A_(b.lvfs, NV); A_(b.lufa, NU); A_(b.lvfa, NV);
        A_(b.ltheta, ny); A_(b.scal, 8);
        tiles = ((nx + kTX - 1) / kTX) * ((ny + kTY - 1) / kTY);
        const size_t np = 3 * (size_t)grid > 6 * (size_t)tiles ? 3 * (size_t)grid : 6 * (size_t)tiles;
        A_(ctl, 1); A_(partials, np); A_(inlet, ny); A_(bar, 1);
#undef A_
        IFC_CK(cudaMemsetAsync(ctl, 0, sizeof(Ctl), stream));
        IFC_CK(cudaMemsetAsync(b.scal, 0, 8 * sizeof(double), stream));
        P.g.inlet = has_inlet ? inlet : nullptr;
        IFC_CK(cudaEventCreate(&e0));
        IFC_CK(cudaEventCreate(&e1));
        if ((rc = prepare_persist(nsm)) != IFC_OK) return rc;
        return build_graphs();
    }

    int prepare_persist(int nsm)
    {
        persist = false;
        const char *env = std::getenv("IFC_ADJOINT_GRAPH");
        if (env && env[0] == '1') return IFC_OK;
        using R = Region<kTX, kTY, 2 * kKS>;
        smem = (size_t)12 * R::NR * sizeof(double);
        auto kern = k_adjoint2d<kTX, kTY, kKS, kNT>;
        IFC_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        IFC_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kNT, smem));
        int dev = 0, coop = 0;
        IFC_CK(cudaGetDevice(&dev));
        IFC_CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        persist = coop && per_sm > 0 && (long long)per_sm * nsm >= tiles;
        return IFC_OK;
    }

    AdjPArgs pargs(int single, int max_iter, double tol) const
    {
        AdjPArgs a;
        std::memset(&a, 0, sizeof(a));
        a.n_iter[0] = n_u;
        a.n_iter[1] = n_v;
        a.n_iter[2] = n_p;
        a.pin = pin;
        a.alpha[0] = A.alpha_u;
        a.alpha[1] = A.alpha_v;
        a.alpha[2] = A.alpha_p;
        a.ru = A.ru;
        a.rv = A.rv;
        a.max_iter = max_iter;
        a.tol = tol;
        a.single = single;
        return a;
    }

    // One cooperative launch of the whole solve (or of one pass).
    int launch_persist(const AdjPArgs &a)
    {
        IFC_CK(cudaMemsetAsync(bar, 0, sizeof(GridBarrier), stream));
        AdjPArgs aa = a;
        void *args[] = {(void *)&P, (void *)&b, (void *)&aa, (void *)&partials, (void *)&bar};
        IFC_CK(cudaLaunchCooperativeKernel((const void *)k_adjoint2d<kTX, kTY, kKS, kNT>, dim3(tiles), dim3(kNT),
                                           args, smem, stream));
        return IFC_OK;
    }

    int barrier_error(bool &timed_out)
    {
        GridBarrier h;
        IFC_CK(cudaMemcpyAsync(&h, bar, sizeof(h), cudaMemcpyDeviceToHost, stream));
        IFC_CK(cudaStreamSynchronize(stream));
        timed_out = h.err != 0;
        return IFC_OK;
    }
};

void adjoint_free(AdjointCtx *ctx) { delete ctx; }

template <typename T>
int adjoint_run(AdjointCtx *&ctx, const ifc_config &cfg, Params<double> Pd, const Fields<T> &f, const T *inlet,
                cudaStream_t stream, const AdjointReq &rq, ifc_adjoint_result *res, std::string &err)
{
    if (Pd.g.dim != 2 || cfg.linear_solver != IFC_GAUSS_SEIDEL || cfg.convection_scheme != IFC_CONV_UPWIND) {
        err = "the adjoint supports 2D red-black Gauss-Seidel solves with upwind convection only";
        return IFC_UNSUPPORTED;
    }
    if (!ctx) {
        ctx = new AdjointCtx();
        const int rc = ctx->init(cfg, Pd, stream, rq.pin, inlet != nullptr);
        if (rc != IFC_OK) {
            err = ctx->err;
            delete ctx;
            ctx = nullptr;
            return rc;
        }
    }
    AdjointCtx &c = *ctx;
    AdjBufs &b = c.b;
    const size_t N = (size_t)c.N, NU = (size_t)c.NU, NV = (size_t)c.NV;
#define CK(call) IFC_CK(call)
    long long launches = 0;
    CK(cudaEventRecord(c.e0, stream));
    if (inlet) {
        k_adj_inlet<T><<<1, 256, 0, stream>>>(inlet, c.inlet, c.ny);
        ++launches;
    }
    k_adj_prep<T><<<c.grid, 256, 0, stream>>>(c.P, f, b);
    k_adj_bcfaces<<<c.grid, 256, 0, stream>>>(c.P, b);
    k_adj_coef<<<c.grid, 256, 0, stream>>>(c.P, b);
    k_adj_pcoef<<<c.grid, 256, 0, stream>>>(c.P, b);
    launches += 4;
    double hs[8] = {0, 0, 0, 0, 0, 0, rq.tol, (double)rq.max_iter};
    if (rq.mode == 0) {
        CK(cudaMemcpyAsync(b.scal + 6, hs + 6, 2 * sizeof(double), cudaMemcpyHostToDevice, stream));
        const bool builtin = rq.objective == IFC_OBJ_PRESSURE_DROP;
        if (!builtin) {
            double *dst[3] = {b.ju, b.jv, b.jp};
            for (int q = 0; q < 3; ++q) {
                if (rq.seed[q]) CK(cudaMemcpyAsync(dst[q], rq.seed[q], N * sizeof(double), cudaMemcpyHostToDevice, stream));
                else CK(cudaMemsetAsync(dst[q], 0, N * sizeof(double), stream));
            }
        }
        k_adj_seed<<<c.grid, 256, 0, stream>>>(c.P, b, builtin ? 1 : 0);
        k_adj_objective<<<1, 256, 0, stream>>>(c.P, b);
        launches += 2;
        if (c.persist) {
            int rc = c.launch_persist(c.pargs(0, rq.max_iter, rq.tol));
            if (rc != IFC_OK) {
                err = c.err;
                return rc;
            }
            ++launches;
        } else if (c.x_loop) {
            CK(cudaGraphLaunch(c.x_loop, stream));
        } else {
            // Host-checked fallback: chunks of 32 passes.
            int done = 0;
            while (done < rq.max_iter) {
                const int n = rq.max_iter - done < 32 ? rq.max_iter - done : 32;
                for (int q = 0; q < n; ++q) CK(cudaGraphLaunch(c.x_body, stream));
                done += n;
                double conv = 0.0;
                CK(cudaMemcpyAsync(&conv, b.scal + 4, sizeof(double), cudaMemcpyDeviceToHost, stream));
                CK(cudaStreamSynchronize(stream));
                if (conv != 0.0) break;
            }
        }
        if (!c.persist) CK(cudaGraphLaunch(c.x_tail, stream));
        CK(cudaEventRecord(c.e1, stream));
        CK(cudaMemcpyAsync(hs, b.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        if (rq.dtheta) CK(cudaMemcpyAsync(rq.dtheta, b.ltheta, c.ny * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        CK(cudaGetLastError());
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c.e0, c.e1));
        if (c.persist) {
            bool to = false;
            if (c.barrier_error(to) != IFC_OK) {
                err = c.err;
                return IFC_CUDA_ERROR;
            }
            if (to) {
                err = "a grid barrier of the single-launch adjoint timed out";
                return IFC_TIMEOUT;
            }
        }
        const int its = (int)hs[3];
        const bool conv = hs[1] <= rq.tol * hs[2];
        if (!c.persist) launches += (long long)(its + 1) * c.per_pass;
        if (res) {
            res->iterations = its;
            res->converged = conv ? 1 : 0;
            res->residual = hs[2] > 0.0 ? hs[1] / hs[2] : 0.0;
            res->objective = builtin ? hs[5] : std::nan("");
            res->dJ_dmu = hs[0];
            res->device_ms = ms;
            res->kernel_launches = launches;
            res->status = conv ? IFC_OK : IFC_NOT_CONVERGED;
        }
        return conv ? IFC_OK : IFC_NOT_CONVERGED;
    }
    // mode 1: one reverse pass of the given lambda, no objective term
    double *dst[5] = {b.lu, b.lv, b.lp, b.luf, b.lvf};
    const size_t len[5] = {N, N, N, NU, NV};
    for (int q = 0; q < 5; ++q) {
        if (rq.seed[q]) CK(cudaMemcpyAsync(dst[q], rq.seed[q], len[q] * sizeof(double), cudaMemcpyHostToDevice, stream));
        else CK(cudaMemsetAsync(dst[q], 0, len[q] * sizeof(double), stream));
    }
    CK(cudaMemsetAsync(b.ju, 0, N * sizeof(double), stream));
    CK(cudaMemsetAsync(b.jv, 0, N * sizeof(double), stream));
    CK(cudaMemsetAsync(b.jp, 0, N * sizeof(double), stream));
    if (c.persist) {
        int rc = c.launch_persist(c.pargs(1, 1, 0.0));
        if (rc != IFC_OK) {
            err = c.err;
            return rc;
        }
    } else {
        CK(cudaGraphLaunch(c.x_tail, stream));
    }
    CK(cudaEventRecord(c.e1, stream));
    double *src[5] = {b.ou, b.ov, b.op, b.ouf, b.ovf};
    for (int q = 0; q < 5; ++q)
        if (rq.out[q]) CK(cudaMemcpyAsync(rq.out[q], src[q], len[q] * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (rq.dtheta) CK(cudaMemcpyAsync(rq.dtheta, b.ltheta, c.ny * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(hs, b.scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    CK(cudaGetLastError());
    if (c.persist) {
        bool to = false;
        if (c.barrier_error(to) != IFC_OK) {
            err = c.err;
            return IFC_CUDA_ERROR;
        }
        if (to) {
            err = "a grid barrier of the single-launch adjoint timed out";
            return IFC_TIMEOUT;
        }
    }
    if (rq.dmu) *rq.dmu = hs[0];
    if (res) {
        std::memset(res, 0, sizeof(*res));
        res->iterations = 1;
        res->dJ_dmu = hs[0];
        res->kernel_launches = launches + (c.persist ? 1 : c.per_pass);
    }
    return IFC_OK;
#undef CK
}

template int adjoint_run<float>(AdjointCtx *&, const ifc_config &, Params<double>, const Fields<float> &,
                                const float *, cudaStream_t, const AdjointReq &, ifc_adjoint_result *,
                                std::string &);
template int adjoint_run<double>(AdjointCtx *&, const ifc_config &, Params<double>, const Fields<double> &,
                                 const double *, cudaStream_t, const AdjointReq &, ifc_adjoint_result *,
                                 std::string &);

}  // namespace ifc
