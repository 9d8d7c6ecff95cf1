// ifc_kernels.cuh -- per-step device kernels of the SIMPLE loop.
//
// These kernels restate one reference step each (kernels named in the
// comments) with grid-stride loops over cells or faces.  They are the 3D path
// and the single-step test path; the 2D hot path replaces the assembly and the
// sweeps with the fused, temporally blocked kernels of ifc_fused2d.cuh.  Every
// norm goes through the deterministic FP64 grid reduction of ifc_common.cuh.
#pragma once

#include "ifc_physics.cuh"
#include "ifc_convection.cuh"

namespace ifc {

// Reset the inner early-exit state of the equations in `mask` (bit q = eq q).
__device__ __forceinline__ void reset_inner(Ctl *ctl, int mask)
{
    for (int q = 0; q < 4; ++q)
        if (mask & (1 << q)) {
            ctl->stop[q] = 0;
            ctl->inner_max[q] = -1e20;
            ctl->sweeps[q] = 0;
        }
}

// Record the sweeps of one pass of equation e (sums of squared changes sq[s],
// s < ns) and apply the inner early-exit rule of src/Solver.cu:955-962 after
// each of them; the rule is evaluated only until it first fires.  Run by one
// thread: the control-block fields are read once, updated in registers and
// written back once, so the epilogue costs one round trip to L2, not one per
// field access.
__device__ __forceinline__ void finish_sweeps(Ctl *ctl, int e, const double *sq, int ns, int N, double tol)
{
    double mx = ctl->inner_max[e];
    int sw = ctl->sweeps[e];
    long long cu = ctl->cell_updates;
    bool stop_now = false;
    for (int s = 0; s < ns; ++s) {
        if (!stop_now) {
            const double rms = sqrt(sq[s] / (double)N);
            if (rms > mx) mx = rms;
            if (rms / (mx + 1e-20) < tol) stop_now = true;
        }
    }
    sw += ns;
    cu += (long long)ns * N;
    ctl->inner_max[e] = mx;
    ctl->sweeps[e] = sw;
    ctl->cell_updates = cu;
    if (ns > 0) ctl->last_sweep_sq[e] = sq[ns - 1];
    if (stop_now) ctl->stop[e] = 1;
}

// ---- face boundary conditions (+ first-iteration face init) ---------------
// kernels.cuh:10-45 (initFaceVelKernel, only while it == 0) and :47-95
// (applyBCsToFaceVelKernel).
template <typename T, int DIM>
__global__ void k_face_bc(Params<T> P, Fields<T> f, const Ctl *ctl)
{
    const Geo<T> &g = P.g;
    const bool init = (ctl->it == 0);
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const long long nuf = (long long)(nx + 1) * ny * nz, nvf = (long long)nx * (ny + 1) * nz;
    const long long nwf = DIM == 3 ? (long long)pl * (nz + 1) : 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nuf + nvf + nwf;
         q += (long long)gridDim.x * blockDim.x) {
        if (q < nuf) {
            int i = (int)(q % (nx + 1));
            int r = (int)(q / (nx + 1));          // j + ny*k
            int c = i + nx * r;
            if (i == 0) f.uf[q] = face_bc(g, WEST, 0, f.u[c], r);
            else if (i == nx) f.uf[q] = face_bc(g, EAST, 0, f.u[c - 1], r);
            else if (init) f.uf[q] = (f.u[c - 1] + f.u[c]) / (T)2;
        } else if (q < nuf + nvf) {
            long long qq = q - nuf;
            int i = (int)(qq % nx);
            int j = (int)((qq / nx) % (ny + 1));
            int k = (int)(qq / ((long long)nx * (ny + 1)));
            int c = i + nx * (j + ny * k);
            if (j == 0) f.vf[qq] = face_bc(g, SOUTH, 1, f.v[c], 0);
            else if (j == ny) f.vf[qq] = face_bc(g, NORTH, 1, f.v[c - nx], 0);
            else if (init) f.vf[qq] = (f.v[c - nx] + f.v[c]) / (T)2;
        } else {
            long long qq = q - nuf - nvf;        // equals the cell index of (i,j,k)
            int k = (int)(qq / pl);
            int c = (int)qq;
            if (k == 0) f.wf[qq] = face_bc(g, BOTTOM, 2, f.w[c], 0);
            else if (k == nz) f.wf[qq] = face_bc(g, TOP, 2, f.w[c - pl], 0);
            else if (init) f.wf[qq] = (f.w[c - pl] + f.w[c]) / (T)2;
        }
    }
}

// Load the inputs of mom_cell for cell c = (i,j,k) from global memory.
template <typename T, int DIM>
__device__ __forceinline__ void mom_cell_global(const Params<T> &P, const Fields<T> &f, int i, int j, int k,
                                                T (&a)[7], T (&b)[3])
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, pl = nx * ny;
    const int c = i + nx * (j + ny * k);
    const int fu = i + (nx + 1) * (j + ny * k);
    const int fv = i + nx * (j + (ny + 1) * k);
    T wb = (T)0, wt = (T)0, pB = (T)0, pT = (T)0;
    if (DIM == 3) {
        wb = f.wf[c];
        wt = f.wf[c + pl];
        pB = k > 0 ? f.p[c - pl] : (T)0;
        pT = k < g.nz - 1 ? f.p[c + pl] : (T)0;
    }
    mom_cell<T, DIM>(P, i, j, k, f.uf[fu], f.uf[fu + 1], f.vf[fv], f.vf[fv + nx], wb, wt, f.p[c],
                     i > 0 ? f.p[c - 1] : (T)0, i < nx - 1 ? f.p[c + 1] : (T)0,
                     j > 0 ? f.p[c - nx] : (T)0, j < ny - 1 ? f.p[c + nx] : (T)0, pB, pT, a, b);
    add_dc<T, DIM>(P, f, c, b);
}

// ---- FP64 momentum residuals (residual convergence rule) ------------------
// Sum of squares of b - aC phi - sum a_nb phi_nb of each momentum component
// at the start of the outer iteration, every product in FP64, for the
// per-field rule on residuals (ifc_config.criterion = IFC_CRIT_RESIDUAL): in
// FP32 the correction norms level off at the rounding noise of the corrected
// fields, the residual of the assembled equations does not.  A library
// addition; the reference tests its corrections only.
template <typename T, int DIM>
__global__ void __launch_bounds__(256) k_mom_residual(Params<T> P, Fields<T> f, Ctl *ctl, double *partials)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int units = row_units(nx, ny * nz);
    const T *phi[3] = {f.u, f.v, f.w};
    double sq[3] = {0.0, 0.0, 0.0};
    for (int u = gw; u < units; u += nw) {
        const RowUnit w = row_unit(u, nx, ny);
        const int j = w.j, k = w.k;
        for (int i = w.i0 + lane; i < w.i1; i += 32) {
            const int c = i + nx * w.r;
            T a[7], b[3];
            mom_cell_global<T, DIM>(P, f, i, j, k, a, b);
#pragma unroll
            for (int m = 0; m < DIM; ++m) {
                const T *x = phi[m];
                double r = (double)b[m] - (double)a[AC] * (double)x[c];
                if (i < nx - 1) r -= (double)a[AE] * (double)x[c + 1];
                if (i > 0) r -= (double)a[AW] * (double)x[c - 1];
                if (j < ny - 1) r -= (double)a[AN] * (double)x[c + nx];
                if (j > 0) r -= (double)a[AS] * (double)x[c - nx];
                if (DIM == 3) {
                    if (k < nz - 1) r -= (double)a[AT] * (double)x[c + pl];
                    if (k > 0) r -= (double)a[AB] * (double)x[c - pl];
                }
                sq[m] += r * r;
            }
        }
    }
    __shared__ double tot[3];
    if (grid_reduce<3>(sq, partials, ctl, tot) && threadIdx.x == 0)
        for (int m = 0; m < 3; ++m) ctl->res_sq[m] = tot[m];
}

// ---- momentum assembly (materialised) ------------------------------------
// kernels.cuh:97-134, :136-250, :252-334 for every cell; writes the coefficient
// planes, the diagonal and the sources.
template <typename T, int DIM>
__global__ void k_mom_assemble(Params<T> P, Fields<T> f, Ctl *ctl)
{
    const Geo<T> &g = P.g;
    if (blockIdx.x == 0 && threadIdx.x == 0) reset_inner(ctl, DIM == 3 ? 7 : 3);
    const int N = g.N, nx = g.nx, ny = g.ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        T a[7], b[3];
        mom_cell_global<T, DIM>(P, f, i, j, k, a, b);
        f.ac[c] = a[AC];
#pragma unroll
        for (int s = 0; s < 2 * DIM + 1; ++s) f.mc[c + (size_t)N * s] = a[s];
        f.su[c] = b[0];
        f.sv[c] = b[1];
        if (DIM == 3) f.sw[c] = b[2];
    }
}

// ---- linear sweeps on materialised coefficients ---------------------------
// kernels.cuh:845-1005.  color 0/1 runs one red-black half sweep (the black
// half completes the sweep); color -1 is a Jacobi sweep reading `old`.
// Up to three right-hand sides share one coefficient set (u, v, w).
template <typename T, int NC>
struct SweepArgs {
    const T *coef;
    T *phi[NC];
    const T *old[NC];
    const T *src[NC];
    int eq[NC];
    int active[NC];
    int color;
};

template <typename T, int DIM, int NC>
__global__ void k_sweep(Params<T> P, SweepArgs<T, NC> A, Ctl *ctl, double *partials)
{
    const Geo<T> &g = P.g;
    bool act[NC];
    bool any = false;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
        act[c] = A.active[c] && !ctl->stop[A.eq[c]];
        any = any || act[c];
    }
    if (!any) return;  // same decision in every block
    const int N = g.N, nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const int hx = (nx + 1) / 2;
    const long long count = A.color >= 0 ? (long long)hx * ny * nz : (long long)N;
    double sq[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) sq[c] = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < count;
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        if (A.color >= 0) {
            int i2 = (int)(q % hx);
            int r = (int)(q / hx);
            j = r % ny;
            k = r / ny;
            i = 2 * i2 + ((A.color + j + k) & 1);
            if (i >= nx) continue;
        } else {
            i = (int)(q % nx);
            j = (int)((q / nx) % ny);
            k = (int)(q / pl);
        }
        const int id = i + nx * (j + ny * k);
        T a[7];
        a[AC] = A.coef[id];
        a[AE] = A.coef[id + (size_t)N * AE];
        a[AW] = A.coef[id + (size_t)N * AW];
        a[AN] = A.coef[id + (size_t)N * AN];
        a[AS] = A.coef[id + (size_t)N * AS];
        a[AT] = DIM == 3 ? A.coef[id + (size_t)N * AT] : (T)0;
        a[AB] = DIM == 3 ? A.coef[id + (size_t)N * AB] : (T)0;
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (!act[c]) continue;
            const T *o = A.old[c];
            T pE = i != nx - 1 ? o[id + 1] : (T)0;
            T pW = i != 0 ? o[id - 1] : (T)0;
            T pN = j != ny - 1 ? o[id + nx] : (T)0;
            T pS = j != 0 ? o[id - nx] : (T)0;
            T pT = (DIM == 3 && k != nz - 1) ? o[id + pl] : (T)0;
            T pB = (DIM == 3 && k != 0) ? o[id - pl] : (T)0;
            T d;
            A.phi[c][id] = point_update<T, DIM>(a, A.src[c][id], o[id], pE, pW, pN, pS, pT, pB,
                                                g.relax[A.eq[c]], d);
            sq[c] += (double)d * (double)d;
        }
    }
    __shared__ double tot[NC];
    if (grid_reduce<NC>(sq, partials, ctl, tot) && threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
            if (!act[c]) continue;
            const int e = A.eq[c];
            if (A.color == 0) {
                ctl->half_sq[e] = tot[c];
            } else {
                double s = (A.color == 1 ? ctl->half_sq[e] : 0.0) + tot[c];
                finish_sweeps(ctl, e, &s, 1, N, g.tol[e]);
            }
        }
    }
}

// Jacobi helper: copy the active fields into their `old` buffers.
template <typename T, int NC>
__global__ void k_copy_active(SweepArgs<T, NC> A, const Ctl *ctl, int N)
{
    for (int c = 0; c < NC; ++c) {
        if (!A.active[c] || ctl->stop[A.eq[c]]) continue;
        T *dst = const_cast<T *>(A.old[c]);
        for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < N; q += gridDim.x * blockDim.x) dst[q] = A.phi[c][q];
    }
}

// ---- Rhie-Chow faces + face BCs -------------------------------------------
// kernels.cuh:336-500 on interior faces, then :47-95 on boundary faces with the
// momentum-solve velocities (src/Solver.cu:186-187).
template <typename T, int DIM>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 3) k_rhie_chow(Params<T> P, Fields<T> f)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int units = row_units(nx, ny * nz);
    for (int u = gw; u < units; u += nw) {
        const RowUnit w = row_unit(u, nx, ny);
        const int j = w.j, k = w.k, r = w.r, c0 = nx * r, f0 = (nx + 1) * r, v0 = nx * (j + (ny + 1) * k);
        for (int i = w.i0 + lane; i < w.i1; i += 32) {
            const int R = c0 + i;
            // x-face i of the row (west face of cell i)
            {
                const int L = R - 1;
                T val;
                if (i == 0) val = face_bc(g, WEST, 0, f.u[R], r);
                else {
                    T pL = f.p[L], pR = f.p[R];
                    T pLL = i >= 2 ? f.p[L - 1] : (g.closed[WEST] ? pL : (T)0);
                    T pRR = i <= nx - 2 ? f.p[R + 1] : (g.closed[EAST] ? pR : (T)0);
                    val = rc_face(f.u[L], f.u[R], f.ac[L], f.ac[R], pLL, pL, pR, pRR, g.Ax);
                }
                f.uf[f0 + i] = val;
                if (i == nx - 1) f.uf[f0 + nx] = face_bc(g, EAST, 0, f.u[R], r);
            }
            // y-face j of the column (south face of cell (i, j))
            {
                const int L = R - nx;
                T val;
                if (j == 0) val = face_bc(g, SOUTH, 1, f.v[R], 0);
                else {
                    T pL = f.p[L], pR = f.p[R];
                    T pLL = j >= 2 ? f.p[L - nx] : (g.closed[SOUTH] ? pL : (T)0);
                    T pRR = j <= ny - 2 ? f.p[R + nx] : (g.closed[NORTH] ? pR : (T)0);
                    val = rc_face(f.v[L], f.v[R], f.ac[L], f.ac[R], pLL, pL, pR, pRR, g.Ay);
                }
                f.vf[v0 + i] = val;
                if (j == ny - 1) f.vf[v0 + nx + i] = face_bc(g, NORTH, 1, f.v[R], 0);
            }
            // z-face k (bottom face of cell (i, j, k))
            if (DIM == 3) {
                const int L = R - pl;
                T val;
                if (k == 0) val = face_bc(g, BOTTOM, 2, f.w[R], 0);
                else {
                    T pL = f.p[L], pR = f.p[R];
                    T pLL = k >= 2 ? f.p[L - pl] : (g.closed[BOTTOM] ? pL : (T)0);
                    T pRR = k <= nz - 2 ? f.p[R + pl] : (g.closed[TOP] ? pR : (T)0);
                    val = rc_face(f.w[L], f.w[R], f.ac[L], f.ac[R], pLL, pL, pR, pRR, g.Az);
                }
                f.wf[R] = val;
                if (k == nz - 1) f.wf[R + pl] = face_bc(g, TOP, 2, f.w[R], 0);
            }
        }
    }
}

// ---- p' source and mass norm, kernels.cuh:542-581 --------------------------
template <typename T, int DIM>
__global__ void k_pcorr_src(Params<T> P, Fields<T> f, Ctl *ctl, double *partials)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int units = row_units(nx, ny * nz);
    double s[1] = {0.0};
    for (int u = gw; u < units; u += nw) {
        const RowUnit w = row_unit(u, nx, ny);
        const int c0 = nx * w.r, f0 = (nx + 1) * w.r, v0 = nx * (w.j + (ny + 1) * w.k);
        for (int i = w.i0 + lane; i < w.i1; i += 32) {
            const int c = c0 + i;
            T wb = DIM == 3 ? f.wf[c] : (T)0, wt = DIM == 3 ? f.wf[c + pl] : (T)0;
            T b = mass_imbalance<T, DIM>(g, f.uf[f0 + i], f.uf[f0 + i + 1], f.vf[v0 + i], f.vf[v0 + i + nx], wb, wt);
            f.sp[c] = b;
            s[0] += (double)b * (double)b;
        }
    }
    __shared__ double tot[1];
    if (grid_reduce<1>(s, partials, ctl, tot) && threadIdx.x == 0) ctl->sq[SQ_MASS] = tot[0];
}

// ---- p' link coefficients (materialised), kernels.cuh:502-540 --------------
template <typename T, int DIM>
__global__ void k_pcorr_coef(Params<T> P, Fields<T> f, Ctl *ctl)
{
    const Geo<T> &g = P.g;
    if (blockIdx.x == 0 && threadIdx.x == 0) reset_inner(ctl, 8);
    const int N = g.N, nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        int i = c % nx, j = (c / nx) % ny, k = c / pl;
        T cc = f.ac[c];
        T aE = i < nx - 1 ? pcorr_link(P.d.Kx, cc, f.ac[c + 1]) : (T)0;
        T aW = i > 0 ? pcorr_link(P.d.Kx, cc, f.ac[c - 1]) : (T)0;
        T aN = j < ny - 1 ? pcorr_link(P.d.Ky, cc, f.ac[c + nx]) : (T)0;
        T aS = j > 0 ? pcorr_link(P.d.Ky, cc, f.ac[c - nx]) : (T)0;
        T aC = -(aE + aW + aN + aS);
        f.pcoef[c + (size_t)N * AE] = aE;
        f.pcoef[c + (size_t)N * AW] = aW;
        f.pcoef[c + (size_t)N * AN] = aN;
        f.pcoef[c + (size_t)N * AS] = aS;
        if (DIM == 3) {
            T aT = k < nz - 1 ? pcorr_link(P.d.Kz, cc, f.ac[c + pl]) : (T)0;
            T aB = k > 0 ? pcorr_link(P.d.Kz, cc, f.ac[c - pl]) : (T)0;
            f.pcoef[c + (size_t)N * AT] = aT;
            f.pcoef[c + (size_t)N * AB] = aB;
            aC += -(aT + aB);
        }
        f.pcoef[c] = aC;
    }
}

// ---- pressure-reference pinning (closed domains) ---------------------------
template <typename T>
__global__ void k_pc_sum(const T *pc, int N, Ctl *ctl, double *partials)
{
    double s[1] = {0.0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) s[0] += (double)pc[c];
    __shared__ double tot[1];
    if (grid_reduce<1>(s, partials, ctl, tot) && threadIdx.x == 0) ctl->sq[SQ_PCSUM] = tot[0];
}

template <typename T>
__global__ void k_pc_shift(T *pc, int N, const Ctl *ctl)
{
    const double mean = ctl->sq[SQ_PCSUM] / (double)N;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x)
        pc[c] = (T)((double)pc[c] - mean);
}

// ---- end of an outer iteration: norms, convergence, log, loop condition ----
// src/Solver.cu:226-289.
template <typename T>
__device__ void finish_iteration(const Geo<T> &g, Ctl *ctl, const double *tot, cudaGraphConditionalHandle cond,
                                 int use_cond)
{
    // Read every control field this epilogue needs at once (one L2 round
    // trip), work in registers, write back at the end.
    const double mass_sq = ctl->sq[SQ_MASS];
    const int it0 = ctl->it, it_begin = ctl->it_begin, it_stop = ctl->it_stop, act = ctl->act;
    const int log_level = ctl->log_level, log_n = ctl->log_n;
    const int status0 = ctl->status;  // 3: a bounded wait of this iteration gave up
    double maxn[8];
    int sweeps[4];
#pragma unroll
    for (int q = 0; q < 8; ++q) maxn[q] = ctl->maxn[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) sweeps[q] = ctl->sweeps[q];

    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const double N = (double)g.N;
    const bool d3 = g.dim == 3;
    double n[8];
    n[0] = sqrt(tot[0] / N);
    n[1] = sqrt(tot[1] / N);
    n[2] = sqrt(tot[2] / N);
    n[3] = d3 ? sqrt(tot[3] / N) : 0.0;
    n[4] = sqrt(tot[4] / ((double)(nx - 1) * ny * nz));
    n[5] = sqrt(tot[5] / ((double)nx * (ny - 1) * nz));
    n[6] = d3 ? sqrt(tot[6] / ((double)nx * ny * (nz - 1))) : 0.0;
    n[7] = sqrt(mass_sq / N);
    bool bad = false;
#pragma unroll
    for (int q = 0; q < 8; ++q) bad = bad || !isfinite(n[q]);
    const int it = it0 + 1;
    if (!bad && it - it_begin > 1)
#pragma unroll
        for (int q = 0; q < 7; ++q) bad = bad || (maxn[q] > 0.0 && n[q] > 1e6 * maxn[q]);
    double rel[7];
    double rmax[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) rmax[q] = ctl->rmax[q];
    if (g.criterion == 2) {
        // per field on the FP64 residuals: u, v, w by their momentum residual,
        // p by the mass imbalance; the faces follow from u and p
        const double r[4] = {sqrt(ctl->res_sq[0] / N), sqrt(ctl->res_sq[1] / N), d3 ? sqrt(ctl->res_sq[2] / N) : 0.0,
                             n[7]};
        double rr[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (r[q] > rmax[q]) rmax[q] = r[q];
            rr[q] = rmax[q] > 0.0 ? r[q] / rmax[q] : 0.0;
        }
        rel[0] = rr[3];
        rel[1] = rr[0];
        rel[2] = rr[1];
        rel[3] = d3 ? rr[2] : 0.0;
        rel[4] = rel[5] = rel[6] = 0.0;
    } else if (g.criterion == 0) {
        // src/Solver.cu:237-256: all relative norms use the running max of the
        // pressure norm.
        if (n[0] > maxn[0]) maxn[0] = n[0];
#pragma unroll
        for (int q = 0; q < 7; ++q) rel[q] = n[q] / maxn[0];
    } else {
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            if (!d3 && (q == 3 || q == 6)) {
                rel[q] = 0.0;
                continue;
            }
            if (n[q] > maxn[q]) maxn[q] = n[q];
            rel[q] = maxn[q] > 0.0 ? n[q] / maxn[q] : 0.0;
        }
    }
    // src/Solver.cu:258-268 (p, u, v, uf, vf [, w, wf]) or the mass norm.
    bool conv = rel[0] < g.tol[EQ_P] && rel[1] < g.tol[EQ_U] && rel[2] < g.tol[EQ_V] && rel[4] < g.tol[EQ_U] &&
                rel[5] < g.tol[EQ_V];
    if (d3) conv = conv && rel[3] < g.tol[EQ_W] && rel[6] < g.tol[EQ_W];
    conv = conv || n[7] < g.tol_mass;
    const int local = it - it_begin;
    const bool last = it >= it_stop || (act && conv) || bad || status0 == 3;

#pragma unroll
    for (int q = 0; q < 7; ++q) ctl->sq[q] = tot[q];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        ctl->norm[q] = n[q];
        ctl->maxn[q] = maxn[q];
    }
#pragma unroll
    for (int q = 0; q < 7; ++q) ctl->rel[q] = rel[q];
#pragma unroll
    for (int q = 0; q < 4; ++q) ctl->rmax[q] = rmax[q];
    ctl->it = it;
    ctl->converged = conv ? 1 : 0;
    if (bad) ctl->status = 2;
    if (log_level > 0 && (local == 1 || local % 1000 == 0 || conv || last)) {
        const int slot = log_n < kLogCap ? log_n : kLogCap - 1;
        LogRec &L = ctl->log[slot];
        L.it = local;
        L.converged = conv;
#pragma unroll
        for (int q = 0; q < 7; ++q) L.rel[q] = rel[q];
        L.mass = n[7];
        if (log_n < kLogCap) ctl->log_n = log_n + 1;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) ctl->it_sweeps[q] = sweeps[q];
    reset_inner(ctl, 15);
    if (use_cond) cudaGraphSetConditional(cond, last ? 0u : 1u);
}

// ---- corrections, kernels.cuh:583-843 ---------------------------------------
// 64 registers (4 blocks of 256 per SM): the loads-first body otherwise takes
// ~100 and halves the warps in flight of this memory-bound kernel.
template <typename T, int DIM>
__global__ void __launch_bounds__(256, 4) k_update(Params<T> P, Fields<T> f, Ctl *ctl, double *partials, cudaGraphConditionalHandle cond,
                         int use_cond)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int units = row_units(nx, ny * nz);
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int u = gw; u < units; u += nw) {
        const RowUnit w = row_unit(u, nx, ny);
        const int j = w.j, k = w.k, r = w.r, c0 = nx * r, f0 = (nx + 1) * r, v0 = nx * (j + (ny + 1) * k);
        for (int i = w.i0 + lane; i < w.i1; i += 32) {
            const int c = c0 + i;
            // every load of the cell first: no store below can alias them
            const T pc = f.pc[c], aC = f.ac[c];
            const T pcW = i > 0 ? f.pc[c - 1] : (T)0, pcE = i < nx - 1 ? f.pc[c + 1] : (T)0;
            const T pcS = j > 0 ? f.pc[c - nx] : (T)0, pcN = j < ny - 1 ? f.pc[c + nx] : (T)0;
            const T acW = i > 0 ? f.ac[c - 1] : (T)1, acS = j > 0 ? f.ac[c - nx] : (T)1;
            const T p0 = f.p[c], u0 = f.u[c], v0c = f.v[c];
            const T uf0 = i > 0 ? f.uf[f0 + i] : (T)0, vf0 = j > 0 ? f.vf[v0 + i] : (T)0;
            T pcB = (T)0, pcT = (T)0, acB = (T)1, w0 = (T)0, wf0 = (T)0;
            if (DIM == 3) {
                pcB = k > 0 ? f.pc[c - pl] : (T)0;
                pcT = k < nz - 1 ? f.pc[c + pl] : (T)0;
                acB = k > 0 ? f.ac[c - pl] : (T)1;
                w0 = f.w[c];
                wf0 = k > 0 ? f.wf[c] : (T)0;
            }
            const T dp = g.relax[EQ_P] * pc;
            f.p[c] = p0 + dp;
            s[0] += (double)dp * (double)dp;
            T L = i > 0 ? pcW : (g.closed[WEST] ? pc : (T)0);
            T R = i < nx - 1 ? pcE : (g.closed[EAST] ? pc : (T)0);
            T d = vel_corr(P.d.ru[0], L, R, g.Ax, aC);
            const T un = u0 + d;
            f.u[c] = un;
            s[1] += (double)d * (double)d;
            // Boundary faces of the next outer iteration (kernels.cuh:47-95 with
            // the corrected velocities, src/Solver.cu:165).
            if (i == 0) f.uf[f0] = face_bc(g, WEST, 0, un, r);
            if (i == nx - 1) f.uf[f0 + nx] = face_bc(g, EAST, 0, un, r);
            L = j > 0 ? pcS : (g.closed[SOUTH] ? pc : (T)0);
            R = j < ny - 1 ? pcN : (g.closed[NORTH] ? pc : (T)0);
            d = vel_corr(P.d.ru[1], L, R, g.Ay, aC);
            const T vn = v0c + d;
            f.v[c] = vn;
            s[2] += (double)d * (double)d;
            if (j == 0) f.vf[v0 + i] = face_bc(g, SOUTH, 1, vn, 0);
            if (j == ny - 1) f.vf[v0 + nx + i] = face_bc(g, NORTH, 1, vn, 0);
            if (DIM == 3) {
                L = k > 0 ? pcB : (g.closed[BOTTOM] ? pc : (T)0);
                R = k < nz - 1 ? pcT : (g.closed[TOP] ? pc : (T)0);
                d = vel_corr(P.d.ru[2], L, R, g.Az, aC);
                const T wn = w0 + d;
                f.w[c] = wn;
                s[3] += (double)d * (double)d;
                if (k == 0) f.wf[c] = face_bc(g, BOTTOM, 2, wn, 0);
                if (k == nz - 1) f.wf[c + pl] = face_bc(g, TOP, 2, wn, 0);
            }
            if (i >= 1) {
                d = face_corr(P.d.ru[0], acW, aC, pcW, pc, g.Ax);
                f.uf[f0 + i] = uf0 + d;
                s[4] += (double)d * (double)d;
            }
            if (j >= 1) {
                d = face_corr(P.d.ru[1], acS, aC, pcS, pc, g.Ay);
                f.vf[v0 + i] = vf0 + d;
                s[5] += (double)d * (double)d;
            }
            if (DIM == 3 && k >= 1) {
                d = face_corr(P.d.ru[2], acB, aC, pcB, pc, g.Az);
                f.wf[c] = wf0 + d;
                s[6] += (double)d * (double)d;
            }
        }
    }
    __shared__ double tot[7];
    if (grid_reduce<7>(s, partials, ctl, tot) && threadIdx.x == 0) finish_iteration(g, ctl, tot, cond, use_cond);
}

// ---- small helpers ---------------------------------------------------------
template <typename T>
__global__ void k_fill(T *x, long long n, T v)
{
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        x[q] = v;
}

static __global__ void k_begin(Ctl *ctl, int n_iter, int act, int log_level)
{
    ctl->it_begin = ctl->it;
    ctl->it_stop = ctl->it + n_iter;
    ctl->act = act;
    ctl->converged = 0;
    ctl->status = 0;
    ctl->log_n = 0;
    ctl->log_level = log_level;
    ctl->cell_updates = 0;
    ctl->counter = 0;
    reset_inner(ctl, 15);
}

static __global__ void k_reset_inner(Ctl *ctl, int mask) { reset_inner(ctl, mask); }
static __global__ void k_reset_inner_p(Ctl *ctl) { reset_inner(ctl, 8); }

}  // namespace ifc
