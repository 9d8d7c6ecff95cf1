// ifc_energy.cuh -- steady temperature transport on the converged flow.
//
// The reference allocates the temperature, carries its boundary conditions
// (TempBCs, include/config.h:45-63) and thermal properties
// (include/config.h:19-23) and writes it to VTK, but never solves for it.
// Here the steady energy equation
//     div(rho u T) = div(Gamma grad T),   Gamma = thermalConductivity / specificHeatCapacity
// (so Gamma / rho is the reference's thermalDiffusivity) is discretised on the
// converged face mass fluxes exactly as the momentum equations are: first-order
// upwind convection and central diffusion links (kernels.cuh:97-134 with Gamma
// in place of mu), and the boundary fold-in of kernels.cuh:252-334 -- the
// wall/inlet form for a Dirichlet face (type 0, the given temperature) and
// the zero-gradient form for a Neumann face (type 1).  The linear system is
// solved with the library's red-black Gauss-Seidel sweep kernel, unrelaxed.
// With a higher-order convection scheme (ifc_convection.cuh) the links stay
// upwind and the deferred correction of the current temperature is added to
// the source at the start of every cycle of sweeps (k_temp_dc).
#pragma once

#include "ifc_persist2d.cuh"

namespace ifc {

template <typename T>
struct TempArgs {
    T Dx, Dy, Dz;  // Gamma * A / d per direction, evaluated in the scalar type
    int type[6];   // 0 Dirichlet, 1 Neumann (zero gradient)
    T val[6];
};

template <typename T, int DIM>
__device__ __forceinline__ void temp_fold(const Params<T> &P, const TempArgs<T> &ta, int face, int ex, int in,
                                          T (&a)[7], T &b)
{
    const T e = a[ex];
    if (ta.type[face] != 0) {
        a[AC] = a[AC] + e;
        a[ex] = (T)0;
        return;
    }
    a[AC] = a[AC] - (T)2 * e;
    a[in] = a[in] + e / (T)3;
    b = b - P.d.c83 * e * ta.val[face];
    a[ex] = (T)0;
}

// Coefficient planes (2*DIM+1, coef[cell + N*slot]) and source of the energy
// equation of every cell.
template <typename T, int DIM>
__global__ void k_temp_assemble(Params<T> P, Fields<T> f, TempArgs<T> ta, T *coef, T *src)
{
    const Geo<T> &g = P.g;
    const int N = g.N, nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        const int i = c % nx, j = (c / nx) % ny, k = c / pl;
        const int fu = i + (nx + 1) * (j + ny * k), fv = i + nx * (j + (ny + 1) * k);
        const T ue = f.uf[fu + 1], uw = f.uf[fu], vn = f.vf[fv + nx], vs = f.vf[fv];
        T a[7];
        a[AE] = g.rho * min0(ue) * g.Ax - ta.Dx;
        a[AW] = g.rho * min0(-uw) * g.Ax - ta.Dx;
        a[AN] = g.rho * min0(vn) * g.Ay - ta.Dy;
        a[AS] = g.rho * min0(-vs) * g.Ay - ta.Dy;
        a[AC] = -(a[AE] + a[AW] + a[AN] + a[AS]);
        a[AT] = (T)0;
        a[AB] = (T)0;
        if (DIM == 3) {
            const T wt = f.wf[c + pl], wb = f.wf[c];
            a[AT] = g.rho * min0(wt) * g.Az - ta.Dz;
            a[AB] = g.rho * min0(-wb) * g.Az - ta.Dz;
            a[AC] += -(a[AT] + a[AB]);
        }
        T b = (T)0;
        if (i == nx - 1) temp_fold<T, DIM>(P, ta, EAST, AE, AW, a, b);
        if (i == 0) temp_fold<T, DIM>(P, ta, WEST, AW, AE, a, b);
        if (j == ny - 1) temp_fold<T, DIM>(P, ta, NORTH, AN, AS, a, b);
        if (j == 0) temp_fold<T, DIM>(P, ta, SOUTH, AS, AN, a, b);
        if (DIM == 3) {
            if (k == nz - 1) temp_fold<T, DIM>(P, ta, TOP, AT, AB, a, b);
            if (k == 0) temp_fold<T, DIM>(P, ta, BOTTOM, AB, AT, a, b);
        }
#pragma unroll
        for (int s = 0; s < 2 * DIM + 1; ++s) coef[c + (size_t)N * s] = a[s];
        src[c] = b;
    }
}

// src_eff = src + the deferred-correction source of the current temperature
// (same face fluxes and limiter as the momentum equations).
template <typename T, int DIM>
__global__ void k_temp_dc(Params<T> P, Fields<T> f, const T *src, T *src_eff)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, pl = nx * ny;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int units = row_units(nx, ny * g.nz);
    for (int u = gw; u < units; u += nw) {
        const RowUnit w = row_unit(u, nx, ny);
        const int c0 = nx * w.r, f0 = (nx + 1) * w.r, v0 = nx * (w.j + (ny + 1) * w.k);
        for (int i = w.i0 + lane; i < w.i1; i += 32) {
            const int c = c0 + i;
            const T wb = DIM == 3 ? f.wf[c] : (T)0, wt = DIM == 3 ? f.wf[c + pl] : (T)0;
            const T d = dc_cell<T, DIM>(g, f.temp, c, i, w.j, w.k, f.uf[f0 + i], f.uf[f0 + i + 1], f.vf[v0 + i],
                                        f.vf[v0 + i + nx], wb, wt);
            src_eff[c] = src[c] + d;
        }
    }
}

static __global__ void k_clear_stop(Ctl *ctl, int eq) { ctl->stop[eq] = 0; }

// ---- 2D: a cycle of sweeps on stored coefficients in one cooperative launch --
// The passes of k_coef_pass2d (below) with one tile per CTA, all CTAs
// co-resident: the coefficients are read into registers once per cycle, the
// passes are separated by the bounded grid barrier of ifc_persist2d.cuh, and
// after each pass every CTA reduces the per-sweep FP64 sums (double-buffered
// by pass parity, so a CTA that runs ahead cannot overwrite sums another is
// still reading) and applies the inner early-exit rule exactly as
// finish_sweeps does.  The result is left in x0.  Values equal those of the
// per-pass launches.
template <typename T, int TX, int TY, int KS, int NT>
__global__ void __launch_bounds__(NT) k_coef_solve2d(Params<T> P, const T *coef, const T *src, Ctl *ctl,
                                                     double *partials, GridBarrier *bar, int eq, int nsweeps, T *x0,
                                                     T *x1, int stall_test)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N, G = gridDim.x;
    const int tiles_x = (nx + TX - 1) / TX;
    const int x0t = (blockIdx.x % tiles_x) * TX, y0t = (blockIdx.x / tiles_x) * TY;
    const int gx0 = x0t - H, gy0 = y0t - H;
    const int tid = threadIdx.x;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sx = reinterpret_cast<T *>(smem_raw);
    __shared__ double wred[NT / 32][KS];
    __shared__ double tot[KS];
    __shared__ int s_stop;

    int cq[2][CPT], dq[2][CPT];
    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
    T cE[2][CPT], cW[2][CPT], cN[2][CPT], cS[2][CPT], cC[2][CPT], cb[2][CPT];
    bool own[2][CPT];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int q = cq[c][k];
            dq[c][k] = tile_distance<W, H, TX, TY>(q);
            own[c][k] = false;
            cE[c][k] = cW[c][k] = cN[c][k] = cS[c][k] = cb[c][k] = (T)0;
            cC[c][k] = (T)1;
            if (q < 0) continue;
            const int a = q % W, b = q / W;
            const int id = gx0 + a + nx * (gy0 + b);
            cC[c][k] = coef[id + (size_t)N * AC];
            cE[c][k] = coef[id + (size_t)N * AE];
            cW[c][k] = coef[id + (size_t)N * AW];
            cN[c][k] = coef[id + (size_t)N * AN];
            cS[c][k] = coef[id + (size_t)N * AS];
            cb[c][k] = src[id];
            own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
        }
    double mx = ctl->inner_max[eq];
    int sw = ctl->sweeps[eq];
    long long cu = ctl->cell_updates;
    double last_sq = ctl->last_sweep_sq[eq];
    if (tid == 0) s_stop = ctl->stop[eq];
    __syncthreads();
    bool stop = s_stop != 0;
    bool failed = false;
    unsigned int epoch = 0;
    T *buf[2] = {x0, x1};
    int cur = 0;
    const T relax = g.relax[eq];

    for (int pass = 0; pass * KS < nsweeps && !stop; ++pass) {
        // Failure-detection test (stall_test = 1): CTA 0 leaves without
        // arriving, so every other CTA's bounded wait at this pass's barrier
        // runs out and the launch ends with the timeout status.
        if (stall_test && blockIdx.x == 0) { failed = true; break; }
        const int ns = clamp_sweeps(nsweeps, pass, KS);
        for (int q = tid; q < NR; q += NT) {
            const int a = q % W, b = q / W;
            const int gi = gx0 + a, gj = gy0 + b;
            const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
            sx[q] = in ? buf[cur][gi + nx * gj] : (T)0;
        }
        __syncthreads();
#pragma unroll 1
        for (int s = 0; s < KS; ++s) {
            if (s >= ns) break;
            double acc = 0.0;
#pragma unroll
            for (int color = 0; color < 2; ++color) {
                const int reach = 2 * ns - 1 - (2 * s + color);
#pragma unroll
                for (int k = 0; k < CPT; ++k) {
                    const int q = cq[color][k];
                    if (q < 0 || dq[color][k] > reach) continue;
                    T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k], (T)0, (T)0};
                    T d;
                    sx[q] = point_update<T, 2>(a7, cb[color][k], sx[q], sx[q + 1], sx[q - 1], sx[q + W], sx[q - W],
                                               (T)0, (T)0, relax, d);
                    if (own[color][k]) acc += (double)d * (double)d;
                }
                __syncthreads();
            }
            acc = warp_sum(acc);
            if ((tid & 31) == 0) wred[tid >> 5][s] = acc;
        }
        for (int q = tid; q < TX * TY; q += NT) {
            const int a = H + q % TX, b = H + q / TX;
            const int gi = gx0 + a, gj = gy0 + b;
            if (gi >= nx || gj >= ny) continue;
            buf[cur ^ 1][gi + nx * gj] = sx[b * W + a];
        }
        cur ^= 1;
        double *part = partials + (size_t)(pass & 1) * KS * G;
        block_partials<KS, KS, NT>(&wred[0][0], part, G);
        if (!grid_sync(bar, G, epoch)) { failed = true; break; }
        reduce_partials<KS, NT>(part, G, tot);
        // the rule of finish_sweeps, evaluated identically in every CTA
        bool stop_now = false;
        for (int s = 0; s < ns; ++s) {
            if (stop_now) break;
            const double rms = sqrt(tot[s] / (double)N);
            if (rms > mx) mx = rms;
            if (rms / (mx + 1e-20) < g.tol[eq]) stop_now = true;
        }
        sw += ns;
        cu += (long long)ns * N;
        last_sq = tot[ns - 1];
        stop = stop_now;
        __syncthreads();  // tot is rewritten only after the next pass's barrier
    }
    if (!failed && cur == 1)  // the last pass staged from x0, and every CTA has passed its barrier
        for (int q = tid; q < TX * TY; q += NT) {
            const int gi = x0t + q % TX, gj = y0t + q / TX;
            if (gi < nx && gj < ny) x0[gi + nx * gj] = x1[gi + nx * gj];
        }
    if (blockIdx.x == 0 && tid == 0 && !failed) {
        ctl->inner_max[eq] = mx;
        ctl->sweeps[eq] = sw;
        ctl->cell_updates = cu;
        ctl->last_sweep_sq[eq] = last_sq;
        if (stop) ctl->stop[eq] = 1;
    }
    if (tid == 0 && (failed || bar->err)) atomicExch(&ctl->status, 3);
}

// ---- 2D: KS red-black sweeps on stored coefficients in one pass ------------
// The temporally blocked pass of ifc_fused2d.cuh for a linear system whose
// coefficient planes (coef[cell + N*slot], slots aC aE aW aN aS) and source
// are stored: the tile plus a halo of 2*KS cells is staged from x_in, every
// thread keeps its cells' coefficients in registers, and the tile after KS
// sweeps goes to x_out (a different buffer, so no tile reads a neighbour's
// values of the same pass).  Per-sweep FP64 sums of the owned cells feed the
// inner early-exit rule of equation eq after the pass (finish_sweeps).  Used
// by the energy solve; the values equal those of per-sweep red-black launches.
template <typename T, int TX, int TY, int KS, int NT>
__global__ void __launch_bounds__(NT) k_coef_pass2d(Params<T> P, const T *coef, const T *src, Ctl *ctl,
                                                    double *partials, int eq, int ns, const T *x_in, T *x_out)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    const Geo<T> &g = P.g;
    const bool active = ns > 0 && !ctl->stop[eq];  // same in every block

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sx = reinterpret_cast<T *>(smem_raw);

    const int nx = g.nx, ny = g.ny, N = g.N;
    const int tiles_x = (nx + TX - 1) / TX;
    const int x0 = (blockIdx.x % tiles_x) * TX, y0 = (blockIdx.x / tiles_x) * TY;
    const int gx0 = x0 - H, gy0 = y0 - H;
    const int tid = threadIdx.x;

    for (int q = tid; q < NR; q += NT) {
        const int a = q % W, b = q / W;
        const int gi = gx0 + a, gj = gy0 + b;
        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        sx[q] = in ? x_in[gi + nx * gj] : (T)0;
    }
    int cq[2][CPT], dq[2][CPT];
    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
    T cE[2][CPT], cW[2][CPT], cN[2][CPT], cS[2][CPT], cC[2][CPT], cb[2][CPT];
    bool own[2][CPT];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int q = cq[c][k];
            dq[c][k] = tile_distance<W, H, TX, TY>(q);
            own[c][k] = false;
            cE[c][k] = cW[c][k] = cN[c][k] = cS[c][k] = cb[c][k] = (T)0;
            cC[c][k] = (T)1;
            if (q < 0) continue;
            const int a = q % W, b = q / W;
            const int id = gx0 + a + nx * (gy0 + b);
            cC[c][k] = coef[id + (size_t)N * AC];
            cE[c][k] = coef[id + (size_t)N * AE];
            cW[c][k] = coef[id + (size_t)N * AW];
            cN[c][k] = coef[id + (size_t)N * AN];
            cS[c][k] = coef[id + (size_t)N * AS];
            cb[c][k] = src[id];
            own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
        }
    __syncthreads();

    double acc[KS];
#pragma unroll
    for (int s = 0; s < KS; ++s) acc[s] = 0.0;
    const T relax = g.relax[eq];
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        if (!active || s >= ns) break;
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            const int reach = 2 * ns - 1 - (2 * s + color);
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int q = cq[color][k];
                if (q < 0 || dq[color][k] > reach) continue;
                T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k], (T)0, (T)0};
                T d;
                sx[q] = point_update<T, 2>(a7, cb[color][k], sx[q], sx[q + 1], sx[q - 1], sx[q + W], sx[q - W],
                                           (T)0, (T)0, relax, d);
                if (own[color][k]) acc[s] += (double)d * (double)d;
            }
            __syncthreads();
        }
    }
    for (int q = tid; q < TX * TY; q += NT) {
        const int a = H + q % TX, b = H + q / TX;
        const int gi = gx0 + a, gj = gy0 + b;
        if (gi >= nx || gj >= ny) continue;
        x_out[gi + nx * gj] = sx[b * W + a];
    }
    if (!active) return;  // uniform: the copy above keeps the output buffer current

    __shared__ double tot[KS];
    if (grid_reduce<KS>(acc, partials, ctl, tot) && tid == 0) finish_sweeps(ctl, eq, tot, ns, N, g.tol[eq]);
}

}  // namespace ifc
