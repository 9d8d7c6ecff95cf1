// ifc_fused2d.cuh -- fused, temporally blocked 2D kernels.
//
// Momentum pass: one CTA owns a TX x TY tile of cells and stages the tile plus
// a halo of H = 2*KS cells in shared memory; it assembles the momentum
// coefficients and sources of every staged cell (kernels.cuh:97-334, computed
// on the fly from the face velocities and the pressure; nothing but the
// diagonal aC is stored), then runs KS red-black Gauss-Seidel sweeps of u and
// v (which share one coefficient set) entirely in shared memory, and writes
// the tile back once.  Each half sweep invalidates one more ring of the halo,
// so after KS sweeps (2*KS half sweeps) the tile holds exactly the values KS
// global red-black sweeps produce.  The p' pass does the same for the
// pressure correction with the link coefficients built from aC on the fly
// (kernels.cuh:502-540).  Both accumulate the FP64 sum of squared changes of
// every sweep over the CTA's own tile and finish the inner early-exit rule
// (src/Solver.cu:955-962) after the pass.
//
// The Rhie-Chow kernel computes the face velocities, the face boundary
// conditions and the p' source of each cell in one pass (kernels.cuh:336-500,
// :47-95, :542-581).
#pragma once

#include "ifc_kernels.cuh"

namespace ifc {

template <typename T>
bool fused2d_supported(const Geo<T> &g)
{
    return g.dim == 2;
}

// Staged region geometry of a tile with a halo of H cells.
template <int TX, int TY, int H>
struct Region {
    static constexpr int W = TX + 2 * H;
    static constexpr int HH = TY + 2 * H;
    static constexpr int NR = W * HH;
    static constexpr int W1 = W - 2;                 // width of the updatable interior ring
    static constexpr int HW = (W1 + 1) / 2;          // cells of one colour per row (upper bound)
    static constexpr int NHALF = HW * (HH - 2);
};

// Local index of the q2-th cell of `color` in the updatable part (rows 1..HH-2,
// columns 1..W-2) of the region whose global origin is (gx0, gy0); returns -1
// when the slot falls outside the row.
template <int W, int HW>
__device__ __forceinline__ int colored_cell(int q2, int color, int gx0, int gy0)
{
    const int b = 1 + q2 / HW;
    const int k = q2 - (b - 1) * HW;
    const int a = 1 + ((color + gx0 + gy0 + b + 1) & 1) + 2 * k;
    if (a > W - 2) return -1;
    return b * W + a;
}

// Sweeps of a solve of n sweeps that fall into pass `pass` of KS sweeps each.
__host__ __device__ __forceinline__ int clamp_sweeps(int n, int pass, int ks)
{
    const int r = n - pass * ks;
    return r < 0 ? 0 : (r > ks ? ks : r);
}

// Tile shapes: FP32 tiles are 32 x 16 cells, FP64 tiles 32 x 8 (the staged
// region of an FP64 tile needs twice the shared memory per cell).
template <typename T>
struct TileShape2D {
    static constexpr int TX = 32, TY = sizeof(T) == 4 ? 16 : 8, NT = sizeof(T) == 4 ? 1024 : 512;
};

struct PassArgs {
    int ns[3];      // sweeps of each component in this pass
    int first;      // first pass of the solve (writes aC / starts p' from 0)
};

// Each thread owns up to CPT cells of each colour inside the updatable part of
// the staged region; their coefficients live in registers for the whole pass,
// so a half sweep only reads neighbour values from shared memory.
template <int W, int HH, int NHALF, int NT, int CPT>
__device__ __forceinline__ void own_cells(int tid, int gx0, int gy0, int nx, int ny, int (&cq)[2][CPT])
{
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int q2 = tid + k * NT;
            int q = q2 < NHALF ? colored_cell<W, (W - 1) / 2>(q2, c, gx0, gy0) : -1;
            if (q >= 0) {
                const int gi = gx0 + q % W, gj = gy0 + q / W;
                if (gi < 0 || gi >= nx || gj < 0 || gj >= ny) q = -1;
            }
            cq[c][k] = q;
        }
}

// Manhattan distance of region cell q from the tile [H, H+TX) x [H, H+TY).
// After half sweep h of a pass of 2*ns half sweeps only cells within distance
// 2*ns-1-h of the tile can still influence the tile's final values (each half
// sweep carries information one cell further), so cells farther out are not
// updated: the tile's result is unchanged, the redundant halo work shrinks.
template <int W, int H, int TX, int TY>
__device__ __forceinline__ int tile_distance(int q)
{
    if (q < 0) return 1 << 20;
    const int a = q % W, b = q / W;
    const int dx = a < H ? H - a : (a >= H + TX ? a - (H + TX - 1) : 0);
    const int dy = b < H ? H - b : (b >= H + TY ? b - (H + TY - 1) : 0);
    return dx + dy;
}

// ---- momentum: assembly + KS red-black sweeps of u and v -------------------
template <typename T, int TX, int TY, int KS, int NT>
__global__ void __launch_bounds__(NT) k_mom_pass2d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials, PassArgs pa,
                                                   const T *u_in, const T *v_in, T *u_out, T *v_out)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    const Geo<T> &g = P.g;
    bool act[2];
    act[0] = pa.ns[0] > 0 && !ctl->stop[EQ_U];
    act[1] = pa.ns[1] > 0 && !ctl->stop[EQ_V];

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *su = reinterpret_cast<T *>(smem_raw);
    T *sv = su + NR;
    T *sp = sv + NR;

    const int nx = g.nx, ny = g.ny;
    const int tiles_x = (nx + TX - 1) / TX;
    const int x0 = (blockIdx.x % tiles_x) * TX, y0 = (blockIdx.x / tiles_x) * TY;
    const int gx0 = x0 - H, gy0 = y0 - H;
    const int tid = threadIdx.x;

    for (int q = tid; q < NR; q += NT) {
        const int a = q % W, b = q / W;
        const int gi = gx0 + a, gj = gy0 + b;
        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        const int id = gi + nx * gj;
        su[q] = in ? u_in[id] : (T)0;
        sv[q] = in ? v_in[id] : (T)0;
        sp[q] = in ? f.p[id] : (T)0;
    }
    int cq[2][CPT];
    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
    __syncthreads();

    // Coefficients and sources of the owned cells (kernels.cuh:97-334).
    T cE[2][CPT], cW[2][CPT], cN[2][CPT], cS[2][CPT], cC[2][CPT], cbu[2][CPT], cbv[2][CPT];
    bool own[2][CPT];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int q = cq[c][k];
            own[c][k] = false;
            cE[c][k] = cW[c][k] = cN[c][k] = cS[c][k] = cbu[c][k] = cbv[c][k] = (T)0;
            cC[c][k] = (T)1;
            if (q < 0) continue;
            const int a = q % W, b = q / W;
            const int gi = gx0 + a, gj = gy0 + b;
            const int fu = gi + (nx + 1) * gj, fv = gi + nx * gj;
            T a7[7], b3[3];
            mom_cell<T, 2>(P, gi, gj, 0, f.uf[fu], f.uf[fu + 1], f.vf[fv], f.vf[fv + nx], (T)0, (T)0, sp[q],
                           sp[q - 1], sp[q + 1], sp[q - W], sp[q + W], (T)0, (T)0, a7, b3);
            add_dc<T, 2>(P, f, gi + nx * gj, b3);
            cE[c][k] = a7[AE];
            cW[c][k] = a7[AW];
            cN[c][k] = a7[AN];
            cS[c][k] = a7[AS];
            cC[c][k] = a7[AC];
            cbu[c][k] = b3[0];
            cbv[c][k] = b3[1];
            own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
            if (pa.first && own[c][k]) f.ac[gi + nx * gj] = a7[AC];
        }

    double acc[2][KS];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int s = 0; s < KS; ++s) acc[c][s] = 0.0;
    const T ru = g.relax[EQ_U], rv = g.relax[EQ_V];

    int dq[2][CPT];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) dq[c][k] = tile_distance<W, H, TX, TY>(cq[c][k]);
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        const bool du = act[0] && s < pa.ns[0];
        const bool dv = act[1] && s < pa.ns[1];
        if (!du && !dv) break;
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            const int hs = 2 * s + color;
#pragma unroll
            for (int k = 0; k < CPT; ++k) {
                const int q = cq[color][k];
                if (q < 0) continue;
                T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k], (T)0, (T)0};
                T d;
                const bool nu = du && dq[color][k] <= 2 * pa.ns[0] - 1 - hs;
                const bool nv = dv && dq[color][k] <= 2 * pa.ns[1] - 1 - hs;
                if (nu) {
                    su[q] = point_update<T, 2>(a7, cbu[color][k], su[q], su[q + 1], su[q - 1], su[q + W], su[q - W],
                                               (T)0, (T)0, ru, d);
                    if (own[color][k]) acc[0][s] += (double)d * (double)d;
                }
                if (nv) {
                    sv[q] = point_update<T, 2>(a7, cbv[color][k], sv[q], sv[q + 1], sv[q - 1], sv[q + W], sv[q - W],
                                               (T)0, (T)0, rv, d);
                    if (own[color][k]) acc[1][s] += (double)d * (double)d;
                }
            }
            __syncthreads();
        }
    }

    for (int q = tid; q < TX * TY; q += NT) {
        const int a = H + q % TX, b = H + q / TX;
        const int gi = gx0 + a, gj = gy0 + b;
        if (gi >= nx || gj >= ny) continue;
        const int id = gi + nx * gj;
        u_out[id] = su[b * W + a];
        v_out[id] = sv[b * W + a];
    }

    double flat[2 * KS];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int s = 0; s < KS; ++s) flat[c * KS + s] = acc[c][s];
    __shared__ double tot[2 * KS];
    if (grid_reduce<2 * KS>(flat, partials, ctl, tot) && tid == 0) {
        if (act[0]) finish_sweeps(ctl, EQ_U, tot, pa.ns[0], g.N, g.tol[EQ_U]);
        if (act[1]) finish_sweeps(ctl, EQ_V, tot + KS, pa.ns[1], g.N, g.tol[EQ_V]);
    }
}

// ---- pressure correction: KS red-black sweeps ------------------------------
template <typename T, int TX, int TY, int KS, int NT>
__global__ void __launch_bounds__(NT) k_pc_pass2d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials, PassArgs pa,
                                                  const T *pc_in, T *pc_out)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    const Geo<T> &g = P.g;
    const bool active = pa.ns[0] > 0 && !ctl->stop[EQ_P];  // same in every block

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sx = reinterpret_cast<T *>(smem_raw);  // p'
    T *sr = sx + NR;                           // 1 / aC of the momentum equations

    const int nx = g.nx, ny = g.ny;
    const int tiles_x = (nx + TX - 1) / TX;
    const int x0 = (blockIdx.x % tiles_x) * TX, y0 = (blockIdx.x / tiles_x) * TY;
    const int gx0 = x0 - H, gy0 = y0 - H;
    const int tid = threadIdx.x;

    for (int q = tid; q < NR; q += NT) {
        const int a = q % W, b = q / W;
        const int gi = gx0 + a, gj = gy0 + b;
        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        const int id = gi + nx * gj;
        sx[q] = (in && !pa.first) ? pc_in[id] : (T)0;
        sr[q] = in ? (T)1 / f.ac[id] : (T)0;
    }
    int cq[2][CPT];
    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
    __syncthreads();

    // Link coefficients of the owned cells, kernels.cuh:517-529: interior
    // faces only, -0.5 rho A^2 (1/aC_C + 1/aC_nb); boundary links stay 0.
    T cE[2][CPT], cW[2][CPT], cN[2][CPT], cS[2][CPT], cC[2][CPT], cb[2][CPT];
    bool own[2][CPT];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            const int q = cq[c][k];
            own[c][k] = false;
            cE[c][k] = cW[c][k] = cN[c][k] = cS[c][k] = cb[c][k] = (T)0;
            cC[c][k] = (T)1;
            if (q < 0) continue;
            const int a = q % W, b = q / W;
            const int gi = gx0 + a, gj = gy0 + b;
            const T r = sr[q];
            const T e = gi < nx - 1 ? (T)(P.d.Kx * (double)(T)(r + sr[q + 1])) : (T)0;
            const T w = gi > 0 ? (T)(P.d.Kx * (double)(T)(r + sr[q - 1])) : (T)0;
            const T n = gj < ny - 1 ? (T)(P.d.Ky * (double)(T)(r + sr[q + W])) : (T)0;
            const T so = gj > 0 ? (T)(P.d.Ky * (double)(T)(r + sr[q - W])) : (T)0;
            cE[c][k] = e;
            cW[c][k] = w;
            cN[c][k] = n;
            cS[c][k] = so;
            cC[c][k] = -(e + w + n + so);
            cb[c][k] = f.sp[gi + nx * gj];
            own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
        }

    double acc[KS];
#pragma unroll
    for (int s = 0; s < KS; ++s) acc[s] = 0.0;
    const T relax = g.relax[EQ_P];
    int dq[2][CPT];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) dq[c][k] = tile_distance<W, H, TX, TY>(cq[c][k]);
#pragma unroll
    for (int s = 0; s < KS; ++s) {
        if (!active || s >= pa.ns[0]) break;
#pragma unroll
        for (int color = 0; color < 2; ++color) {
            const int reach = 2 * pa.ns[0] - 1 - (2 * s + color);
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
        pc_out[gi + nx * gj] = sx[b * W + a];
    }
    if (!active) return;  // uniform: the copy above keeps the output buffer current

    __shared__ double tot[KS];
    if (grid_reduce<KS>(acc, partials, ctl, tot) && tid == 0) finish_sweeps(ctl, EQ_P, tot, pa.ns[0], g.N, g.tol[EQ_P]);
}

// ---- Rhie-Chow faces + face BCs + p' source + mass norm, one pass ----------
template <typename T>
__device__ __forceinline__ T rc_x(const Params<T> &P, const Fields<T> &f, int i, int row)
{
    const Geo<T> &g = P.g;
    const int R = i + g.nx * row, L = R - 1;
    const T pL = f.p[L], pR = f.p[R];
    const T pLL = i >= 2 ? f.p[L - 1] : (g.closed[WEST] ? pL : (T)0);
    const T pRR = i <= g.nx - 2 ? f.p[R + 1] : (g.closed[EAST] ? pR : (T)0);
    return rc_face(f.u[L], f.u[R], f.ac[L], f.ac[R], pLL, pL, pR, pRR, g.Ax);
}

template <typename T>
__device__ __forceinline__ T rc_y(const Params<T> &P, const Fields<T> &f, int i, int j)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx;
    const int R = i + nx * j, L = R - nx;
    const T pL = f.p[L], pR = f.p[R];
    const T pLL = j >= 2 ? f.p[L - nx] : (g.closed[SOUTH] ? pL : (T)0);
    const T pRR = j <= g.ny - 2 ? f.p[R + nx] : (g.closed[NORTH] ? pR : (T)0);
    return rc_face(f.v[L], f.v[R], f.ac[L], f.ac[R], pLL, pL, pR, pRR, g.Ay);
}

template <typename T>
__global__ void k_rc_mass2d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials)
{
    const Geo<T> &g = P.g;
    if (blockIdx.x == 0 && threadIdx.x == 0) reset_inner(ctl, 8);
    const int N = g.N, nx = g.nx, ny = g.ny;
    double s[1] = {0.0};
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) {
        const int i = c % nx, j = c / nx;
        const T uw = i == 0 ? face_bc(g, WEST, 0, f.u[c], j) : rc_x(P, f, i, j);
        const T ue = i == nx - 1 ? face_bc(g, EAST, 0, f.u[c], j) : rc_x(P, f, i + 1, j);
        const T vs = j == 0 ? face_bc(g, SOUTH, 1, f.v[c], 0) : rc_y(P, f, i, j);
        const T vn = j == ny - 1 ? face_bc(g, NORTH, 1, f.v[c], 0) : rc_y(P, f, i, j + 1);
        f.uf[i + (nx + 1) * j] = uw;
        if (i == nx - 1) f.uf[nx + (nx + 1) * j] = ue;
        f.vf[c] = vs;
        if (j == ny - 1) f.vf[c + nx] = vn;
        const T b = mass_imbalance<T, 2>(g, uw, ue, vs, vn, (T)0, (T)0);
        f.sp[c] = b;
        s[0] += (double)b * (double)b;
    }
    __shared__ double tot[1];
    if (grid_reduce<1>(s, partials, ctl, tot) && threadIdx.x == 0) ctl->sq[SQ_MASS] = tot[0];
}

}  // namespace ifc
