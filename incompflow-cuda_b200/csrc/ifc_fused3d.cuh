// ifc_fused3d.cuh -- 3D red-black half sweeps with on-the-fly coefficients.
//
// The reference streams 7 coefficient planes per cell and sweep
// (include/kernels.cuh:926-1005 reading the planes written by :97-334 and
// :502-540).  Here the momentum half sweep rebuilds the coefficients, the
// pressure source and the boundary fold-in of each cell from its six face
// velocities and seven pressures (mom_cell), and sweeps u, v and w together
// (they share the coefficients); the p' half sweep builds its six links from
// the reciprocals 1/aC of the cell and its neighbours (kernels.cuh:518-537),
// stored once per outer iteration.  Same arithmetic as ifc_physics.cuh, so
// the results are bit-identical to the per-step kernels and the CPU oracle.
#pragma once

#include "ifc_kernels.cuh"
#include "ifc_persist2d.cuh"

namespace ifc {

struct Half3D {
    int color;      // 0 red, 1 black (completes the sweep)
    int active[3];  // component takes part in this sweep (s < n_iter)
    int first;      // first sweep of the solve: store aC
};

// Bound to 40 registers in FP32 (6 blocks of 256 per SM): the half sweep is
// bound by the latency of its ~34 cached loads per cell, and the extra warps
// in flight took it from 34.5 to 27.8 us at 128^3.
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 3) k_mom_half3d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials, Half3D h)
{
    const Geo<T> &g = P.g;
    bool act[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) act[c] = h.active[c] && !ctl->stop[c];
    if (!act[0] && !act[1] && !act[2] && !h.first) return;  // uniform
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny, N = g.N;
    const int nrows = ny * nz, lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nwg = (int)((gridDim.x * blockDim.x) >> 5);
    T *phi[3] = {f.u, f.v, f.w};
    double sq[3] = {0.0, 0.0, 0.0};
    // one warp per x-row, lanes over the row's cells of this colour
    for (int r = gw; r < nrows; r += nwg) {
        const int j = r % ny, k = r / ny;
        for (int i = ((h.color + j + k) & 1) + 2 * lane; i < nx; i += 64) {
            const int c = i + nx * (j + ny * k);
            const int fu = i + (nx + 1) * (j + ny * k), fv = i + nx * (j + (ny + 1) * k);
            T a[7], b[3];
            mom_cell<T, 3>(P, i, j, k, f.uf[fu], f.uf[fu + 1], f.vf[fv], f.vf[fv + nx], f.wf[c], f.wf[c + pl], f.p[c],
                           i > 0 ? f.p[c - 1] : (T)0, i < nx - 1 ? f.p[c + 1] : (T)0, j > 0 ? f.p[c - nx] : (T)0,
                           j < ny - 1 ? f.p[c + nx] : (T)0, k > 0 ? f.p[c - pl] : (T)0, k < nz - 1 ? f.p[c + pl] : (T)0,
                           a, b);
            add_dc<T, 3>(P, f, c, b);
            if (h.first) f.ac[c] = a[AC];
#pragma unroll
            for (int m = 0; m < 3; ++m) {
                if (!act[m]) continue;
                const T *o = phi[m];
                const T pE = i != nx - 1 ? o[c + 1] : (T)0, pW = i != 0 ? o[c - 1] : (T)0;
                const T pN = j != ny - 1 ? o[c + nx] : (T)0, pS = j != 0 ? o[c - nx] : (T)0;
                const T pT = k != nz - 1 ? o[c + pl] : (T)0, pB = k != 0 ? o[c - pl] : (T)0;
                T d;
                phi[m][c] = point_update<T, 3>(a, b[m], o[c], pE, pW, pN, pS, pT, pB, g.relax[m], d);
                sq[m] += (double)d * (double)d;
            }
        }
    }
    __shared__ double tot[3];
    if (grid_reduce<3>(sq, partials, ctl, tot) && threadIdx.x == 0) {
        for (int m = 0; m < 3; ++m) {
            if (!act[m]) continue;
            if (h.color == 0) {
                ctl->half_sq[m] = tot[m];
            } else {
                double s = ctl->half_sq[m] + tot[m];
                finish_sweeps(ctl, m, &s, 1, N, g.tol[m]);
            }
        }
    }
}

// 1/aC of every cell, for the p' links (IEEE division, as the reference's 1/aC).
template <typename T>
__global__ void k_recip_ac(const T *ac, T *rac, int N)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < N; c += gridDim.x * blockDim.x) rac[c] = (T)1 / ac[c];
}

template <typename T>
__global__ void __launch_bounds__(256) k_pc_half3d(Params<T> P, Fields<T> f, const T *rac, Ctl *ctl,
                                                   double *partials, int color, int zero_mode)
{
    const Geo<T> &g = P.g;
    if (ctl->stop[EQ_P]) return;  // uniform
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny, N = g.N;
    const int nrows = ny * nz, lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nwg = (int)((gridDim.x * blockDim.x) >> 5);
    double sq[1] = {0.0};
    // one warp per x-row, lanes over the row's cells of this colour
    for (int r = gw; r < nrows; r += nwg) {
        const int j = r % ny, k = r / ny;
        for (int i = ((color + j + k) & 1) + 2 * lane; i < nx; i += 64) {
            const int c = i + nx * (j + ny * k);
            const T rr = rac[c];
            T a[7];
            a[AE] = i < nx - 1 ? (T)(P.d.Kx * (double)(T)(rr + rac[c + 1])) : (T)0;
            a[AW] = i > 0 ? (T)(P.d.Kx * (double)(T)(rr + rac[c - 1])) : (T)0;
            a[AN] = j < ny - 1 ? (T)(P.d.Ky * (double)(T)(rr + rac[c + nx])) : (T)0;
            a[AS] = j > 0 ? (T)(P.d.Ky * (double)(T)(rr + rac[c - nx])) : (T)0;
            a[AT] = k < nz - 1 ? (T)(P.d.Kz * (double)(T)(rr + rac[c + pl])) : (T)0;
            a[AB] = k > 0 ? (T)(P.d.Kz * (double)(T)(rr + rac[c - pl])) : (T)0;
            a[AC] = -(a[AE] + a[AW] + a[AN] + a[AS]);
            a[AC] += -(a[AT] + a[AB]);
            const T *o = f.pc;
            // The solve starts from p' = 0 (src/Solver.cu:193) without clearing the
            // array: in the first red half every value is 0 (zero_mode 1); in the
            // first black half the neighbours are the red cells just written and
            // only the cell itself is still 0 (zero_mode 2).
            const bool zn = zero_mode == 1;
            const T pE = (!zn && i != nx - 1) ? o[c + 1] : (T)0, pW = (!zn && i != 0) ? o[c - 1] : (T)0;
            const T pN = (!zn && j != ny - 1) ? o[c + nx] : (T)0, pS = (!zn && j != 0) ? o[c - nx] : (T)0;
            const T pT = (!zn && k != nz - 1) ? o[c + pl] : (T)0, pB = (!zn && k != 0) ? o[c - pl] : (T)0;
            const T pc = zero_mode ? (T)0 : o[c];
            T d;
            f.pc[c] = point_update<T, 3>(a, f.sp[c], pc, pE, pW, pN, pS, pT, pB, g.relax[EQ_P], d);
            sq[0] += (double)d * (double)d;
        }
    }
    __shared__ double tot[1];
    if (grid_reduce<1>(sq, partials, ctl, tot) && threadIdx.x == 0) {
        if (color == 0) {
            ctl->half_sq[EQ_P] = tot[0];
        } else {
            double s = ctl->half_sq[EQ_P] + tot[0];
            finish_sweeps(ctl, EQ_P, &s, 1, N, g.tol[EQ_P]);
        }
    }
}

// ---- the whole 3D p' solve in one cooperative launch -----------------------
// Each CTA owns a rectangular block of x-rows (all i, j in [j0, j0+bj), k in
// [k0, k0+bk)) and keeps p' and b_p' of its cells in shared memory for every
// sweep of the solve.  The p' links do not change during the solve, so each
// CTA first builds them for its cells (kernels.cuh:518-537, the same FP64
// products as k_pc_half3d) into the coefficient planes aC, aE, aN, aT; a
// cell's west, south and bottom links are its neighbours' east, north and top
// links.  A half sweep then updates the CTA's cells of one colour; p'
// neighbours in rows owned by another CTA come from global memory, where every
// CTA publishes the cells of its boundary rows after each half sweep; a
// bounded grid barrier separates the half sweeps.  The per-sweep FP64 sums are
// reduced in a fixed order by every CTA, so each takes the same inner
// early-exit decision (src/Solver.cu:955-962).  Per cell the arithmetic is
// k_pc_half3d's, so the result is bit-identical to the per-half-sweep kernels.
struct PcBlocks {
    int bj, bk;    // rows per block along j and k
    int nbj, nbk;  // blocks along j and k
};

// Dynamic shared memory of k_pc_solve3d for row blocks of `rows` rows of nx
// cells: per row an int4 (global row offset, j, k, in-block neighbour flags),
// the list of the block's boundary rows (rounded up to 4 entries), then p'
// and b_p' of every cell.
template <typename T>
__host__ __device__ inline size_t pc3d_smem_bytes(int rows, int nx)
{
    return (size_t)rows * 16 + (size_t)((rows + 3) & ~3) * 4 + (size_t)rows * nx * 2 * sizeof(T);
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_pc_solve3d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials,
                                                      GridBarrier *bar, PcBlocks B, int n_sweeps)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny, N = g.N;
    const int G = gridDim.x, tid = threadIdx.x;
    const int j0 = (blockIdx.x % B.nbj) * B.bj, k0 = (blockIdx.x / B.nbj) * B.bk;
    const int nj = min(B.bj, ny - j0), nk = min(B.bk, nz - k0);
    const int rows_cap = B.bj * B.bk;
    const int cap = nx * rows_cap;
    const int nrow = nj * nk;
    const int warp = tid >> 5, lane = tid & 31;
    const int ln = nx, lt = nx * nj;  // local strides to the next row in j and in k
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // Row table (built once per solve, so the sweeps need no integer division
    // per row): x = global offset of the row, y = j, z = k, w = flags
    // (1: row j+1 in this block, 2: j-1, 4: k+1, 8: k-1); then the boundary
    // rows, which every half sweep publishes.
    int4 *s_row = reinterpret_cast<int4 *>(smem_raw);
    int *s_bnd = reinterpret_cast<int *>(s_row + rows_cap);
    T *s_pc = reinterpret_cast<T *>(s_bnd + ((rows_cap + 3) & ~3));
    T *s_sp = s_pc + cap;
    __shared__ int nbnd;
    T *cC = f.pcoef + (size_t)N * AC, *cE = f.pcoef + (size_t)N * AE;
    T *cN = f.pcoef + (size_t)N * AN, *cT = f.pcoef + (size_t)N * AT;
    __shared__ double red[NT / 32];
    __shared__ double tot2[2];

    for (int r = tid; r < nrow; r += NT) {
        const int jj = r % nj, kk = r / nj;
        const int j = j0 + jj, k = k0 + kk;
        const int fl = (jj + 1 < nj ? 1 : 0) | (jj > 0 ? 2 : 0) | (kk + 1 < nk ? 4 : 0) | (kk > 0 ? 8 : 0);
        s_row[r] = make_int4(nx * (j + ny * k), j, k, fl);
    }
    if (tid == 0) {
        int n = 0;
        for (int r = 0; r < nrow; ++r) {
            const int jj = r % nj, kk = r / nj;
            if (jj == 0 || jj == nj - 1 || kk == 0 || kk == nk - 1) s_bnd[n++] = r;
        }
        nbnd = n;
    }
    // links of the CTA's cells, b_p', p' = 0
    for (int r = warp; r < nrow; r += NT / 32) {
        const int j = j0 + r % nj, k = k0 + r / nj;
        const int lrow = nx * r, crow = nx * (j + ny * k);
        for (int i = lane; i < nx; i += 32) {
            const int c = crow + i;
            const T rr = f.rac[c];
            T a[7];
            a[AE] = i < nx - 1 ? (T)(P.d.Kx * (double)(T)(rr + f.rac[c + 1])) : (T)0;
            a[AW] = i > 0 ? (T)(P.d.Kx * (double)(T)(rr + f.rac[c - 1])) : (T)0;
            a[AN] = j < ny - 1 ? (T)(P.d.Ky * (double)(T)(rr + f.rac[c + nx])) : (T)0;
            a[AS] = j > 0 ? (T)(P.d.Ky * (double)(T)(rr + f.rac[c - nx])) : (T)0;
            a[AT] = k < nz - 1 ? (T)(P.d.Kz * (double)(T)(rr + f.rac[c + pl])) : (T)0;
            a[AB] = k > 0 ? (T)(P.d.Kz * (double)(T)(rr + f.rac[c - pl])) : (T)0;
            a[AC] = -(a[AE] + a[AW] + a[AN] + a[AS]);
            a[AC] += -(a[AT] + a[AB]);
            cC[c] = a[AC];
            cE[c] = a[AE];
            cN[c] = a[AN];
            cT[c] = a[AT];
            s_sp[lrow + i] = f.sp[c];
            s_pc[lrow + i] = (T)0;
        }
    }
    double mx = ctl->inner_max[EQ_P];
    int sw = ctl->sweeps[EQ_P];
    bool stop = ctl->stop[EQ_P] != 0;
    double last_sq = 0.0;
    unsigned int epoch = 0;
    bool failed = !grid_sync(bar, G, epoch);

    for (int s = 0; s < n_sweeps && !stop && !failed; ++s) {
        for (int color = 0; color < 2; ++color) {
            const int zero_mode = s == 0 ? (color == 0 ? 1 : 2) : 0;
            const bool zn = zero_mode == 1;
            double sq = 0.0;
            // one warp per row of the block (row r = jj + nj*kk), lanes along x
            for (int r = warp; r < nrow; r += NT / 32) {
                const int4 ri = s_row[r];
                const int j = ri.y, k = ri.z;
                const int lrow = nx * r, crow = ri.x;
                const bool inN = ri.w & 1, inS = ri.w & 2, inT = ri.w & 4, inB = ri.w & 8;
                for (int i = ((color + j + k) & 1) + 2 * lane; i < nx; i += 64) {
                    const int l = lrow + i, c = crow + i;
                    T a[7];
                    a[AC] = cC[c];
                    a[AE] = cE[c];
                    a[AW] = i > 0 ? cE[c - 1] : (T)0;
                    a[AN] = cN[c];
                    a[AS] = j > 0 ? cN[c - nx] : (T)0;
                    a[AT] = cT[c];
                    a[AB] = k > 0 ? cT[c - pl] : (T)0;
                    const T pE = (!zn && i != nx - 1) ? s_pc[l + 1] : (T)0;
                    const T pW = (!zn && i != 0) ? s_pc[l - 1] : (T)0;
                    const T pN = (!zn && j != ny - 1) ? (inN ? s_pc[l + ln] : __ldcg(&f.pc[c + nx])) : (T)0;
                    const T pS = (!zn && j != 0) ? (inS ? s_pc[l - ln] : __ldcg(&f.pc[c - nx])) : (T)0;
                    const T pT = (!zn && k != nz - 1) ? (inT ? s_pc[l + lt] : __ldcg(&f.pc[c + pl])) : (T)0;
                    const T pB = (!zn && k != 0) ? (inB ? s_pc[l - lt] : __ldcg(&f.pc[c - pl])) : (T)0;
                    const T pc = zero_mode ? (T)0 : s_pc[l];
                    T d;
                    s_pc[l] = point_update<T, 3>(a, s_sp[l], pc, pE, pW, pN, pS, pT, pB, g.relax[EQ_P], d);
                    sq += (double)d * (double)d;
                }
            }
            __syncthreads();
            // publish this colour's cells of the boundary rows
            for (int b = warp; b < nbnd; b += NT / 32) {
                const int r = s_bnd[b];
                const int4 ri = s_row[r];
                const int lrow = nx * r, crow = ri.x;
                for (int i = ((color + ri.y + ri.z) & 1) + 2 * lane; i < nx; i += 64) f.pc[crow + i] = s_pc[lrow + i];
            }
            // this CTA's sum of the half sweep, in warp order
            sq = warp_sum(sq);
            if (lane == 0) red[warp] = sq;
            __syncthreads();
            if (tid == 0) {
                double x = 0.0;
                for (int w = 0; w < NT / 32; ++w) x += red[w];
                partials[(size_t)(2 * (s & 1) + color) * G + blockIdx.x] = x;
            }
            if (!grid_sync(bar, G, epoch)) { failed = true; break; }
        }
        if (failed) break;
        // grid sums of both halves, fixed order, identical in every CTA
        if (tid < 64) {
            const int color = tid >> 5;
            double x = 0.0;
            for (int b = lane; b < G; b += 32) x += __ldcg(&partials[(size_t)(2 * (s & 1) + color) * G + b]);
            x = warp_sum(x);
            if (lane == 0) tot2[color] = x;
        }
        __syncthreads();
        const double ssq = tot2[0] + tot2[1];
        const double rms = sqrt(ssq / (double)N);
        if (rms > mx) mx = rms;
        if (rms / (mx + 1e-20) < g.tol[EQ_P]) stop = true;
        ++sw;
        last_sq = ssq;
        __syncthreads();  // tot2 is rewritten only after the next sweep's barriers
    }
    for (int r = warp; r < nrow; r += NT / 32) {
        const int j = j0 + r % nj, k = k0 + r / nj;
        const int lrow = nx * r, crow = nx * (j + ny * k);
        for (int i = lane; i < nx; i += 32) f.pc[crow + i] = s_pc[lrow + i];
    }
    if (blockIdx.x == 0 && tid == 0 && !failed) {
        const int done = sw - ctl->sweeps[EQ_P];
        ctl->cell_updates += (long long)done * N;
        ctl->inner_max[EQ_P] = mx;
        ctl->sweeps[EQ_P] = sw;
        if (done > 0) ctl->last_sweep_sq[EQ_P] = last_sq;
        if (stop) ctl->stop[EQ_P] = 1;
    }
    if (tid == 0 && (failed || bar->err)) atomicExch(&ctl->status, 3);
}

}  // namespace ifc
