// ifc_coop3d.cuh -- a 3D linear solve (the p' equation, or a system with
// stored coefficients such as the temperature) as one cooperative launch,
// with the unknown resident in shared memory and the links and source of
// every cell packed once per solve in sweep order.
//
// Work split: each CTA owns a rectangular block of x-rows (all i, j in
// [j0, j0+bj), k in [k0, k0+bk)) for the whole solve (PcBlocks, chosen on the
// host so that one CTA per SM holds its block).  Set-up: every cell of the
// block gets its six links -- for p' from 1/aC (kernels.cuh:518-537, FP64
// products as in k_pc_half3d), otherwise from the stored planes -- its
// diagonal and its source, written to a packed array in the order the sweeps
// consume them: per (row, colour) the cells of that colour, one 16-byte
// vector of four values per plane and cell slot.  A half sweep then reads
// each updated cell's coefficients with two coalesced 128-bit loads and its
// neighbours from shared memory (or, in the rows of a neighbouring block,
// from global memory, to which a CTA writes the cells of its edge rows as it
// updates them); a bounded grid barrier separates the half sweeps.  Rows
// inside the block take a path with every neighbour in shared memory.  The
// per-sweep FP64 sums are reduced by every CTA in one fixed order, so every
// CTA takes the same inner early-exit decision (src/Solver.cu:955-962).  The
// arithmetic of each update is that of point_update on the same
// coefficients, so the results equal the per-half-sweep kernels and the CPU
// oracle bit for bit.  Only the unknown takes shared memory (the source
// travels with the links), so FP64 grids of the size FP32 ones run at fit
// as well; each row keeps its even-i cells, then its odd-i cells, so the
// cells a warp updates and all their neighbours are consecutive words (no
// bank conflicts; FP64 solves 6 % faster, FP32 unchanged).
#pragma once

#include "ifc_fused3d.cuh"

namespace ifc {

// Packed slots: per CTA rows_cap rows x 2 colours x hx cells, hx = (nx+1)/2;
// the cell (i, row r, colour c) sits in slot (2r + c) * hx + (i >> 1) of its
// CTA's range.  Two planes of 4 values per slot follow each other, each
// spanning all CTAs' slots.
__host__ __device__ inline long long coop3d_slots(const PcBlocks &B, int nx)
{
    return (long long)B.nbj * B.nbk * B.bj * B.bk * 2 * ((nx + 1) / 2);
}

// Shared memory: the row table (int4 per row), then the unknown of every
// cell of the block.
template <typename T>
__host__ __device__ inline size_t coop3d_smem_bytes(int rows, int nx)
{
    return (size_t)rows * 16 + (size_t)rows * 2 * ((nx + 1) / 2) * sizeof(T);
}

// The linear system a cooperative solve works on: the p' equation (coef null:
// links from 1/aC, start from p' = 0 without clearing the array, as the
// per-half-sweep kernel does) or a system with stored coefficient planes
// coef[cell + N*slot] (slots aC aE aW aN aS aT aB), e.g. the temperature.
// Unknown x, source src, equation slot eq of the control block (relaxation,
// tolerance, sweep bookkeeping).
template <typename T>
struct CSys {
    const T *coef;
    const T *src;
    T *x;
    int eq;
};

template <typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_csolve3d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials,
                                                    GridBarrier *bar, PcBlocks B, int n_sweeps, T *pk, CSys<T> sys,
                                                    int stall_test)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny, N = g.N;
    const int G = gridDim.x, tid = threadIdx.x;
    const int j0 = (blockIdx.x % B.nbj) * B.bj, k0 = (blockIdx.x / B.nbj) * B.bk;
    const int nj = min(B.bj, ny - j0), nk = min(B.bk, nz - k0);
    const int rows_cap = B.bj * B.bk;
    const int nrow = nj * nk;
    const int warp = tid >> 5, lane = tid & 31;
    // shared layout: each local row holds its even-i cells, then its odd-i
    // cells (hx each), so a warp's cells of one colour and their neighbours
    // are consecutive words
    const int hx2 = 2 * ((nx + 1) / 2);
    const int ln = hx2, lt = hx2 * nj;  // local strides to the next row in j and in k
    const int hx = (nx + 1) / 2;
    const long long S = coop3d_slots(B, nx);
    const long long cbase = (long long)blockIdx.x * rows_cap * 2 * hx;
    T *pA = pk, *pB = pk + 4 * S;  // {aC, aE, aW, aN}, {aS, aT, aB, b}
    extern __shared__ __align__(16) unsigned char smem_raw[];
    int4 *s_row = reinterpret_cast<int4 *>(smem_raw);
    T *s_x = reinterpret_cast<T *>(s_row + rows_cap);
    __shared__ double red[NT / 32];
    __shared__ double tot2[2];
    const int eq = sys.eq;
    const bool zero_start = sys.coef == nullptr;
    T *x = sys.x;

    // row table: x = global offset of the row, y = j, z = k, w = flags (1: row
    // j+1 in this block, 2: j-1, 4: k+1, 8: k-1)
    for (int r = tid; r < nrow; r += NT) {
        const int jj = r % nj, kk = r / nj;
        const int j = j0 + jj, k = k0 + kk;
        const int fl = (jj + 1 < nj ? 1 : 0) | (jj > 0 ? 2 : 0) | (kk + 1 < nk ? 4 : 0) | (kk > 0 ? 8 : 0);
        s_row[r] = make_int4(nx * (j + ny * k), j, k, fl);
    }
    __syncthreads();
    // packed links and sources of the CTA's cells, the unknown into shared memory
    for (int r = warp; r < nrow; r += NT / 32) {
        const int4 ri = s_row[r];
        const int j = ri.y, k = ri.z, crow = ri.x, lrow = hx2 * r;
        for (int i = lane; i < nx; i += 32) {
            const int c = crow + i;
            T a[7];
            if (zero_start) {
                const T rr = f.rac[c];
                a[AE] = i < nx - 1 ? (T)(P.d.Kx * (double)(T)(rr + f.rac[c + 1])) : (T)0;
                a[AW] = i > 0 ? (T)(P.d.Kx * (double)(T)(rr + f.rac[c - 1])) : (T)0;
                a[AN] = j < ny - 1 ? (T)(P.d.Ky * (double)(T)(rr + f.rac[c + nx])) : (T)0;
                a[AS] = j > 0 ? (T)(P.d.Ky * (double)(T)(rr + f.rac[c - nx])) : (T)0;
                a[AT] = k < nz - 1 ? (T)(P.d.Kz * (double)(T)(rr + f.rac[c + pl])) : (T)0;
                a[AB] = k > 0 ? (T)(P.d.Kz * (double)(T)(rr + f.rac[c - pl])) : (T)0;
                a[AC] = -(a[AE] + a[AW] + a[AN] + a[AS]);
                a[AC] += -(a[AT] + a[AB]);
            } else {
#pragma unroll
                for (int q = 0; q < 7; ++q) a[q] = sys.coef[c + (size_t)N * q];
            }
            const long long slot = cbase + (long long)(2 * r + ((i + j + k) & 1)) * hx + (i >> 1);
            st4(pA + 4 * slot, a[AC], a[AE], a[AW], a[AN]);
            st4(pB + 4 * slot, a[AS], a[AT], a[AB], sys.src[c]);
            s_x[lrow + (i & 1) * (hx2 >> 1) + (i >> 1)] = zero_start ? (T)0 : x[c];
        }
    }
    double mx = ctl->inner_max[eq];
    int sw = ctl->sweeps[eq];
    bool stop = ctl->stop[eq] != 0;
    double last_sq = 0.0;
    unsigned int epoch = 0;
    __syncthreads();  // the packed values are read back by the same CTA only

    // Failure-detection test (IFC_TEST_STALL_BARRIER=1): CTA 0 leaves before
    // its first grid barrier, so every other CTA's bounded wait runs out and
    // the launch ends with the timeout status.
    bool failed = stall_test && blockIdx.x == 0;
    for (int s = 0; s < n_sweeps && !stop && !failed; ++s) {
        for (int color = 0; color < 2; ++color) {
            const int zero_mode = (zero_start && s == 0) ? (color == 0 ? 1 : 2) : 0;
            const bool zn = zero_mode == 1;
            double sq = 0.0;
            for (int r = warp; r < nrow; r += NT / 32) {
                const int4 ri = s_row[r];
                const int j = ri.y, k = ri.z;
                const int lrow = hx2 * r, crow = ri.x;
                const bool inN = ri.w & 1, inS = ri.w & 2, inT = ri.w & 4, inB = ri.w & 8;
                const int off = (color + j + k) & 1;
                const long long sbase = cbase + (long long)(2 * r + color) * hx;
                // a row on the block's edge: its cells also go to global
                // memory at once, for the neighbouring blocks' next half sweep
                const bool edge_row = (ri.w & 15) != 15;
                if (!edge_row && !zero_mode) {
                    // all four off-row neighbours are rows of this block
                    for (int i = off + 2 * lane; i < nx; i += 64) {
                        const int l = lrow + off * (hx2 >> 1) + (i >> 1);
                        const int le = lrow + (1 - off) * (hx2 >> 1) + (i >> 1);  // i+1 is le + off, i-1 is le + off - 1
                        const long long slot = sbase + (i >> 1);
                        T q0[4], q1[4];
                        ld4(pA + 4 * slot, q0);
                        ld4(pB + 4 * slot, q1);
                        const T a[7] = {q0[0], q0[1], q0[2], q0[3], q1[0], q1[1], q1[2]};
                        const T pE = i != nx - 1 ? s_x[le + off] : (T)0;
                        const T pW = i != 0 ? s_x[le + off - 1] : (T)0;
                        T d;
                        s_x[l] = point_update<T, 3>(a, q1[3], s_x[l], pE, pW, s_x[l + ln], s_x[l - ln], s_x[l + lt],
                                                    s_x[l - lt], g.relax[eq], d);
                        sq += (double)d * (double)d;
                    }
                    continue;
                }
                for (int i = off + 2 * lane; i < nx; i += 64) {
                    const int l = lrow + off * (hx2 >> 1) + (i >> 1), c = crow + i;
                    const int le = lrow + (1 - off) * (hx2 >> 1) + (i >> 1);
                    const long long slot = sbase + (i >> 1);
                    T q0[4], q1[4];
                    ld4(pA + 4 * slot, q0);
                    ld4(pB + 4 * slot, q1);
                    const T a[7] = {q0[0], q0[1], q0[2], q0[3], q1[0], q1[1], q1[2]};
                    const T pE = (!zn && i != nx - 1) ? s_x[le + off] : (T)0;
                    const T pW = (!zn && i != 0) ? s_x[le + off - 1] : (T)0;
                    const T pN = (!zn && j != ny - 1) ? (inN ? s_x[l + ln] : __ldcg(&x[c + nx])) : (T)0;
                    const T pS = (!zn && j != 0) ? (inS ? s_x[l - ln] : __ldcg(&x[c - nx])) : (T)0;
                    const T pT = (!zn && k != nz - 1) ? (inT ? s_x[l + lt] : __ldcg(&x[c + pl])) : (T)0;
                    const T pB_ = (!zn && k != 0) ? (inB ? s_x[l - lt] : __ldcg(&x[c - pl])) : (T)0;
                    const T pc = zero_mode ? (T)0 : s_x[l];
                    T d;
                    const T v = point_update<T, 3>(a, q1[3], pc, pE, pW, pN, pS, pT, pB_, g.relax[eq], d);
                    s_x[l] = v;
                    if (edge_row) x[c] = v;
                    sq += (double)d * (double)d;
                }
            }
            sq = warp_sum(sq);
            if (lane == 0) red[warp] = sq;
            __syncthreads();
            if (tid == 0) {
                double t = 0.0;
                for (int w = 0; w < NT / 32; ++w) t += red[w];
                partials[(size_t)(2 * (s & 1) + color) * G + blockIdx.x] = t;
            }
            if (!grid_sync(bar, G, epoch)) {
                failed = true;
                break;
            }
        }
        if (failed) break;
        // grid sums of both halves, fixed order, identical in every CTA
        if (tid < 64) {
            const int color = tid >> 5;
            double t = 0.0;
            for (int b = lane; b < G; b += 32) t += __ldcg(&partials[(size_t)(2 * (s & 1) + color) * G + b]);
            t = warp_sum(t);
            if (lane == 0) tot2[color] = t;
        }
        __syncthreads();
        const double ssq = tot2[0] + tot2[1];
        const double rms = sqrt(ssq / (double)N);
        if (rms > mx) mx = rms;
        if (rms / (mx + 1e-20) < g.tol[eq]) stop = true;
        ++sw;
        last_sq = ssq;
        __syncthreads();  // tot2 is rewritten only after the next sweep's barriers
    }
    for (int r = warp; r < nrow; r += NT / 32) {
        const int crow = s_row[r].x, lrow = hx2 * r;
        for (int i = lane; i < nx; i += 32) x[crow + i] = s_x[lrow + (i & 1) * (hx2 >> 1) + (i >> 1)];
    }
    if (blockIdx.x == 0 && tid == 0 && !failed) {
        const int done = sw - ctl->sweeps[eq];
        ctl->cell_updates += (long long)done * N;
        ctl->inner_max[eq] = mx;
        ctl->sweeps[eq] = sw;
        if (done > 0) ctl->last_sweep_sq[eq] = last_sq;
        if (stop) ctl->stop[eq] = 1;
    }
    if (tid == 0 && (failed || bar->err)) atomicExch(&ctl->status, 3);
}

}  // namespace ifc
