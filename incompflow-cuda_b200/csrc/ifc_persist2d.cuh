// ifc_persist2d.cuh -- the whole 2D SIMPLE loop in one cooperative launch.
//
// Every CTA owns one TX x TY tile for the whole solve (MT = false) or, when
// the grid has more tiles than co-resident CTAs, a fixed set of tiles that it
// visits in turn inside every phase (MT = true), and walks through the phases
// of each outer iteration (src/Solver.cu:160-289):
//   momentum passes (assembly + KS red-black sweeps of u and v, temporally
//   blocked in shared memory as in ifc_fused2d.cuh), Rhie-Chow faces + p'
//   source, p' passes, [p' mean removal], corrections + convergence test,
// separated by grid barriers instead of kernel boundaries.  After each barrier
// every CTA reads all CTAs' FP64 partial sums and reduces them in one fixed
// order, so every CTA takes the same early-exit and convergence decisions
// without another barrier.  Barrier waits are bounded: a CTA that waits longer
// than kBarrierTimeoutNs sets the error flag, every CTA leaves the loop, and
// the host reports IFC_TIMEOUT.  The launch is cooperative, so all CTAs are
// co-resident or the launch fails (the engine then uses the multi-kernel graph).
#pragma once

#include "ifc_fused2d.cuh"

namespace ifc {

struct GridBarrier {
    unsigned int count;  // arrivals since the launch; barrier k completes at (k+1)*G
    unsigned int gen;    // unused, kept for layout
    int err;
};

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid barrier on a monotonically increasing arrival counter: each CTA adds
// one arrival and waits until all G arrivals of this barrier are in, so the
// critical path is one atomic plus the pollers' next read.  `epoch` counts
// the barriers this CTA has passed (same in every CTA).  Returns false in
// every thread of the CTA when the wait timed out or another CTA reported an
// error.
__device__ __forceinline__ bool grid_sync(GridBarrier *b, unsigned int nblocks, unsigned int &epoch)
{
    __shared__ int ok;
    __syncthreads();
    ++epoch;
    if (threadIdx.x == 0) {
        int good = 1;
        const unsigned int target = epoch * nblocks;
        // The arrival releases this CTA's writes (ordered before it by the
        // __syncthreads above) and, for the last CTA to arrive, acquires the
        // others'; the pollers acquire them through ld.acquire.
        unsigned int old;
        asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(&b->count) : "memory");
        if (old + 1 < target) {
            // One L2 round trip per poll; the error flag and the clock are
            // read every 64 polls only, so they stay off the critical path.
            // A CTA that passes this barrier while another gave up meets the
            // flag at the next barrier, which the other never reaches.
            const unsigned long long t0 = global_ns();
            unsigned int spins = 0;
            while (ld_acquire(&b->count) < target) {
                if ((++spins & 63u) == 0) {
                    if (*(volatile int *)&b->err) { good = 0; break; }
                    if (global_ns() - t0 > kBarrierTimeoutNs) {
                        atomicExch(&b->err, 1);
                        good = 0;
                        break;
                    }
                }
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Sum column r of partials (one value per CTA) for r < NRV in a fixed order;
// identical in every CTA.  Warp w sums columns w, w + NT/32, ... (each
// lane-strided, then one shuffle tree), so the columns are reduced in
// parallel with one round trip to L2.  out: shared, NRV entries.
template <int NRV, int NT>
__device__ __forceinline__ void reduce_partials(const double *partials, int G, double *out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < NRV; r += NT / 32) {
        const double *col = partials + (size_t)r * G;
        double x = 0.0;
#pragma unroll 4
        for (int b = lane; b < G; b += 32) x += __ldcg(&col[b]);
        x = warp_sum(x);
        if (lane == 0) out[r] = x;
    }
    __syncthreads();
}

// Block-wide sum of per-thread values written as this CTA's partials.
template <int NRV, int NT>
__device__ __forceinline__ void write_partials(double (&v)[NRV], double *partials, int G)
{
    __shared__ double red[NT / 32][NRV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < NRV; ++r) {
        double x = warp_sum(v[r]);
        if (lane == 0) red[warp][r] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < NRV; ++r) {
            double x = lane < NT / 32 ? red[lane][r] : 0.0;
            x = warp_sum(x);
            if (lane == 0) partials[(size_t)r * G + blockIdx.x] = x;
        }
    }
}

// This CTA's partials from per-warp sums: slot r = sum over warps, in order.
template <int NRV, int STRIDE, int NT>
__device__ __forceinline__ void block_partials(const double *wred, double *partials, int G)
{
    __syncthreads();
    if (threadIdx.x < NRV) {
        double x = 0.0;
        for (int w = 0; w < NT / 32; ++w) x += wred[w * STRIDE + threadIdx.x];
        partials[(size_t)threadIdx.x * G + blockIdx.x] = x;
    }
}

// Block-uniform loop state, kept in shared memory.
struct LoopState {
    int it, it_begin, it_stop, act, log_level, log_n, status, done;
    int stop[4], sweeps[4];
    long long cell_updates;
    double inner_max[4];
    double maxn[8];
};

struct PersistArgs {
    int n_iter[4];
    int pin;
    int stall_test;  // failure-detection test: CTA 0 leaves before its first barrier
};

// Inner early-exit bookkeeping for one equation after a pass (the rule of
// src/Solver.cu:955-962 evaluated after each sweep of the pass).
__device__ __forceinline__ void pass_done(LoopState &L, int e, const double *sq, int ns, int N, double tol)
{
    double mx = L.inner_max[e];
    bool stop_now = false;
    for (int s = 0; s < ns; ++s) {
        if (stop_now) break;
        const double rms = sqrt(sq[s] / (double)N);
        if (rms > mx) mx = rms;
        if (rms / (mx + 1e-20) < tol) stop_now = true;
    }
    L.inner_max[e] = mx;
    L.sweeps[e] += ns;
    L.cell_updates += (long long)ns * N;
    if (stop_now) L.stop[e] = 1;
}

// Bookkeeping of the last pass of a phase: its sums could only set an
// early-exit flag for passes that do not follow (the flags are reset with
// every outer iteration), so they are not reduced.
__device__ __forceinline__ void pass_count(LoopState &L, int e, int ns, int N)
{
    L.sweeps[e] += ns;
    L.cell_updates += (long long)ns * N;
}

// Origin of tile t (tiles numbered row-major, tiles_x per row) and of its
// staged region.
struct Tile {
    int x0, y0, gx0, gy0;
};

template <int TX, int TY, int H>
__device__ __forceinline__ Tile tile_at(int t, int tiles_x)
{
    Tile tl;
    tl.x0 = (t % tiles_x) * TX;
    tl.y0 = (t / tiles_x) * TY;
    tl.gx0 = tl.x0 - H;
    tl.gy0 = tl.y0 - H;
    return tl;
}

// This thread's cells of each colour in the staged region of tile tl (cq),
// their distance from the tile (dq); returns whether the warp owns any tile
// cell (warps that own none contribute only zeros to the per-sweep sums: they
// skip the shuffle reduction -- the shuffle unit is shared by the whole SM --
// and report 0.0, the value the reduction gives).
template <int W, int H, int TX, int TY, int HH, int NHALF, int NT, int CPT>
__device__ __forceinline__ bool map_tile(int tid, const Tile &tl, int nx, int ny, int (&cq)[2][CPT], int (&dq)[2][CPT])
{
    own_cells<W, HH, NHALF, NT, CPT>(tid, tl.gx0, tl.gy0, nx, ny, cq);
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) dq[c][k] = tile_distance<W, H, TX, TY>(cq[c][k]);
    bool mine = false;
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) mine |= dq[c][k] == 0;
    return __any_sync(0xffffffffu, mine);
}

template <typename T, int TX, int TY, int KS, int NT, bool MT>
__global__ void __launch_bounds__(NT) k_simple2d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials,
                                                 GridBarrier *bar, PersistArgs pa)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const int G = gridDim.x;
    const int tid = threadIdx.x;
    const int tiles_x = (nx + TX - 1) / TX;
    const int ntiles = tiles_x * ((ny + TY - 1) / TY);
    // MT: this CTA's tiles are blockIdx.x, blockIdx.x + G, ...; otherwise its
    // one tile (the tile loops below then have a compile-time trip count of 1).

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s0 = reinterpret_cast<T *>(smem_raw);
    T *s1 = s0 + NR;
    T *s2 = s1 + NR;
    __shared__ LoopState L;
    __shared__ double tot[16];
    __shared__ double wred[NT / 32][2 * KS];  // per-warp sums of each sweep

    if (tid == 0) {
        L.it = ctl->it;
        L.it_begin = ctl->it_begin;
        L.it_stop = ctl->it_stop;
        L.act = ctl->act;
        L.log_level = ctl->log_level;
        L.log_n = ctl->log_n;
        L.status = 0;
        L.done = L.it >= L.it_stop;
        L.cell_updates = 0;
        for (int q = 0; q < 8; ++q) L.maxn[q] = ctl->maxn[q];
    }
    int cq[2][CPT], dq[2][CPT];
    const Tile tile0 = tile_at<TX, TY, H>(blockIdx.x, tiles_x);
    bool wsum = map_tile<W, H, TX, TY, R::HH, R::NHALF, NT, CPT>(tid, tile0, nx, ny, cq, dq);
    __syncthreads();

    const int npass_m = (max(pa.n_iter[0], pa.n_iter[1]) + KS - 1) / KS;
    const int npass_p = (pa.n_iter[3] + KS - 1) / KS;
    bool failed = false;
    unsigned int epoch = 0;
    // A pass stages halos from one buffer and writes its tile to the other, so
    // no tile reads a neighbour tile's values of the same pass; `mcur`/`pcur`
    // (the same in every CTA) say which buffer holds the current u, v / p'.
    T *bu[2] = {f.u, f.tmp}, *bv[2] = {f.v, f.tmp + N}, *bp[2] = {f.pc, f.tmp + 2 * (size_t)N};

    while (!L.done) {
        int mcur = 0, pcur = 0;
        if (tid == 0)
            for (int q = 0; q < 4; ++q) {
                L.stop[q] = 0;
                L.sweeps[q] = 0;
                L.inner_max[q] = -1e20;
            }
        __syncthreads();

        // Failure-detection test (IFC_TEST_STALL_BARRIER=1 in the environment):
        // CTA 0 leaves without arriving, so every other CTA's bounded wait at the
        // next barrier runs out and the launch ends with the timeout status.
        if (pa.stall_test && blockIdx.x == 0) { failed = true; break; }

        // ---- deferred-correction sources (higher-order convection), from the
        // fields at the start of the outer iteration; the momentum passes read
        // them for their halos too, so a barrier follows ----
        if (g.conv != CONV_UPWIND) {
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = tl.x0 + q % TX, j = tl.y0 + q / TX;
                    if (i >= nx || j >= ny) continue;
                    const int c = i + nx * j;
                    f.sdc[c] = dc_cell<T, 2>(P, f, f.u, i, j, 0);
                    f.sdc[N + c] = dc_cell<T, 2>(P, f, f.v, i, j, 0);
                }
            }
            if (!grid_sync(bar, G, epoch)) { failed = true; break; }
        }

        // ---------------- momentum passes ----------------
        for (int pass = 0; pass < (npass_m > 0 ? npass_m : 1); ++pass) {
            int ns[2] = {clamp_sweeps(pa.n_iter[0], pass, KS), clamp_sweeps(pa.n_iter[1], pass, KS)};
            const bool au = ns[0] > 0 && !L.stop[EQ_U];
            const bool av = ns[1] > 0 && !L.stop[EQ_V];
            if (!au && !av && pass > 0) continue;
            // The sums of a phase's last pass are never reduced.
            const bool last = pass >= npass_m - 1;
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const bool first = t == (int)blockIdx.x;
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                if (MT) wsum = map_tile<W, H, TX, TY, R::HH, R::NHALF, NT, CPT>(tid, tl, nx, ny, cq, dq);
                const int gx0 = tl.gx0, gy0 = tl.gy0;
                for (int q = tid; q < NR; q += NT) {
                    const int a = q % W, b = q / W;
                    const int gi = gx0 + a, gj = gy0 + b;
                    const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
                    const int id = gi + nx * gj;
                    s0[q] = in ? bu[mcur][id] : (T)0;
                    s1[q] = in ? bv[mcur][id] : (T)0;
                    // p does not change in the momentum passes: with one tile per
                    // CTA its region stays in s2 after the first pass
                    if (MT || pass == 0) s2[q] = in ? f.p[id] : (T)0;
                }
                __syncthreads();
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
                        mom_cell<T, 2>(P, gi, gj, 0, f.uf[fu], f.uf[fu + 1], f.vf[fv], f.vf[fv + nx], (T)0, (T)0, s2[q],
                                       s2[q - 1], s2[q + 1], s2[q - W], s2[q + W], (T)0, (T)0, a7, b3);
                        add_dc<T, 2>(P, f, fv, b3);
                        cE[c][k] = a7[AE];
                        cW[c][k] = a7[AW];
                        cN[c][k] = a7[AN];
                        cS[c][k] = a7[AS];
                        cC[c][k] = a7[AC];
                        cbu[c][k] = b3[0];
                        cbv[c][k] = b3[1];
                        own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
                    }
                if (pass == 0) {
#pragma unroll
                    for (int c = 0; c < 2; ++c)
#pragma unroll
                        for (int k = 0; k < CPT; ++k)
                            if (own[c][k]) f.ac[gx0 + cq[c][k] % W + nx * (gy0 + cq[c][k] / W)] = cC[c][k];
                }
                const T ru = g.relax[EQ_U], rv = g.relax[EQ_V];
#pragma unroll 1
                for (int s = 0; s < KS; ++s) {
                    const bool du = au && s < ns[0];
                    const bool dv = av && s < ns[1];
                    if (!du && !dv) break;
                    double su = 0.0, sv = 0.0;
#pragma unroll
                    for (int color = 0; color < 2; ++color) {
                        const int hs = 2 * s + color;
#pragma unroll
                        for (int k = 0; k < CPT; ++k) {
                            const int q = cq[color][k];
                            if (q < 0) continue;
                            T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k], (T)0, (T)0};
                            T d;
                            if (du && dq[color][k] <= 2 * ns[0] - 1 - hs) {
                                s0[q] = point_update<T, 2>(a7, cbu[color][k], s0[q], s0[q + 1], s0[q - 1], s0[q + W],
                                                           s0[q - W], (T)0, (T)0, ru, d);
                                if (!last && own[color][k]) su += (double)d * (double)d;
                            }
                            if (dv && dq[color][k] <= 2 * ns[1] - 1 - hs) {
                                s1[q] = point_update<T, 2>(a7, cbv[color][k], s1[q], s1[q + 1], s1[q - 1], s1[q + W],
                                                           s1[q - W], (T)0, (T)0, rv, d);
                                if (!last && own[color][k]) sv += (double)d * (double)d;
                            }
                        }
                        __syncthreads();
                    }
                    if (!last) {
                        if (wsum) {
                            su = warp_sum(su);
                            sv = warp_sum(sv);
                        }
                        if ((tid & 31) == 0) {
                            if (MT && !first) {
                                wred[tid >> 5][s] += su;
                                wred[tid >> 5][KS + s] += sv;
                            } else {
                                wred[tid >> 5][s] = su;
                                wred[tid >> 5][KS + s] = sv;
                            }
                        }
                    }
                }
                for (int q = tid; q < TX * TY; q += NT) {
                    const int a = H + q % TX, b = H + q / TX;
                    const int gi = gx0 + a, gj = gy0 + b;
                    if (gi >= nx || gj >= ny) continue;
                    const int id = gi + nx * gj;
                    bu[mcur ^ 1][id] = s0[b * W + a];
                    bv[mcur ^ 1][id] = s1[b * W + a];
                }
                if (MT) __syncthreads();  // the next tile's staging overwrites the region
            }
            mcur ^= 1;
            if (!last) block_partials<2 * KS, 2 * KS, NT>(&wred[0][0], partials, G);
            if (!grid_sync(bar, G, epoch)) { failed = true; break; }
            if (!last) reduce_partials<2 * KS, NT>(partials, G, tot);
            if (tid == 0) {
                if (au) {
                    if (last) pass_count(L, EQ_U, ns[0], N);
                    else pass_done(L, EQ_U, tot, ns[0], N, g.tol[EQ_U]);
                }
                if (av) {
                    if (last) pass_count(L, EQ_V, ns[1], N);
                    else pass_done(L, EQ_V, tot + KS, ns[1], N, g.tol[EQ_V]);
                }
            }
            __syncthreads();
        }
        if (failed) break;

        // ------------- Rhie-Chow faces, face BCs, p' source -------------
        Fields<T> fc = f;  // the current u, v
        fc.u = bu[mcur];
        fc.v = bv[mcur];
        {
            double m[1] = {0.0};
            // The tile's (TX+1) x TY x-faces and TX x (TY+1) y-faces, one per
            // thread, into shared memory (the staged region is free here);
            // then every cell's mass imbalance from its four faces.  A face on
            // the tile's east or north edge is also computed by the next
            // tile, which owns and stores it (same operations, same value).
            constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
            static_assert(NFX + NFY <= 3 * NR, "faces of a tile must fit the staged region");
            T *s_f = s0;
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                for (int q = tid; q < NFX + NFY; q += NT) {
                    if (q < NFX) {
                        const int a = q % (TX + 1), b = q / (TX + 1);
                        const int i = tl.x0 + a, j = tl.y0 + b;  // face i of row j
                        if (i > nx || j >= ny) continue;
                        const int c = i + nx * j;
                        const T val = i == 0 ? face_bc(g, WEST, 0, fc.u[c], j)
                                              : (i == nx ? face_bc(g, EAST, 0, fc.u[c - 1], j) : rc_x(P, fc, i, j));
                        s_f[q] = val;
                        if (a < TX || i == nx) f.uf[i + (nx + 1) * j] = val;
                    } else {
                        const int q2 = q - NFX;
                        const int a = q2 % TX, b = q2 / TX;
                        const int i = tl.x0 + a, j = tl.y0 + b;  // face j of column i
                        if (i >= nx || j > ny) continue;
                        const int c = i + nx * j;
                        const T val = j == 0 ? face_bc(g, SOUTH, 1, fc.v[c], 0)
                                              : (j == ny ? face_bc(g, NORTH, 1, fc.v[c - nx], 0) : rc_y(P, fc, i, j));
                        s_f[q] = val;
                        if (b < TY || j == ny) f.vf[c] = val;
                    }
                }
                __syncthreads();
                for (int q = tid; q < TX * TY; q += NT) {
                    const int a = q % TX, b = q / TX;
                    const int i = tl.x0 + a, j = tl.y0 + b;
                    if (i >= nx || j >= ny) continue;
                    const T uw = s_f[a + (TX + 1) * b], ue = s_f[a + 1 + (TX + 1) * b];
                    const T vs = s_f[NFX + a + TX * b], vn = s_f[NFX + a + TX * (b + 1)];
                    const T bm = mass_imbalance<T, 2>(g, uw, ue, vs, vn, (T)0, (T)0);
                    f.sp[i + nx * j] = bm;
                    m[0] += (double)bm * (double)bm;
                }
                if (MT) __syncthreads();  // the next tile's faces overwrite s_f
            }
            write_partials<1, NT>(m, partials + 15 * (size_t)G, G);
            if (!grid_sync(bar, G, epoch)) break;
        }

        // ---------------- p' passes ----------------
        for (int pass = 0; pass < npass_p; ++pass) {
            const int ns = clamp_sweeps(pa.n_iter[3], pass, KS);
            if (ns <= 0 || L.stop[EQ_P]) continue;
            const bool last = pass == npass_p - 1;
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const bool first = t == (int)blockIdx.x;
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                if (MT) wsum = map_tile<W, H, TX, TY, R::HH, R::NHALF, NT, CPT>(tid, tl, nx, ny, cq, dq);
                const int gx0 = tl.gx0, gy0 = tl.gy0;
                for (int q = tid; q < NR; q += NT) {
                    const int a = q % W, b = q / W;
                    const int gi = gx0 + a, gj = gy0 + b;
                    const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
                    const int id = gi + nx * gj;
                    s0[q] = (in && pass > 0) ? bp[pcur][id] : (T)0;
                    // 1/aC does not change in the p' passes: with one tile per
                    // CTA its region stays in s1 after the first pass
                    if (MT || pass == 0) s1[q] = in ? (T)1 / f.ac[id] : (T)0;
                }
                __syncthreads();
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
                        const T r = s1[q];
                        const T e = gi < nx - 1 ? (T)(P.d.Kx * (double)(T)(r + s1[q + 1])) : (T)0;
                        const T w = gi > 0 ? (T)(P.d.Kx * (double)(T)(r + s1[q - 1])) : (T)0;
                        const T n = gj < ny - 1 ? (T)(P.d.Ky * (double)(T)(r + s1[q + W])) : (T)0;
                        const T so = gj > 0 ? (T)(P.d.Ky * (double)(T)(r + s1[q - W])) : (T)0;
                        cE[c][k] = e;
                        cW[c][k] = w;
                        cN[c][k] = n;
                        cS[c][k] = so;
                        cC[c][k] = -(e + w + n + so);
                        cb[c][k] = f.sp[gi + nx * gj];
                        own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
                    }
                const T relax = g.relax[EQ_P];
#pragma unroll 1
                for (int s = 0; s < KS; ++s) {
                    if (s >= ns) break;
                    double sx = 0.0;
#pragma unroll
                    for (int color = 0; color < 2; ++color) {
                        const int reach = 2 * ns - 1 - (2 * s + color);
#pragma unroll
                        for (int k = 0; k < CPT; ++k) {
                            const int q = cq[color][k];
                            if (q < 0 || dq[color][k] > reach) continue;
                            T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k], (T)0, (T)0};
                            T d;
                            s0[q] = point_update<T, 2>(a7, cb[color][k], s0[q], s0[q + 1], s0[q - 1], s0[q + W],
                                                       s0[q - W], (T)0, (T)0, relax, d);
                            if (!last && own[color][k]) sx += (double)d * (double)d;
                        }
                        __syncthreads();
                    }
                    if (!last) {
                        if (wsum) sx = warp_sum(sx);
                        if ((tid & 31) == 0) {
                            if (MT && !first) wred[tid >> 5][s] += sx;
                            else wred[tid >> 5][s] = sx;
                        }
                    }
                }
                for (int q = tid; q < TX * TY; q += NT) {
                    const int a = H + q % TX, b = H + q / TX;
                    const int gi = gx0 + a, gj = gy0 + b;
                    if (gi >= nx || gj >= ny) continue;
                    bp[pcur ^ 1][gi + nx * gj] = s0[b * W + a];
                }
                if (MT) __syncthreads();  // the next tile's staging overwrites the region
            }
            pcur ^= 1;
            if (!last) block_partials<KS, 2 * KS, NT>(&wred[0][0], partials, G);
            if (!grid_sync(bar, G, epoch)) { failed = true; break; }
            if (!last) reduce_partials<KS, NT>(partials, G, tot);
            if (tid == 0) {
                if (last) pass_count(L, EQ_P, ns, N);
                else pass_done(L, EQ_P, tot, ns, N, g.tol[EQ_P]);
            }
            __syncthreads();
        }
        if (failed) break;

        T *const pcc = bp[pcur];  // the current p'
        if (npass_p == 0) {       // no p' sweeps: p' = 0 (src/Solver.cu:193)
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = tl.x0 + q % TX, j = tl.y0 + q / TX;
                    if (i < nx && j < ny) pcc[i + nx * j] = (T)0;
                }
            }
            if (!grid_sync(bar, G, epoch)) break;
        }

        // -------- optional p' mean removal (closed domains, FP64) --------
        if (pa.pin) {
            double m[1] = {0.0};
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = tl.x0 + q % TX, j = tl.y0 + q / TX;
                    if (i < nx && j < ny) m[0] += (double)pcc[i + nx * j];
                }
            }
            write_partials<1, NT>(m, partials, G);
            if (!grid_sync(bar, G, epoch)) break;
            reduce_partials<1, NT>(partials, G, tot);
            const double mean = tot[0] / (double)N;
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = tl.x0 + q % TX, j = tl.y0 + q / TX;
                    if (i < nx && j < ny) pcc[i + nx * j] = (T)((double)pcc[i + nx * j] - mean);
                }
            }
            if (!grid_sync(bar, G, epoch)) break;
        }

        // ---- corrections + next iteration's boundary faces, kernels.cuh:583-843 ----
        {
            double s[7] = {0, 0, 0, 0, 0, 0, 0};
            for (int t = blockIdx.x, tn = 0; MT ? t < ntiles : tn < 1; t += G, ++tn) {
                const Tile tl = MT ? tile_at<TX, TY, H>(t, tiles_x) : tile0;
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = tl.x0 + q % TX, j = tl.y0 + q / TX;
                    if (i >= nx || j >= ny) continue;
                    const int c = i + nx * j;
                    const int fu = i + (nx + 1) * j;
                    // loads first
                    const T pc = pcc[c], aC = f.ac[c];
                    const T pcW = i > 0 ? pcc[c - 1] : (T)0, pcE = i < nx - 1 ? pcc[c + 1] : (T)0;
                    const T pcS = j > 0 ? pcc[c - nx] : (T)0, pcN = j < ny - 1 ? pcc[c + nx] : (T)0;
                    const T acW = i > 0 ? f.ac[c - 1] : (T)1, acS = j > 0 ? f.ac[c - nx] : (T)1;
                    const T p0 = f.p[c], u0 = fc.u[c], v0 = fc.v[c];
                    const T uf0 = i > 0 ? f.uf[fu] : (T)0, vf0 = j > 0 ? f.vf[c] : (T)0;
                    const T dp = g.relax[EQ_P] * pc;
                    const T L_ = i > 0 ? pcW : (g.closed[WEST] ? pc : (T)0);
                    const T R_ = i < nx - 1 ? pcE : (g.closed[EAST] ? pc : (T)0);
                    const T du = vel_corr(P.d.ru[0], L_, R_, g.Ax, aC);
                    const T S_ = j > 0 ? pcS : (g.closed[SOUTH] ? pc : (T)0);
                    const T N_ = j < ny - 1 ? pcN : (g.closed[NORTH] ? pc : (T)0);
                    const T dv = vel_corr(P.d.ru[1], S_, N_, g.Ay, aC);
                    const T un = u0 + du, vn = v0 + dv;
                    f.p[c] = p0 + dp;
                    f.u[c] = un;
                    f.v[c] = vn;
                    if (pcc != f.pc) f.pc[c] = pc;  // keep the p' field current for readers
                    s[0] += (double)dp * (double)dp;
                    s[1] += (double)du * (double)du;
                    s[2] += (double)dv * (double)dv;
                    if (i >= 1) {
                        const T d = face_corr(P.d.ru[0], acW, aC, pcW, pc, g.Ax);
                        f.uf[fu] = uf0 + d;
                        s[4] += (double)d * (double)d;
                    }
                    if (j >= 1) {
                        const T d = face_corr(P.d.ru[1], acS, aC, pcS, pc, g.Ay);
                        f.vf[c] = vf0 + d;
                        s[5] += (double)d * (double)d;
                    }
                    if (i == 0) f.uf[fu] = face_bc(g, WEST, 0, un, j);
                    if (i == nx - 1) f.uf[fu + 1] = face_bc(g, EAST, 0, un, j);
                    if (j == 0) f.vf[c] = face_bc(g, SOUTH, 1, vn, 0);
                    if (j == ny - 1) f.vf[c + nx] = face_bc(g, NORTH, 1, vn, 0);
                }
            }
            write_partials<7, NT>(s, partials, G);
            if (!grid_sync(bar, G, epoch)) break;
            reduce_partials<7, NT>(partials, G, tot);
            reduce_partials<1, NT>(partials + 15 * (size_t)G, G, tot + 8);
        }

        // ---- norms, convergence test, log: src/Solver.cu:226-289 ----
        if (tid == 0) {
            double n[8];
            n[0] = sqrt(tot[0] / (double)N);
            n[1] = sqrt(tot[1] / (double)N);
            n[2] = sqrt(tot[2] / (double)N);
            n[3] = 0.0;
            n[4] = sqrt(tot[4] / ((double)(nx - 1) * ny));
            n[5] = sqrt(tot[5] / ((double)nx * (ny - 1)));
            n[6] = 0.0;
            n[7] = sqrt(tot[8] / (double)N);
            bool bad = false;
            for (int q = 0; q < 8; ++q) bad = bad || !isfinite(n[q]);
            const int it = L.it + 1;
            if (!bad && it - L.it_begin > 1)
                for (int q = 0; q < 7; ++q) bad = bad || (L.maxn[q] > 0.0 && n[q] > 1e6 * L.maxn[q]);
            double rel[7];
            if (g.criterion == 0) {
                if (n[0] > L.maxn[0]) L.maxn[0] = n[0];
                for (int q = 0; q < 7; ++q) rel[q] = n[q] / L.maxn[0];
            } else {
                for (int q = 0; q < 7; ++q) {
                    if (q == 3 || q == 6) { rel[q] = 0.0; continue; }
                    if (n[q] > L.maxn[q]) L.maxn[q] = n[q];
                    rel[q] = L.maxn[q] > 0.0 ? n[q] / L.maxn[q] : 0.0;
                }
            }
            bool conv = rel[0] < g.tol[EQ_P] && rel[1] < g.tol[EQ_U] && rel[2] < g.tol[EQ_V] &&
                        rel[4] < g.tol[EQ_U] && rel[5] < g.tol[EQ_V];
            conv = conv || n[7] < g.tol_mass;
            const int local = it - L.it_begin;
            const bool last = it >= L.it_stop || (L.act && conv) || bad;
            L.it = it;
            if (bad) L.status = 2;
            if (blockIdx.x == 0) {
                for (int q = 0; q < 7; ++q) ctl->sq[q] = tot[q];
                ctl->sq[SQ_MASS] = tot[8];
                for (int q = 0; q < 8; ++q) {
                    ctl->norm[q] = n[q];
                    ctl->maxn[q] = L.maxn[q];
                }
                for (int q = 0; q < 7; ++q) ctl->rel[q] = rel[q];
                ctl->it = it;
                ctl->converged = conv ? 1 : 0;
                if (bad) ctl->status = 2;
                for (int q = 0; q < 4; ++q) ctl->it_sweeps[q] = L.sweeps[q];
                ctl->cell_updates = L.cell_updates;
                if (L.log_level > 0 && (local == 1 || local % 1000 == 0 || conv || last)) {
                    const int slot = L.log_n < kLogCap ? L.log_n : kLogCap - 1;
                    LogRec &R2 = ctl->log[slot];
                    R2.it = local;
                    R2.converged = conv;
                    for (int q = 0; q < 7; ++q) R2.rel[q] = rel[q];
                    R2.mass = n[7];
                    if (L.log_n < kLogCap) L.log_n++;
                    ctl->log_n = L.log_n;
                }
            }
            L.done = last;
        }
        __syncthreads();
    }
    if (tid == 0) {
        const bool to = bar->err != 0;
        if (to) atomicExch(&ctl->status, 3);
        if (blockIdx.x == 0) {
            for (int q = 0; q < 4; ++q) {
                ctl->stop[q] = 0;
                ctl->sweeps[q] = 0;
                ctl->inner_max[q] = -1e20;
            }
        }
    }
}

}  // namespace ifc
