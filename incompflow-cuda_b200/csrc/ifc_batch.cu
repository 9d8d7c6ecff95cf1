// ifc_batch.cu -- many independent 2D SIMPLE solves in one persistent kernel.
//
// Work distribution: the kernel is launched as thread-block clusters of kCL
// CTAs; each cluster takes the next case from a device queue (cases are queued
// largest first), runs up to `chunk` SIMPLE outer iterations of it
// (src/Solver.cu:160-289, the same per-cell arithmetic as every other path,
// ifc_physics.cuh), saves its loop state and takes the next case.  The CTAs of
// a cluster split a case's rows between their warps and synchronise with the
// hardware cluster barrier; block sums are combined across the cluster through
// distributed shared memory in rank order, so every norm is deterministic and
// every CTA of the cluster takes the same decisions.  Fields live in global
// memory (L1/L2 resident for these sizes).  The host runs the kernel inside a
// CUDA graph whose conditional WHILE node relaunches it until every case has
// converged, diverged or used its iteration budget.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cooperative_groups.h>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "ifc.h"
#include "ifc_engine.cuh"

namespace cg = cooperative_groups;

namespace ifc {
namespace {

constexpr int kCL = 8;     // CTAs per cluster (portable cluster size)
constexpr int kBNT = 256;  // threads per CTA

template <typename T>
struct BCase {
    Params<T> P;
    long long off_c, off_uf, off_vf;  // offsets into the pools
    int n_iter[4];
    int pin;
    int max_outer;
};

struct BState {
    int it, done, converged, status;
    int sweeps[4];
    double maxn[8];
    double norm[8];
    double rel[7];
};

template <typename T>
struct BPools {
    T *u, *v, *p, *pc, *uf, *vf, *ac, *rac, *sp;
    T *le, *ln, *lc;  // p' links of each cell: east, north, diagonal
    T *sdu, *sdv;     // deferred-correction sources (higher-order convection; null when no case uses it)
};

struct BQueue {
    unsigned int next;
    unsigned int exited;
    int pad[2];
};

// Case-local loop state shared by the threads of one CTA.
struct CaseLoop {
    int stop[4];
    double inner_max[4];
    int sweeps[4];
};

// Sum NV values over the threads of the CTA into this CTA's slot `part`
// (shared memory); call with every thread.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *part)
{
    __shared__ double red[kBNT / 32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < NV; ++r) {
        const double t = warp_sum(v[r]);
        if (lane == 0) red[warp][r] = t;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int w = 0; w < kBNT / 32; ++w) t += red[w][threadIdx.x];
        part[threadIdx.x] = t;
    }
}

// After a cluster barrier: the cluster-wide sums of the NV slots `part` of
// every CTA, added in rank order (identical in every CTA).
template <int NV>
__device__ __forceinline__ void cluster_total(cg::cluster_group &cl, double *part, double *out)
{
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int r = 0; r < kCL; ++r) t += cl.map_shared_rank(part, r)[threadIdx.x];
        out[threadIdx.x] = t;
    }
    __syncthreads();
}

template <typename T>
__device__ __forceinline__ T rcx(const Geo<T> &g, const T *u, const T *ac, const T *p, int i, int row)
{
    const int R = i + g.nx * row, L = R - 1;
    const T pL = p[L], pR = p[R];
    const T pLL = i >= 2 ? p[L - 1] : (g.closed[WEST] ? pL : (T)0);
    const T pRR = i <= g.nx - 2 ? p[R + 1] : (g.closed[EAST] ? pR : (T)0);
    return rc_face(u[L], u[R], ac[L], ac[R], pLL, pL, pR, pRR, g.Ax);
}

template <typename T>
__device__ __forceinline__ T rcy(const Geo<T> &g, const T *v, const T *ac, const T *p, int i, int j)
{
    const int nx = g.nx, R = i + nx * j, L = R - nx;
    const T pL = p[L], pR = p[R];
    const T pLL = j >= 2 ? p[L - nx] : (g.closed[SOUTH] ? pL : (T)0);
    const T pRR = j <= g.ny - 2 ? p[R + nx] : (g.closed[NORTH] ? pR : (T)0);
    return rc_face(v[L], v[R], ac[L], ac[R], pLL, pL, pR, pRR, g.Ay);
}

template <typename T>
__global__ void __cluster_dims__(kCL, 1, 1) __launch_bounds__(kBNT, 4)
    k_batch2d(const BCase<T> *cases, BState *states, BPools<T> pool, int ncases, BQueue *q, int chunk,
              cudaGraphConditionalHandle cond, int use_cond)
{
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int tid = threadIdx.x, lane = tid & 31;
    const int gw = (int)rank * (kBNT / 32) + (tid >> 5);  // warp index within the cluster
    constexpr int TW = kCL * kBNT / 32;                   // warps per cluster

    __shared__ int s_case;
    __shared__ BCase<T> C;
    __shared__ CaseLoop L;
    __shared__ BState S;
    // This CTA's block sums.  Slots: momentum sweeps [b][0..1] and p' sweeps
    // [b][2] double-buffered by sweep parity (a buffer is rewritten only two
    // cluster barriers after every CTA read it), mass [0][3], p' mean [0][4],
    // corrections [0][5..9]; no two phases share a slot.
    __shared__ double part[2][16];
    __shared__ double tot[16];      // cluster totals

    for (;;) {
        if (rank == 0 && tid == 0) s_case = (int)atomicAdd(&q->next, 1u);
        cl.sync();
        const int cid = *cl.map_shared_rank(&s_case, 0);
        if (cid >= ncases) break;
        // every CTA has read rank 0's s_case before rank 0 overwrites it
        if (tid == 0) {
            C = cases[cid];
            S = states[cid];
        }
        cl.sync();
        if (S.done) continue;

        const Params<T> &P = C.P;
        const Geo<T> &g = P.g;
        const int nx = g.nx, ny = g.ny, N = g.N;
        const int hx = (nx + 1) / 2;
        T *u = pool.u + C.off_c, *v = pool.v + C.off_c, *p = pool.p + C.off_c, *pc = pool.pc + C.off_c;
        T *ac = pool.ac + C.off_c, *rac = pool.rac + C.off_c, *sp = pool.sp + C.off_c;
        T *uf = pool.uf + C.off_uf, *vf = pool.vf + C.off_vf;
        T *le = pool.le + C.off_c, *ln = pool.ln + C.off_c, *lc = pool.lc + C.off_c;

        // First iteration of the case: interior faces from cell means, then
        // the face boundary conditions (kernels.cuh:10-95).
        if (S.it == 0) {
            for (int j = gw; j < ny + 1; j += TW)
                for (int i = lane; i < nx + 1; i += 32) {
                    if (j < ny) {
                        const int c = i + nx * j;
                        T val;
                        if (i == 0) val = face_bc(g, WEST, 0, u[c], j);
                        else if (i == nx) val = face_bc(g, EAST, 0, u[c - 1], j);
                        else val = (u[c - 1] + u[c]) / (T)2;
                        uf[i + (nx + 1) * j] = val;
                    }
                    if (i < nx) {
                        const int c = i + nx * j;
                        T val;
                        if (j == 0) val = face_bc(g, SOUTH, 1, v[c], 0);
                        else if (j == ny) val = face_bc(g, NORTH, 1, v[c - nx], 0);
                        else val = (v[c - nx] + v[c]) / (T)2;
                        vf[c] = val;
                    }
                }
            cl.sync();
        }

        for (int k = 0; k < chunk && !S.done; ++k) {
            if (tid == 0)
                for (int e = 0; e < 4; ++e) {
                    L.stop[e] = 0;
                    L.inner_max[e] = -1e20;
                    L.sweeps[e] = 0;
                }
            __syncthreads();

            // ---- deferred-correction sources of a higher-order convection scheme
            // (ifc_convection.cuh), from the fields at the start of the iteration
            if (g.conv != CONV_UPWIND) {
                T *du = pool.sdu + C.off_c, *dv = pool.sdv + C.off_c;
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) {
                        const int c = i + nx * j, fu = i + (nx + 1) * j;
                        const T uw = uf[fu], ue = uf[fu + 1], vs = vf[c], vn = vf[c + nx];
                        du[c] = dc_cell<T, 2>(g, u, c, i, j, 0, uw, ue, vs, vn, (T)0, (T)0);
                        dv[c] = dc_cell<T, 2>(g, v, c, i, j, 0, uw, ue, vs, vn, (T)0, (T)0);
                    }
                cl.sync();
            }

            // ---- momentum sweeps, coefficients on the fly (kernels.cuh:97-334, 926-1005)
            const int nm = max(C.n_iter[0], C.n_iter[1]);
            for (int s = 0; s < (nm > 0 ? nm : 1); ++s) {
                const bool du = s < C.n_iter[0] && !L.stop[EQ_U];
                const bool dv = s < C.n_iter[1] && !L.stop[EQ_V];
                if (!du && !dv && s > 0) break;
                double sq[2] = {0.0, 0.0};
                for (int color = 0; color < 2; ++color) {
                    for (int j = gw; j < ny; j += TW)
                        for (int i2 = lane; i2 < hx; i2 += 32) {
                            const int i = 2 * i2 + ((color + j) & 1);
                            if (i >= nx) continue;
                            const int c = i + nx * j;
                            const int fu = i + (nx + 1) * j;
                            T a[7], b[3];
                            mom_cell<T, 2>(P, i, j, 0, uf[fu], uf[fu + 1], vf[c], vf[c + nx], (T)0, (T)0, p[c],
                                           i > 0 ? p[c - 1] : (T)0, i < nx - 1 ? p[c + 1] : (T)0,
                                           j > 0 ? p[c - nx] : (T)0, j < ny - 1 ? p[c + nx] : (T)0, (T)0, (T)0, a,
                                           b);
                            if (g.conv != CONV_UPWIND) {
                                b[0] = b[0] + pool.sdu[C.off_c + c];
                                b[1] = b[1] + pool.sdv[C.off_c + c];
                            }
                            if (s == 0) ac[c] = a[AC];
                            T d;
                            if (du) {
                                const T e = i < nx - 1 ? u[c + 1] : (T)0, w = i > 0 ? u[c - 1] : (T)0;
                                const T n = j < ny - 1 ? u[c + nx] : (T)0, so = j > 0 ? u[c - nx] : (T)0;
                                u[c] = point_update<T, 2>(a, b[0], u[c], e, w, n, so, (T)0, (T)0, g.relax[EQ_U], d);
                                sq[0] += (double)d * (double)d;
                            }
                            if (dv) {
                                const T e = i < nx - 1 ? v[c + 1] : (T)0, w = i > 0 ? v[c - 1] : (T)0;
                                const T n = j < ny - 1 ? v[c + nx] : (T)0, so = j > 0 ? v[c - nx] : (T)0;
                                v[c] = point_update<T, 2>(a, b[1], v[c], e, w, n, so, (T)0, (T)0, g.relax[EQ_V], d);
                                sq[1] += (double)d * (double)d;
                            }
                        }
                    if (color == 1) block_sum<2>(sq, part[s & 1]);
                    cl.sync();
                }
                // early-exit rule of src/Solver.cu:955-962 on this sweep's norms
                cluster_total<2>(cl, part[s & 1], tot);
                if (tid == 0) {
                    for (int m = 0; m < 2; ++m) {
                        if (!(m == 0 ? du : dv)) continue;
                        const double rms = sqrt(tot[m] / (double)N);
                        if (rms > L.inner_max[m]) L.inner_max[m] = rms;
                        if (rms / (L.inner_max[m] + 1e-20) < g.tol[m]) L.stop[m] = 1;
                        L.sweeps[m]++;
                    }
                }
                __syncthreads();
            }

            // ---- Rhie-Chow faces, face BCs, p' source, 1/aC (kernels.cuh:336-581)
            {
                double m[1] = {0.0};
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) {
                        const int c = i + nx * j;
                        const T uw = i == 0 ? face_bc(g, WEST, 0, u[c], j) : rcx(g, u, ac, p, i, j);
                        const T ue = i == nx - 1 ? face_bc(g, EAST, 0, u[c], j) : rcx(g, u, ac, p, i + 1, j);
                        const T vs = j == 0 ? face_bc(g, SOUTH, 1, v[c], 0) : rcy(g, v, ac, p, i, j);
                        const T vn = j == ny - 1 ? face_bc(g, NORTH, 1, v[c], 0) : rcy(g, v, ac, p, i, j + 1);
                        const T bb = mass_imbalance<T, 2>(g, uw, ue, vs, vn, (T)0, (T)0);
                        const T r = (T)1 / ac[c];
                        uf[i + (nx + 1) * j] = uw;
                        if (i == nx - 1) uf[nx + (nx + 1) * j] = ue;
                        vf[c] = vs;
                        if (j == ny - 1) vf[c + nx] = vn;
                        sp[c] = bb;
                        rac[c] = r;
                        m[0] += (double)bb * (double)bb;
                    }
                block_sum<1>(m, &part[0][3]);
                cl.sync();
                cluster_total<1>(cl, &part[0][3], &tot[8]);  // tot[8]: mass
            }

            // ---- p' links, once per outer iteration (kernels.cuh:517-537):
            // -0.5 rho A^2 (1/aC_C + 1/aC_nb) on interior faces, 0 on boundaries.
            for (int j = gw; j < ny; j += TW)
                for (int i = lane; i < nx; i += 32) {
                    const int c = i + nx * j;
                    const T r = rac[c];
                    const T e = i < nx - 1 ? (T)(P.d.Kx * (double)(T)(r + rac[c + 1])) : (T)0;
                    const T w = i > 0 ? (T)(P.d.Kx * (double)(T)(r + rac[c - 1])) : (T)0;
                    const T n = j < ny - 1 ? (T)(P.d.Ky * (double)(T)(r + rac[c + nx])) : (T)0;
                    const T so = j > 0 ? (T)(P.d.Ky * (double)(T)(r + rac[c - nx])) : (T)0;
                    le[c] = e;
                    ln[c] = n;
                    lc[c] = -(e + w + n + so);
                }
            cl.sync();

            // ---- p' sweeps from p' = 0 (src/Solver.cu:193-196, kernels.cuh:502-540)
            const double mass_sq = tot[8];
            for (int s = 0; s < C.n_iter[3]; ++s) {
                if (L.stop[EQ_P]) break;
                double sq[1] = {0.0};
                for (int color = 0; color < 2; ++color) {
                    const int zm = s == 0 ? (color == 0 ? 1 : 2) : 0;
                    for (int j = gw; j < ny; j += TW)
                        for (int i2 = lane; i2 < hx; i2 += 32) {
                            const int i = 2 * i2 + ((color + j) & 1);
                            if (i >= nx) continue;
                            const int c = i + nx * j;
                            T a[7];
                            a[AE] = le[c];
                            a[AW] = i > 0 ? le[c - 1] : (T)0;
                            a[AN] = ln[c];
                            a[AS] = j > 0 ? ln[c - nx] : (T)0;
                            a[AT] = a[AB] = (T)0;
                            a[AC] = lc[c];
                            const bool zn = zm == 1;
                            const T e = (!zn && i < nx - 1) ? pc[c + 1] : (T)0, w = (!zn && i > 0) ? pc[c - 1] : (T)0;
                            const T n = (!zn && j < ny - 1) ? pc[c + nx] : (T)0;
                            const T so = (!zn && j > 0) ? pc[c - nx] : (T)0;
                            T d;
                            pc[c] = point_update<T, 2>(a, sp[c], zm ? (T)0 : pc[c], e, w, n, so, (T)0, (T)0,
                                                       g.relax[EQ_P], d);
                            sq[0] += (double)d * (double)d;
                        }
                    if (color == 1) block_sum<1>(sq, &part[s & 1][2]);
                    cl.sync();
                }
                cluster_total<1>(cl, &part[s & 1][2], tot);
                if (tid == 0) {
                    const double rms = sqrt(tot[0] / (double)N);
                    if (rms > L.inner_max[EQ_P]) L.inner_max[EQ_P] = rms;
                    if (rms / (L.inner_max[EQ_P] + 1e-20) < g.tol[EQ_P]) L.stop[EQ_P] = 1;
                    L.sweeps[EQ_P]++;
                }
                __syncthreads();
            }
            if (C.n_iter[3] == 0) {
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) pc[i + nx * j] = (T)0;
                cl.sync();
            }

            // ---- FP64 removal of the p' mean (closed cavities)
            if (C.pin) {
                double m[1] = {0.0};
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) m[0] += (double)pc[i + nx * j];
                block_sum<1>(m, &part[0][4]);
                cl.sync();
                cluster_total<1>(cl, &part[0][4], &tot[12]);
                const double mean = tot[12] / (double)N;
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) pc[i + nx * j] = (T)((double)pc[i + nx * j] - mean);
                cl.sync();
            }

            // ---- corrections + next iteration's boundary faces (kernels.cuh:583-843)
            {
                double sq[5] = {0, 0, 0, 0, 0};
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) {
                        const int c = i + nx * j, fu = i + (nx + 1) * j;
                        const T x = pc[c], aC = ac[c];
                        const T xW = i > 0 ? pc[c - 1] : (T)0, xE = i < nx - 1 ? pc[c + 1] : (T)0;
                        const T xS = j > 0 ? pc[c - nx] : (T)0, xN = j < ny - 1 ? pc[c + nx] : (T)0;
                        const T aW = i > 0 ? ac[c - 1] : (T)1, aS = j > 0 ? ac[c - nx] : (T)1;
                        const T p0 = p[c], u0 = u[c], v0 = v[c];
                        const T uf0 = i > 0 ? uf[fu] : (T)0, vf0 = j > 0 ? vf[c] : (T)0;
                        const T dp = g.relax[EQ_P] * x;
                        const T Lx = i > 0 ? xW : (g.closed[WEST] ? x : (T)0);
                        const T Rx = i < nx - 1 ? xE : (g.closed[EAST] ? x : (T)0);
                        const T dU = vel_corr(P.d.ru[0], Lx, Rx, g.Ax, aC);
                        const T Sy = j > 0 ? xS : (g.closed[SOUTH] ? x : (T)0);
                        const T Ny = j < ny - 1 ? xN : (g.closed[NORTH] ? x : (T)0);
                        const T dV = vel_corr(P.d.ru[1], Sy, Ny, g.Ay, aC);
                        const T un = u0 + dU, vn = v0 + dV;
                        p[c] = p0 + dp;
                        u[c] = un;
                        v[c] = vn;
                        sq[0] += (double)dp * (double)dp;
                        sq[1] += (double)dU * (double)dU;
                        sq[2] += (double)dV * (double)dV;
                        if (i >= 1) {
                            const T d = face_corr(P.d.ru[0], aW, aC, xW, x, g.Ax);
                            uf[fu] = uf0 + d;
                            sq[3] += (double)d * (double)d;
                        }
                        if (j >= 1) {
                            const T d = face_corr(P.d.ru[1], aS, aC, xS, x, g.Ay);
                            vf[c] = vf0 + d;
                            sq[4] += (double)d * (double)d;
                        }
                        if (i == 0) uf[fu] = face_bc(g, WEST, 0, un, j);
                        if (i == nx - 1) uf[fu + 1] = face_bc(g, EAST, 0, un, j);
                        if (j == 0) vf[c] = face_bc(g, SOUTH, 1, vn, 0);
                        if (j == ny - 1) vf[c + nx] = face_bc(g, NORTH, 1, vn, 0);
                    }
                block_sum<5>(sq, &part[0][5]);
                cl.sync();
                cluster_total<5>(cl, &part[0][5], tot);
            }

            // ---- norms and convergence test (src/Solver.cu:226-268), per-field rule
            if (tid == 0) {
                double n[8];
                n[0] = sqrt(tot[0] / (double)N);
                n[1] = sqrt(tot[1] / (double)N);
                n[2] = sqrt(tot[2] / (double)N);
                n[3] = 0.0;
                n[4] = sqrt(tot[3] / ((double)(nx - 1) * ny));
                n[5] = sqrt(tot[4] / ((double)nx * (ny - 1)));
                n[6] = 0.0;
                n[7] = sqrt(mass_sq / (double)N);
                bool bad = false;
                for (int e = 0; e < 8; ++e) bad = bad || !isfinite(n[e]);
                double rel[7];
                if (g.criterion == 0) {
                    if (n[0] > S.maxn[0]) S.maxn[0] = n[0];
                    for (int e = 0; e < 7; ++e) rel[e] = n[e] / S.maxn[0];
                } else {
                    for (int e = 0; e < 7; ++e) {
                        if (e == 3 || e == 6) { rel[e] = 0.0; continue; }
                        if (n[e] > S.maxn[e]) S.maxn[e] = n[e];
                        rel[e] = S.maxn[e] > 0.0 ? n[e] / S.maxn[e] : 0.0;
                    }
                }
                bool conv = rel[0] < g.tol[EQ_P] && rel[1] < g.tol[EQ_U] && rel[2] < g.tol[EQ_V] &&
                            rel[4] < g.tol[EQ_U] && rel[5] < g.tol[EQ_V];
                conv = conv || n[7] < g.tol_mass;
                S.it += 1;
                S.converged = conv ? 1 : 0;
                if (bad) S.status = 2;
                S.done = conv || bad || S.it >= C.max_outer;
                for (int e = 0; e < 8; ++e) S.norm[e] = n[e];
                for (int e = 0; e < 7; ++e) S.rel[e] = rel[e];
                for (int e = 0; e < 4; ++e) S.sweeps[e] = L.sweeps[e];
            }
            __syncthreads();
        }
        if (rank == 0 && tid == 0) states[cid] = S;
        // no CTA may start the next case (and overwrite its shared state)
        // while another still reads rank 0's slots
        cl.sync();
    }
    // Loop control for the next graph iteration: the last CTA to leave checks
    // whether any case still has work and resets the queue.
    cl.sync();
    if (tid == 0) {
        __threadfence();
        const unsigned int t = atomicAdd(&q->exited, 1u);
        if (t == gridDim.x - 1) {
            __threadfence();
            int left = 0;
            for (int c = 0; c < ncases; ++c) left |= !((volatile BState *)states)[c].done;
            q->next = 0;
            q->exited = 0;
            __threadfence();
            if (use_cond) cudaGraphSetConditional(cond, left ? 1u : 0u);
        }
    }
}

#include "ifc_batch_tb.cuh"

// ---- variants and the autotuner ---------------------------------------------
// Variant 0 sweeps whole rows with one cluster barrier per half sweep
// (k_batch2d); the others are temporally blocked (k_batch_tb) with the tile
// shape and sweeps per pass of the table.  A case's size class selects its
// variant: the autotuner times every variant on copies of the class's median
// case (a fixed number of outer iterations) the first time a class is met in a
// process, and keeps the fastest.  IFC_BATCH_VARIANT=<k> forces variant k.
struct BVariant {
    int tx, ty, ks, nt;
};
constexpr int kNumVariants = 3;
constexpr BVariant kVariants[kNumVariants] = {{0, 0, 1, kBNT}, {32, 8, 3, 256}, {32, 16, 5, 512}};
constexpr int kNumClasses = 3;

static int size_class(int nx, int ny)
{
    const long long cells = (long long)nx * ny;
    return cells <= 64 * 64 ? 0 : (cells <= 160 * 160 ? 1 : 2);
}

template <typename T>
static const void *variant_kernel(int v)
{
    switch (v) {
    case 1: return (const void *)k_batch_tb<T, 32, 8, 3, 256>;
    case 2: return (const void *)k_batch_tb<T, 32, 16, 5, 512>;
    default: return (const void *)k_batch2d<T>;
    }
}

template <typename T>
static size_t variant_smem(int v)
{
    const BVariant &b = kVariants[v];
    if (b.tx == 0) return 0;
    const int W = b.tx + 4 * b.ks, HH = b.ty + 4 * b.ks;
    return (size_t)3 * W * HH * sizeof(T);
}

template <typename T>
static cudaError_t variant_clusters(int v, int *nclusters)
{
    const void *kern = variant_kernel<T>(v);
    const size_t smem = variant_smem<T>(v);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(kCL);
    lc.blockDim = dim3(kVariants[v].nt);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = kCL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(nclusters, kern, &lc);
}

template <typename T>
static void launch_variant(int v, int nclusters, cudaStream_t st, const BCase<T> *dc, BState *ds, BPools<T> pool,
                           TBPools<T> tp, int n, BQueue *dq, int chunk, cudaGraphConditionalHandle cond)
{
    const size_t smem = variant_smem<T>(v);
    switch (v) {
    case 1:
        k_batch_tb<T, 32, 8, 3, 256><<<nclusters * kCL, 256, smem, st>>>(dc, ds, pool, tp, n, dq, chunk, cond, 1);
        break;
    case 2:
        k_batch_tb<T, 32, 16, 5, 512><<<nclusters * kCL, 512, smem, st>>>(dc, ds, pool, tp, n, dq, chunk, cond, 1);
        break;
    default: k_batch2d<T><<<nclusters * kCL, kBNT, 0, st>>>(dc, ds, pool, n, dq, chunk, cond, 1); break;
    }
}

#define BCK(call)                                                                  \
    do {                                                                           \
        if ((call) != cudaSuccess) {                                               \
            rc = IFC_CUDA_ERROR;                                                   \
            goto done;                                                             \
        }                                                                          \
    } while (0)

template <typename T>
static int batch_run(const ifc_config *cfgs, int n, int force_variant, ifc_batch_result *res, void *const *fields_out,
                     double *ms_out);

// Variant chosen for each size class and precision in this process.
static std::mutex g_tune_mu;
static int g_tuned[2][kNumClasses] = {{-1, -1, -1}, {-1, -1, -1}};

template <typename T>
static int autotune(int cls, const ifc_config &rep)
{
    // Probe: copies of the class's median case, 20 outer iterations each (no
    // early stop), enough copies to fill the GPU with any variant.
    constexpr int kCopies = 96;
    std::vector<ifc_config> probe(kCopies, rep);
    for (ifc_config &c : probe) {
        c.convection_scheme = IFC_CONV_UPWIND;  // the variants differ in their sweeps only
        c.tol_u = c.tol_v = c.tol_w = c.tol_p = 0.0;
        c.tol_mass = 0.0;
        c.num_outer_iter = 20;
    }
    std::vector<ifc_batch_result> r(kCopies);
    int best = 0;
    double best_ms = 0.0;
    for (int v = 0; v < kNumVariants; ++v) {
        double ms = 0.0;
        if (batch_run<T>(probe.data(), kCopies, v, r.data(), nullptr, &ms) != IFC_OK) continue;
        if (getenv("IFC_VERBOSE"))
            fprintf(stderr, "ifc_batch autotune: class %d (%dx%d) variant %d: %.3f ms\n", cls, rep.nx, rep.ny, v, ms);
        if (best_ms == 0.0 || ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    return best;
}

template <typename T>
static int batch_solve(const ifc_config *cfgs, int n, ifc_batch_result *res, void *const *fields_out, double *ms_out)
{
    const char *env = getenv("IFC_BATCH_VARIANT");
    if (env && env[0] >= '0' && env[0] < '0' + kNumVariants)
        return batch_run<T>(cfgs, n, env[0] - '0', res, fields_out, ms_out);
    const int prec = sizeof(T) == 8 ? 1 : 0;
    for (int cls = 0; cls < kNumClasses; ++cls) {
        std::vector<int> members;
        for (int c = 0; c < n; ++c)
            if (size_class(cfgs[c].nx, cfgs[c].ny) == cls) members.push_back(c);
        if (members.empty()) continue;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            if (g_tuned[prec][cls] >= 0) continue;
        }
        std::sort(members.begin(), members.end(), [&](int x, int y) {
            return (long long)cfgs[x].nx * cfgs[x].ny < (long long)cfgs[y].nx * cfgs[y].ny;
        });
        const int v = autotune<T>(cls, cfgs[members[members.size() / 2]]);
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[prec][cls] = v;
    }
    return batch_run<T>(cfgs, n, -1, res, fields_out, ms_out);
}

// Solves the cases; force_variant >= 0 runs every case with that variant,
// otherwise each size class runs its tuned variant, largest class first, each
// class as one persistent launch relaunched by a CUDA graph WHILE node.
template <typename T>
static int batch_run(const ifc_config *cfgs, int n, int force_variant, ifc_batch_result *res, void *const *fields_out,
                     double *ms_out)
{
    int rc = IFC_OK;
    const int prec = sizeof(T) == 8 ? 1 : 0;
    std::vector<BCase<T>> hc(n);
    std::vector<int> variant(n);
    long long nc = 0, nuf = 0, nvf = 0;
    for (int c = 0; c < n; ++c) {
        BCase<T> &b = hc[c];
        std::memset(&b, 0, sizeof(b));
        b.P = make_params<T>(cfgs[c]);
        b.off_c = nc;
        b.off_uf = nuf;
        b.off_vf = nvf;
        nc += (long long)cfgs[c].nx * cfgs[c].ny;
        nuf += (long long)(cfgs[c].nx + 1) * cfgs[c].ny;
        nvf += (long long)cfgs[c].nx * (cfgs[c].ny + 1);
        b.n_iter[0] = cfgs[c].n_iter_u;
        b.n_iter[1] = cfgs[c].n_iter_v;
        b.n_iter[2] = 0;
        b.n_iter[3] = cfgs[c].n_iter_p;
        bool closed = true;
        for (int f = 0; f < 4; ++f) closed = closed && cfgs[c].vel_bc_type[f] != IFC_OUTLET;
        b.pin = cfgs[c].pin_pressure == 1 || (cfgs[c].pin_pressure < 0 && closed);
        b.max_outer = cfgs[c].num_outer_iter;
        if (cfgs[c].convection_scheme != IFC_CONV_UPWIND) {
            variant[c] = 0;  // only the whole-row kernel applies the deferred correction
        } else if (force_variant >= 0) {
            variant[c] = force_variant;
        } else {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            const int v = g_tuned[prec][size_class(cfgs[c].nx, cfgs[c].ny)];
            variant[c] = v < 0 ? 0 : v;
        }
    }
    // One queue per variant, largest grids first (longest-processing-time
    // heuristic); the queue with the most work runs first.
    std::vector<std::vector<int>> groups(kNumVariants);
    std::vector<long long> work(kNumVariants, 0);
    for (int c = 0; c < n; ++c) {
        groups[variant[c]].push_back(c);
        work[variant[c]] += (long long)cfgs[c].nx * cfgs[c].ny;
    }
    std::vector<int> vorder;
    for (int v = 0; v < kNumVariants; ++v)
        if (!groups[v].empty()) vorder.push_back(v);
    std::sort(vorder.begin(), vorder.end(), [&](int x, int y) { return work[x] > work[y]; });
    std::vector<int> order;  // queue position -> case
    std::vector<int> qbegin, qsize;
    for (int v : vorder) {
        std::vector<int> &g = groups[v];
        std::stable_sort(g.begin(), g.end(), [&](int x, int y) {
            return (long long)cfgs[x].nx * cfgs[x].ny > (long long)cfgs[y].nx * cfgs[y].ny;
        });
        qbegin.push_back((int)order.size());
        qsize.push_back((int)g.size());
        order.insert(order.end(), g.begin(), g.end());
    }
    std::vector<BCase<T>> queued(n);
    for (int k = 0; k < n; ++k) queued[k] = hc[order[k]];

    BPools<T> pool;
    std::memset(&pool, 0, sizeof(pool));
    TBPools<T> tp = {nullptr, nullptr, nullptr};
    BCase<T> *dcases = nullptr;
    BState *dstates = nullptr;
    BQueue *dq = nullptr;
    cudaStream_t st = nullptr;
    std::vector<cudaGraph_t> graphs;
    std::vector<cudaGraphExec_t> execs;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<BState> hs(n);
    {
        T **cell_arrays[] = {&pool.u, &pool.v, &pool.p, &pool.pc, &pool.ac, &pool.rac, &pool.sp,
                             &pool.le, &pool.ln, &pool.lc, &tp.tu, &tp.tv, &tp.tpc};
        for (T **a : cell_arrays) {
            BCK(cudaMalloc(a, nc * sizeof(T)));
            BCK(cudaMemset(*a, 0, nc * sizeof(T)));
        }
        bool any_dc = false;
        for (int c = 0; c < n; ++c) any_dc = any_dc || cfgs[c].convection_scheme != IFC_CONV_UPWIND;
        if (any_dc) {
            BCK(cudaMalloc(&pool.sdu, nc * sizeof(T)));
            BCK(cudaMalloc(&pool.sdv, nc * sizeof(T)));
        }
        BCK(cudaMalloc(&pool.uf, nuf * sizeof(T)));
        BCK(cudaMalloc(&pool.vf, nvf * sizeof(T)));
        BCK(cudaMemset(pool.uf, 0, nuf * sizeof(T)));
        BCK(cudaMemset(pool.vf, 0, nvf * sizeof(T)));
        BCK(cudaMalloc(&dcases, n * sizeof(BCase<T>)));
        BCK(cudaMemcpy(dcases, queued.data(), n * sizeof(BCase<T>), cudaMemcpyHostToDevice));
        BCK(cudaMalloc(&dstates, n * sizeof(BState)));
        BCK(cudaMemset(dstates, 0, n * sizeof(BState)));
        BCK(cudaMalloc(&dq, sizeof(BQueue)));
        BCK(cudaMemset(dq, 0, sizeof(BQueue)));
        BCK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        BCK(cudaEventCreate(&e0));
        BCK(cudaEventCreate(&e1));
        const int chunk = 250;

        // One graph per queue: WHILE (a case of the queue is unfinished) { kernel }
        for (size_t gq = 0; gq < vorder.size(); ++gq) {
            const int v = vorder[gq];
            int nclusters = 0;
            BCK(variant_clusters<T>(v, &nclusters));
            if (nclusters < 1) nclusters = 1;
            if (nclusters > qsize[gq]) nclusters = qsize[gq];
            if (getenv("IFC_VERBOSE"))
                fprintf(stderr, "ifc_batch_solve: queue of %d cases, variant %d, %d clusters of %d CTAs\n", qsize[gq],
                        v, nclusters, kCL);
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            cudaGraphConditionalHandle cond;
            BCK(cudaGraphCreate(&graph, 0));
            graphs.push_back(graph);
            BCK(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = cond;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            BCK(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            BCK(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
            launch_variant<T>(v, nclusters, st, dcases + qbegin[gq], dstates + qbegin[gq], pool, tp, qsize[gq], dq,
                              chunk, cond);
            BCK(cudaStreamEndCapture(st, &body));
            BCK(cudaGraphInstantiate(&exec, graph, 0));
            execs.push_back(exec);
        }
        BCK(cudaEventRecord(e0, st));
        for (cudaGraphExec_t x : execs) BCK(cudaGraphLaunch(x, st));
        BCK(cudaEventRecord(e1, st));
        BCK(cudaStreamSynchronize(st));
        BCK(cudaGetLastError());
        float ms = 0.f;
        BCK(cudaEventElapsedTime(&ms, e0, e1));
        if (ms_out) *ms_out = ms;
        BCK(cudaMemcpy(hs.data(), dstates, n * sizeof(BState), cudaMemcpyDeviceToHost));
        for (int k = 0; k < n; ++k) {
            const int c = order[k];
            const BState &s = hs[k];
            ifc_batch_result &r = res[c];
            std::memset(&r, 0, sizeof(r));
            r.status = s.status == 2 ? IFC_DIVERGED : (s.converged ? IFC_OK : IFC_NOT_CONVERGED);
            r.outer_iterations = s.it;
            r.converged = s.converged;
            for (int e = 0; e < 4; ++e) r.sweeps[e] = s.sweeps[e];
            r.rel_p = s.rel[0];
            r.rel_u = s.rel[1];
            r.rel_v = s.rel[2];
            r.rel_uf = s.rel[4];
            r.rel_vf = s.rel[5];
            r.norm_mass = s.norm[7];
            const BVariant &bv = kVariants[variant[c]];
            r.tile_x = bv.tx;
            r.tile_y = bv.ty;
            r.sweeps_per_pass = bv.ks;
            if (fields_out && fields_out[c]) {
                const size_t cells = (size_t)cfgs[c].nx * cfgs[c].ny;
                T *out = (T *)fields_out[c];
                BCK(cudaMemcpy(out, pool.u + queued[k].off_c, cells * sizeof(T), cudaMemcpyDeviceToHost));
                BCK(cudaMemcpy(out + cells, pool.v + queued[k].off_c, cells * sizeof(T), cudaMemcpyDeviceToHost));
                BCK(cudaMemcpy(out + 2 * cells, pool.p + queued[k].off_c, cells * sizeof(T), cudaMemcpyDeviceToHost));
            }
        }
    }
done:
    for (cudaGraphExec_t x : execs)
        if (x) cudaGraphExecDestroy(x);
    for (cudaGraph_t gph : graphs)
        if (gph) cudaGraphDestroy(gph);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (st) cudaStreamDestroy(st);
    T *all[] = {pool.u, pool.v, pool.p, pool.pc, pool.ac, pool.rac, pool.sp, pool.uf, pool.vf,
                pool.le, pool.ln, pool.lc, tp.tu, tp.tv, tp.tpc, pool.sdu, pool.sdv};
    for (T *a : all)
        if (a) cudaFree(a);
    if (dcases) cudaFree(dcases);
    if (dstates) cudaFree(dstates);
    if (dq) cudaFree(dq);
    return rc;
}

}  // namespace
}  // namespace ifc

extern "C" int ifc_batch_solve(const ifc_config *cases, int n, ifc_batch_result *results, void *const *fields_out,
                               double *device_ms)
{
    nvtxRangePushA("ifc_batch_solve");
    struct Pop {
        ~Pop() { nvtxRangePop(); }
    } pop;
    if (!cases || n <= 0 || !results) return IFC_BAD_ARGUMENT;
    const int prec = cases[0].precision;
    for (int c = 0; c < n; ++c) {
        const int rc = ifc_config_check(&cases[c]);
        if (rc != IFC_OK) return rc;
        if (cases[c].dim != 2 || cases[c].linear_solver != IFC_GAUSS_SEIDEL || cases[c].precision != prec ||
            cases[c].criterion == IFC_CRIT_RESIDUAL || cases[c].slab_axis_cells != 0)
            return IFC_UNSUPPORTED;
    }
    try {
        return prec == IFC_FP64 ? ifc::batch_solve<double>(cases, n, results, fields_out, device_ms)
                                : ifc::batch_solve<float>(cases, n, results, fields_out, device_ms);
    } catch (...) {
        return IFC_CUDA_ERROR;
    }
}
