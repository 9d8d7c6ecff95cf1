// ifc_fused3d.cuh -- 3D red-black half sweeps with on-the-fly coefficients.
//
// The reference streams 7 coefficient planes per cell and sweep
// (include/kernels.cuh:926-1005 reading the planes written by :97-334 and
// :502-540).  Here the momentum solve's first sweep builds the coefficients,
// the pressure source and the boundary fold-in of each cell from its six face
// velocities and seven pressures (mom_cell) and packs them in sweep order for
// the later sweeps, and every half sweep updates u, v and w together (they
// share the coefficients); the p' half sweep builds its six links from
// the reciprocals 1/aC of the cell and its neighbours (kernels.cuh:518-537),
// stored once per outer iteration.  Same arithmetic as ifc_physics.cuh, so
// the results are bit-identical to the per-step kernels and the CPU oracle.
#pragma once

#include "ifc_kernels.cuh"
#include "ifc_persist2d.cuh"

namespace ifc {

// Four consecutive values from a 16-byte aligned address, bypassing L1 (each
// packed value is read once per half sweep).
__device__ __forceinline__ void ld4(const float *p, float (&o)[4])
{
    const float4 v = __ldcg(reinterpret_cast<const float4 *>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}
__device__ __forceinline__ void ld4(const double *p, double (&o)[4])
{
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}
template <typename T>
__device__ __forceinline__ void st4(T *p, T a, T b, T c, T d)
{
    p[0] = a;
    p[1] = b;
    p[2] = c;
    p[3] = d;
}

// Two consecutive values from an aligned address, bypassing L1.
__device__ __forceinline__ void ld2(const float *p, float (&o)[2])
{
    const float2 v = __ldcg(reinterpret_cast<const float2 *>(p));
    o[0] = v.x;
    o[1] = v.y;
}
__device__ __forceinline__ void ld2(const double *p, double (&o)[2])
{
    const double2 v = __ldcg(reinterpret_cast<const double2 *>(p));
    o[0] = v.x;
    o[1] = v.y;
}

struct Half3D {
    int color;      // 0 red, 1 black (completes the sweep)
    int active[3];  // component takes part in this sweep (s < n_iter)
    int first;      // first sweep of the solve: store aC
};

// Bound to 48 registers in FP32 (5 blocks of 256 per SM; at 40 registers and
// 6 blocks the packed form spills): the half sweep is bound by the latency
// of its cached loads.
//
// The coefficients and sources do not change within the momentum solve, so
// the first sweep's two launches (FIRST) build them from the faces and
// pressures of each cell (mom_cell) and store them packed, per (row, colour)
// the cells of that colour in order -- slot (2 r + colour) hx + (i >> 1),
// r = j + ny k, hx = (nx + 1) / 2 -- as {aC, aE, aW, aN}, {aS, aT, aB, b_u}
// and {b_v, b_w} in three arrays of `slots` entries; the later sweeps read
// them back with two 4-wide and one 2-wide load instead of the thirteen
// loads and the arithmetic of mom_cell (128^3 cavity, FP32: momentum solve
// 0.286 -> 0.265 ms; FP64 with QUICK 0.706 -> 0.640 ms; same bits).
template <typename T, bool FIRST>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 5 : 3) k_mom_half3d(Params<T> P, Fields<T> f, Ctl *ctl, double *partials, Half3D h,
                                                                          T *pk, long long slots)
{
    const Geo<T> &g = P.g;
    bool act[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) act[c] = h.active[c] && !ctl->stop[c];
    if (!act[0] && !act[1] && !act[2] && !FIRST) return;  // uniform
    const int nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny, N = g.N;
    const int nrows = ny * nz, lane = threadIdx.x & 31, hx = (nx + 1) / 2;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nwg = (int)((gridDim.x * blockDim.x) >> 5);
    T *phi[3] = {f.u, f.v, f.w};
    double sq[3] = {0.0, 0.0, 0.0};
    // one warp per x-row, lanes over the row's cells of this colour
    for (int r = gw; r < nrows; r += nwg) {
        const int j = r % ny, k = r / ny;
        const long long sb = (long long)(2 * r + h.color) * hx;
        for (int i = ((h.color + j + k) & 1) + 2 * lane; i < nx; i += 64) {
            const int c = i + nx * (j + ny * k);
            const long long slot = sb + (i >> 1);
            T a[7], b[3];
            if (FIRST) {
                const int fu = i + (nx + 1) * (j + ny * k), fv = i + nx * (j + (ny + 1) * k);
                mom_cell<T, 3>(P, i, j, k, f.uf[fu], f.uf[fu + 1], f.vf[fv], f.vf[fv + nx], f.wf[c], f.wf[c + pl],
                               f.p[c], i > 0 ? f.p[c - 1] : (T)0, i < nx - 1 ? f.p[c + 1] : (T)0,
                               j > 0 ? f.p[c - nx] : (T)0, j < ny - 1 ? f.p[c + nx] : (T)0,
                               k > 0 ? f.p[c - pl] : (T)0, k < nz - 1 ? f.p[c + pl] : (T)0, a, b);
                add_dc<T, 3>(P, f, c, b);
                f.ac[c] = a[AC];
                st4(pk + 4 * slot, a[AC], a[AE], a[AW], a[AN]);
                st4(pk + 4 * (slots + slot), a[AS], a[AT], a[AB], b[0]);
                pk[8 * slots + 2 * slot] = b[1];
                pk[8 * slots + 2 * slot + 1] = b[2];
            } else {
                T q0[4], q1[4], q2[2];
                ld4(pk + 4 * slot, q0);
                ld4(pk + 4 * (slots + slot), q1);
                ld2(pk + 8 * slots + 2 * slot, q2);
                a[AC] = q0[0];
                a[AE] = q0[1];
                a[AW] = q0[2];
                a[AN] = q0[3];
                a[AS] = q1[0];
                a[AT] = q1[1];
                a[AB] = q1[2];
                b[0] = q1[3];
                b[1] = q2[0];
                b[2] = q2[1];
            }
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

// Row blocks of the cooperative 3D solves (ifc_coop3d.cuh): each CTA owns
// the x-rows j in [j0, j0+bj), k in [k0, k0+bk).
struct PcBlocks {
    int bj, bk;    // rows per block along j and k
    int nbj, nbk;  // blocks along j and k
};

}  // namespace ifc
