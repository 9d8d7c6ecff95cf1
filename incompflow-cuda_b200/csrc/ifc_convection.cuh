// ifc_convection.cuh -- higher-order convection by deferred correction.
//
// The reference discretises convection with first-order upwind only
// (include/kernels.cuh:97-134) and lists higher-order schemes as planned
// (README.md:412).  Here the links stay upwind and the difference between a
// higher-order face value and the upwind one, times the face's mass flux, is
// lagged into the source (deferred correction, Khosla & Rubin 1974), evaluated
// with the fields at the start of the outer iteration:
//
//   b_C += sum over faces f of -F_f,out (phi_f - phi_U,f).
//
// With phi_U the upwind cell of a face, phi_D the downwind one and phi_UU the
// cell beyond phi_U, dd = phi_D - phi_U and du = phi_U - phi_UU, the face value
// is phi_f = phi_U + 0.5 L(du, dd):
//   central                 L = dd
//   second-order upwind     L = du
//   QUICK (Leonard 1979)    L = (3 dd + du) / 4
//   minmod (Roe 1986)       L = du or dd, the smaller in magnitude, if du dd > 0, else 0
//   van Leer (1974)         L = 2 du dd / (du + dd) if du dd > 0, else 0
// Boundary faces, and faces whose far-upwind cell lies outside the domain, keep
// the upwind value.  A face contributes Q = (rho u_f A) (0.5 L); a cell's
// correction is (Q_w - Q_e) + (Q_s - Q_n) [+ (Q_b - Q_t)], and it is added to
// the cell's source after the boundary fold-in.  Every operation is rounded in
// T in the order written (the library builds without FMA contraction).
#pragma once

#include "ifc_physics.cuh"

namespace ifc {

enum { CONV_UPWIND = 0, CONV_CENTRAL = 1, CONV_SOU = 2, CONV_QUICK = 3, CONV_MINMOD = 4, CONV_VAN_LEER = 5 };

template <typename T>
__host__ __device__ __forceinline__ T dc_limit(int scheme, T du, T dd)
{
    switch (scheme) {
    case CONV_CENTRAL: return dd;
    case CONV_SOU: return du;
    case CONV_QUICK: return ((T)3 * dd + du) / (T)4;
    case CONV_MINMOD:
        if (!(du * dd > (T)0)) return (T)0;
        return (du < (T)0 ? -du : du) < (dd < (T)0 ? -dd : dd) ? du : dd;
    case CONV_VAN_LEER:
        if (!(du * dd > (T)0)) return (T)0;
        return (T)2 * du * dd / (du + dd);
    default: return (T)0;
    }
}

// Q of one interior face between cells L and R along one axis; ll / rr are
// the cells beyond L and R (has_ll / has_rr: inside the domain).
template <typename T>
__host__ __device__ __forceinline__ T dc_face(int scheme, T rho, T uf, T A, T pll, T pl, T pr, T prr, bool has_ll,
                                              bool has_rr)
{
    const T F = rho * uf * A;
    T U, D, UU;
    if (F > (T)0) {
        if (!has_ll) return (T)0;
        U = pl;
        D = pr;
        UU = pll;
    } else if (F < (T)0) {
        if (!has_rr) return (T)0;
        U = pr;
        D = pl;
        UU = prr;
    } else {
        return (T)0;
    }
    return F * ((T)0.5 * dc_limit<T>(scheme, U - UU, D - U));
}

// Correction of cell c = (i, j, k) for the field phi (global, cell layout),
// given the velocities of the cell's six faces (west, east, south, north,
// bottom, top).
template <typename T, int DIM>
__device__ __forceinline__ T dc_cell(const Geo<T> &g, const T *phi, int c, int i, int j, int k, T uw, T ue, T vs,
                                     T vn, T wb, T wt)
{
    const int sc = g.conv, nx = g.nx, ny = g.ny, nz = g.nz;
    const int sx = 1, sy = nx, sz = nx * ny;
    const T rho = g.rho;
    T qw = (T)0, qe = (T)0, qs = (T)0, qn = (T)0;
    if (i > 0)
        qw = dc_face<T>(sc, rho, uw, g.Ax, i > 1 ? phi[c - 2 * sx] : (T)0, phi[c - sx], phi[c],
                        i < nx - 1 ? phi[c + sx] : (T)0, i > 1, i < nx - 1);
    if (i < nx - 1)
        qe = dc_face<T>(sc, rho, ue, g.Ax, i > 0 ? phi[c - sx] : (T)0, phi[c], phi[c + sx],
                        i < nx - 2 ? phi[c + 2 * sx] : (T)0, i > 0, i < nx - 2);
    if (j > 0)
        qs = dc_face<T>(sc, rho, vs, g.Ay, j > 1 ? phi[c - 2 * sy] : (T)0, phi[c - sy], phi[c],
                        j < ny - 1 ? phi[c + sy] : (T)0, j > 1, j < ny - 1);
    if (j < ny - 1)
        qn = dc_face<T>(sc, rho, vn, g.Ay, j > 0 ? phi[c - sy] : (T)0, phi[c], phi[c + sy],
                        j < ny - 2 ? phi[c + 2 * sy] : (T)0, j > 0, j < ny - 2);
    T dc = (qw - qe) + (qs - qn);
    if (DIM == 3) {
        T qb = (T)0, qt = (T)0;
        if (k > 0)
            qb = dc_face<T>(sc, rho, wb, g.Az, k > 1 ? phi[c - 2 * sz] : (T)0, phi[c - sz], phi[c],
                            k < nz - 1 ? phi[c + sz] : (T)0, k > 1, k < nz - 1);
        if (k < nz - 1)
            qt = dc_face<T>(sc, rho, wt, g.Az, k > 0 ? phi[c - sz] : (T)0, phi[c], phi[c + sz],
                            k < nz - 2 ? phi[c + 2 * sz] : (T)0, k > 0, k < nz - 2);
        dc = dc + (qb - qt);
    }
    return dc;
}

// The same with the face velocities read from f.
template <typename T, int DIM>
__device__ __forceinline__ T dc_cell(const Params<T> &P, const Fields<T> &f, const T *phi, int i, int j, int k)
{
    const Geo<T> &g = P.g;
    const int nx = g.nx, ny = g.ny;
    const int c = i + nx * (j + ny * k);
    const int fu = i + (nx + 1) * (j + ny * k), fv = i + nx * (j + (ny + 1) * k);
    const T wb = DIM == 3 ? f.wf[c] : (T)0, wt = DIM == 3 ? f.wf[c + nx * ny] : (T)0;
    return dc_cell<T, DIM>(g, phi, c, i, j, k, f.uf[fu], f.uf[fu + 1], f.vf[fv], f.vf[fv + nx], wb, wt);
}

// f.sdc[q*N + id] = correction of momentum component q (u, v, w) at cell id,
// from the current u, v, w and face velocities; row-segment work units (the
// six face velocities are read once for the three components).
template <typename T, int DIM>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 3) k_dc_source(Params<T> P, Fields<T> f)
{
    const Geo<T> &g = P.g;
    const int N = g.N, nx = g.nx, ny = g.ny, nz = g.nz, pl = nx * ny;
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int units = row_units(nx, ny * nz);
    for (int u = gw; u < units; u += nw) {
        const RowUnit w = row_unit(u, nx, ny);
        const int c0 = nx * w.r, f0 = (nx + 1) * w.r, v0 = nx * (w.j + (ny + 1) * w.k);
        for (int i = w.i0 + lane; i < w.i1; i += 32) {
            const int c = c0 + i;
            const T uw = f.uf[f0 + i], ue = f.uf[f0 + i + 1], vs = f.vf[v0 + i], vn = f.vf[v0 + i + nx];
            const T wb = DIM == 3 ? f.wf[c] : (T)0, wt = DIM == 3 ? f.wf[c + pl] : (T)0;
            const T du = dc_cell<T, DIM>(g, f.u, c, i, w.j, w.k, uw, ue, vs, vn, wb, wt);
            const T dv = dc_cell<T, DIM>(g, f.v, c, i, w.j, w.k, uw, ue, vs, vn, wb, wt);
            T dw = (T)0;
            if (DIM == 3) dw = dc_cell<T, DIM>(g, f.w, c, i, w.j, w.k, uw, ue, vs, vn, wb, wt);
            f.sdc[c] = du;
            f.sdc[(size_t)N + c] = dv;
            if (DIM == 3) f.sdc[2 * (size_t)N + c] = dw;
        }
    }
    (void)nz;
}

}  // namespace ifc
