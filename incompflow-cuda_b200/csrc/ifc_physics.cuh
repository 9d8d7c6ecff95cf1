// ifc_physics.cuh -- per-cell and per-face arithmetic of the SIMPLE method.
//
// Each function restates one piece of the reference's kernels
// (WanZijun271/IncompFlow-CUDA include/kernels.cuh) operation by operation:
// the library is compiled with --fmad=false and IEEE division, so a value
// computed here is bit-identical to the same value computed by the CPU oracle.
// Where the reference multiplies a float by a double literal (0.5, -0.5) the
// expression is evaluated in FP64 and rounded on store, as the reference's
// float build does.  Every kernel (the simple per-step kernels, the fused
// temporally blocked sweeps and the batched solver) calls these functions, so
// all of them share one definition of the method.
#pragma once

#include "ifc_common.cuh"

namespace ifc {

template <typename T>
__host__ __device__ __forceinline__ T min0(T x) { return x < (T)0 ? x : (T)0; }

// Host-side precomputed constants that the reference evaluates as constexpr or
// as the leading part of a left-to-right product.
template <typename T>
struct Derived {
    T Dx, Dy, Dz;           // mu*A/d per direction (kernels.cuh:116-130)
    double Kx, Ky, Kz;      // ((-0.5*rho)*A)*A (kernels.cuh:518-535)
    double ru[3];           // relax*0.5 for u, v, w (kernels.cuh:630,793)
    T c83;                  // (scalar)8/3 (kernels.cuh:307)
};

template <typename T>
struct Params {
    Geo<T> g;
    Derived<T> d;
};

// Face velocity at a boundary face, kernels.cuh:87-93: wall 0, inlet the
// prescribed normal component, outlet the adjacent cell's velocity.
template <typename T>
__device__ __forceinline__ T face_bc(const Geo<T> &g, int face, int comp, T adjacent, int inlet_index)
{
    const int t = g.bc[face];
    if (t == WALL) return (T)0;
    if (t == INLET) return (face == WEST && g.inlet) ? g.inlet[inlet_index] : g.bcv[face][comp];
    return adjacent;
}

// Boundary fold-in of one face for one cell, kernels.cuh:304-331.
template <typename T, int DIM>
__device__ __forceinline__ void fold_face(const Params<T> &P, int face, int ex, int in, T ubc, T vbc, T wbc,
                                          T (&a)[7], T (&b)[3])
{
    const T e = a[ex];
    if (P.g.bc[face] == OUTLET) {
        a[AC] = a[AC] + e;
        a[ex] = (T)0;
        return;
    }
    a[AC] = a[AC] - (T)2 * e;
    a[in] = a[in] + e / (T)3;
    b[0] = b[0] - P.d.c83 * e * ubc;
    b[1] = b[1] - P.d.c83 * e * vbc;
    if (DIM == 3) b[2] = b[2] - P.d.c83 * e * wbc;
    a[ex] = (T)0;
}

// Momentum link coefficients, source and boundary fold-in of cell (i,j,k):
// kernels.cuh:97-134 (coefficients), :136-250 (pressure source), :252-334
// (fold-in, faces in the launch order E W N S T B of src/Solver.cu:583-608).
// One coefficient set serves u, v and w; b[c] is the source of component c.
// uf/vf/wf/p may point to global or shared memory; the caller passes the
// face-array index of the cell's low face and the strides.
template <typename T, int DIM>
__device__ __forceinline__ void mom_cell(const Params<T> &P, int i, int j, int k,
                                         T uw, T ue, T vs, T vn, T wb, T wt,
                                         T pC, T pW, T pE, T pS, T pN, T pB, T pT,
                                         T (&a)[7], T (&b)[3])
{
    const Geo<T> &g = P.g;
    a[AE] = g.rho * min0(ue) * g.Ax - P.d.Dx;
    a[AW] = g.rho * min0(-uw) * g.Ax - P.d.Dx;
    a[AN] = g.rho * min0(vn) * g.Ay - P.d.Dy;
    a[AS] = g.rho * min0(-vs) * g.Ay - P.d.Dy;
    a[AC] = -(a[AE] + a[AW] + a[AN] + a[AS]);
    a[AT] = (T)0;
    a[AB] = (T)0;
    if (DIM == 3) {
        a[AT] = g.rho * min0(wt) * g.Az - P.d.Dz;
        a[AB] = g.rho * min0(-wb) * g.Az - P.d.Dz;
        a[AC] += -(a[AT] + a[AB]);
    }
    // Pressure at the faces: neighbour inside, cell value at wall/inlet, 0 at outlet.
    T pl = i > 0 ? pW : (g.closed[WEST] ? pC : (T)0);
    T pr = i < g.nx - 1 ? pE : (g.closed[EAST] ? pC : (T)0);
    b[0] = (T)(0.5 * (double)(T)(pl - pr) * (double)g.Ax);
    pl = j > 0 ? pS : (g.closed[SOUTH] ? pC : (T)0);
    pr = j < g.ny - 1 ? pN : (g.closed[NORTH] ? pC : (T)0);
    b[1] = (T)(0.5 * (double)(T)(pl - pr) * (double)g.Ay);
    b[2] = (T)0;
    if (DIM == 3) {
        pl = k > 0 ? pB : (g.closed[BOTTOM] ? pC : (T)0);
        pr = k < g.nz - 1 ? pT : (g.closed[TOP] ? pC : (T)0);
        b[2] = (T)(0.5 * (double)(T)(pl - pr) * (double)g.Az);
    }
    if (i == g.nx - 1) fold_face<T, DIM>(P, EAST, AE, AW, g.bcv[EAST][0], g.bcv[EAST][1], g.bcv[EAST][2], a, b);
    if (i == 0) {
        const T uin = (g.inlet && g.bc[WEST] == INLET) ? g.inlet[j + g.ny * k] : g.bcv[WEST][0];
        fold_face<T, DIM>(P, WEST, AW, AE, uin, g.bcv[WEST][1], g.bcv[WEST][2], a, b);
    }
    if (j == g.ny - 1) fold_face<T, DIM>(P, NORTH, AN, AS, g.bcv[NORTH][0], g.bcv[NORTH][1], g.bcv[NORTH][2], a, b);
    if (j == 0) fold_face<T, DIM>(P, SOUTH, AS, AN, g.bcv[SOUTH][0], g.bcv[SOUTH][1], g.bcv[SOUTH][2], a, b);
    if (DIM == 3) {
        if (k == g.nz - 1) fold_face<T, DIM>(P, TOP, AT, AB, g.bcv[TOP][0], g.bcv[TOP][1], g.bcv[TOP][2], a, b);
        if (k == 0) fold_face<T, DIM>(P, BOTTOM, AB, AT, g.bcv[BOTTOM][0], g.bcv[BOTTOM][1], g.bcv[BOTTOM][2], a, b);
    }
}

// Adds the deferred-correction sources of cell c (higher-order convection,
// ifc_convection.cuh) to the momentum sources b after the boundary fold-in.
template <typename T, int DIM>
__device__ __forceinline__ void add_dc(const Params<T> &P, const Fields<T> &f, int c, T (&b)[3])
{
    if (P.g.conv == 0) return;
    const int N = P.g.N;
    b[0] = b[0] + f.sdc[c];
    b[1] = b[1] + f.sdc[N + c];
    if (DIM == 3) b[2] = b[2] + f.sdc[2 * N + c];
}

// One relaxed point update, kernels.cuh:976-988: out-of-domain neighbours
// enter as 0 (their links are 0 after the fold-in anyway).
template <typename T, int DIM>
__device__ __forceinline__ T point_update(const T (&a)[7], T src, T pc, T pE, T pW, T pN, T pS, T pT, T pB,
                                          T relax, T &d)
{
    T np = src - a[AE] * pE - a[AW] * pW - a[AN] * pN - a[AS] * pS;
    if (DIM == 3) np -= a[AT] * pT + a[AB] * pB;
    np /= a[AC];
    d = relax * (np - pc);
    return pc + d;
}

// Rhie-Chow face velocity, kernels.cuh:394-395 and :497-498.
template <typename T>
__device__ __forceinline__ T rc_face(T uL, T uR, T aCL, T aCR, T pLL, T pL, T pR, T pRR, T A)
{
    double t0 = 0.5 * (double)(T)(uL + uR);
    T t1 = (pR - pLL) * A / ((T)4 * aCL);
    T t2 = (pRR - pL) * A / ((T)4 * aCR);
    T sr = (T)1 / aCL + (T)1 / aCR;
    double t3 = 0.5 * (double)sr * (double)(T)(pL - pR) * (double)A;
    return (T)(t0 + (double)t1 + (double)t2 + t3);
}

// p' link across one interior face, kernels.cuh:518-535.
template <typename T>
__device__ __forceinline__ T pcorr_link(double K, T aCC, T aCN)
{
    return (T)(K * (double)(T)((T)1 / aCC + (T)1 / aCN));
}

// p' source (mass imbalance) of one cell, kernels.cuh:558-563.
template <typename T, int DIM>
__device__ __forceinline__ T mass_imbalance(const Geo<T> &g, T uw, T ue, T vs, T vn, T wb, T wt)
{
    T b = g.rho * (g.Ax * (uw - ue) + g.Ay * (vs - vn));
    if (DIM == 3) b += g.rho * g.Az * (wb - wt);
    return b;
}

// Cell velocity correction, kernels.cuh:630 and :729.
template <typename T>
__device__ __forceinline__ T vel_corr(double ru, T pcl, T pcr, T A, T aC)
{
    return (T)(ru * (double)(T)(pcl - pcr) * (double)A / (double)aC);
}

// Face velocity correction, kernels.cuh:793.
template <typename T>
__device__ __forceinline__ T face_corr(double ru, T aCL, T aCR, T pcl, T pcr, T A)
{
    T sr = (T)1 / aCL + (T)1 / aCR;
    return (T)(ru * (double)sr * (double)(T)(pcl - pcr) * (double)A);
}

}  // namespace ifc
