// ifc_adjoint2d.cuh -- discrete adjoint of the 2D SIMPLE fixed point (FP64).
//
// One SIMPLE outer iteration maps the persistent state x = (u, v, p, interior
// uf, interior vf) to G(x, theta, mu); at convergence x = G(x).  For an
// objective J(x) the adjoint lambda solves lambda = G_x^T lambda + dJ/dx, and
// dJ/dtheta = G_theta^T lambda, dJ/dmu = G_mu^T lambda (theta: the west-inlet
// velocity of each boundary row).  One reverse pass applies G_x^T by running
// the steps of an outer iteration backwards; at the fixed point every momentum
// Gauss-Seidel iterate equals the converged field and p' is 0 throughout, so
// nothing from the forward iterations has to be stored:
//   corrections^T -> [p' mean removal]^T -> transposed p' sweeps -> p' source^T
//   -> Rhie-Chow^T and face BCs^T -> transposed momentum sweeps (u and v share
//   the coefficients; their adjoint and the sources' are accumulated) ->
//   boundary fold-in^T -> pressure source^T -> link coefficients^T (upwind
//   derivative [u_f < 0]) -> face BCs^T.
// Every kernel is written in gather form (each thread owns the outputs it
// writes), so the results are deterministic; the transposed half sweeps
// ping-pong between two buffers.  All adjoint arithmetic is FP64.  The
// forward steps transposed here are kernels.cuh:87-134 (face BCs, links),
// :136-334 (sources, fold-in), :394-498 (Rhie-Chow), :517-563 (p' links and
// source), :583-843 (corrections) and :926-1005 (sweeps) of the reference.
#pragma once

#include "ifc_kernels.cuh"

namespace ifc {

struct AdjBufs {
    // linearisation point (FP64 copies) and coefficients
    double *u, *v, *p, *uf, *vf;
    double *araw, *afold, *ap;  // 5 planes each: raw links, folded links, p' links
    // adjoint state: current iterate and the operator's output
    double *lu, *lv, *lp, *luf, *lvf;
    double *ou, *ov, *op, *ouf, *ovf;
    // objective gradient dJ/dx (cells)
    double *ju, *jv, *jp;
    // work
    double *lpc[2], *lus[2], *lvs[2];
    double *lbp, *lbu, *lbv, *la, *lufs, *lvfs, *lufa, *lvfa;
    double *ltheta;  // ny
    double *scal;    // [0] dJ/dmu, [1] max |delta lambda|, [2] max |lambda|, [3] iterations,
                     // [4] converged, [5] J, [6] tolerance, [7] iteration limit
};

struct AdjArgs {
    double alpha_u, alpha_v, alpha_p, ru, rv;  // relaxations, relax*0.5
};

#define ADJ_LOOP(q, n) for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < (n); q += gridDim.x * blockDim.x)

// ---- set-up: FP64 copies of the state and the coefficients --------------
template <typename T>
__global__ void k_adj_prep(Params<double> P, Fields<T> f, AdjBufs b)
{
    const int nx = P.g.nx, ny = P.g.ny, N = P.g.N;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    ADJ_LOOP(q, N)
    {
        b.u[q] = (double)f.u[q];
        b.v[q] = (double)f.v[q];
        b.p[q] = (double)f.p[q];
    }
    ADJ_LOOP(q, NU) b.uf[q] = (double)f.uf[q];
    ADJ_LOOP(q, NV) b.vf[q] = (double)f.vf[q];
}

template <typename T>
__global__ void k_adj_inlet(const T *in, double *out, int n)
{
    ADJ_LOOP(q, n) out[q] = (double)in[q];
}

// Boundary faces from the current velocities (the first step of an
// iteration, kernels.cuh:87-93).
__global__ void k_adj_bcfaces(Params<double> P, AdjBufs b)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny;
    ADJ_LOOP(q, ny + nx)
    {
        if (q < ny) {
            const int j = q;
            b.uf[(nx + 1) * j] = face_bc(g, WEST, 0, b.u[nx * j], j);
            b.uf[nx + (nx + 1) * j] = face_bc(g, EAST, 0, b.u[nx - 1 + nx * j], j);
        } else {
            const int i = q - ny;
            b.vf[i] = face_bc(g, SOUTH, 1, b.v[i], 0);
            b.vf[i + nx * ny] = face_bc(g, NORTH, 1, b.v[i + nx * (ny - 1)], 0);
        }
    }
}

// Raw and folded momentum links (kernels.cuh:97-134, 252-334).
__global__ void k_adj_coef(Params<double> P, AdjBufs b)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        const int fu = i + (nx + 1) * j;
        const double ue = b.uf[fu + 1], uw = b.uf[fu], vn = b.vf[c + nx], vs = b.vf[c];
        double r[5];
        r[AE] = g.rho * min0(ue) * g.Ax - P.d.Dx;
        r[AW] = g.rho * min0(-uw) * g.Ax - P.d.Dx;
        r[AN] = g.rho * min0(vn) * g.Ay - P.d.Dy;
        r[AS] = g.rho * min0(-vs) * g.Ay - P.d.Dy;
        r[AC] = -(r[AE] + r[AW] + r[AN] + r[AS]);
        double a[7], s[3];
        mom_cell<double, 2>(P, i, j, 0, uw, ue, vs, vn, 0.0, 0.0, b.p[c], i > 0 ? b.p[c - 1] : 0.0,
                            i < nx - 1 ? b.p[c + 1] : 0.0, j > 0 ? b.p[c - nx] : 0.0, j < ny - 1 ? b.p[c + nx] : 0.0,
                            0.0, 0.0, a, s);
        for (int k = 0; k < 5; ++k) {
            b.araw[c + (size_t)N * k] = r[k];
            b.afold[c + (size_t)N * k] = a[k];
        }
    }
}

// p' links from the folded diagonal (kernels.cuh:517-529).
__global__ void k_adj_pcoef(Params<double> P, AdjBufs b)
{
    const int nx = P.g.nx, ny = P.g.ny, N = P.g.N;
    const double *aC = b.afold;
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        const double e = i < nx - 1 ? pcorr_link<double>(P.d.Kx, aC[c], aC[c + 1]) : 0.0;
        const double w = i > 0 ? pcorr_link<double>(P.d.Kx, aC[c], aC[c - 1]) : 0.0;
        const double n = j < ny - 1 ? pcorr_link<double>(P.d.Ky, aC[c], aC[c + nx]) : 0.0;
        const double s = j > 0 ? pcorr_link<double>(P.d.Ky, aC[c], aC[c - nx]) : 0.0;
        b.ap[c + (size_t)N * AE] = e;
        b.ap[c + (size_t)N * AW] = w;
        b.ap[c + (size_t)N * AN] = n;
        b.ap[c + (size_t)N * AS] = s;
        b.ap[c] = -(e + w + n + s);
    }
}

// Objective J = mean p over the first cell column - mean over the last (the
// area-weighted inlet-minus-outlet pressure drop on a uniform grid) and its
// gradient as the seed; the adjoint starts from lambda = dJ/dx.
__global__ void k_adj_seed(Params<double> P, AdjBufs b, int builtin)
{
    const int nx = P.g.nx, ny = P.g.ny, N = P.g.N;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    ADJ_LOOP(c, N)
    {
        if (builtin) {
            const int i = c % nx;
            b.ju[c] = 0.0;
            b.jv[c] = 0.0;
            b.jp[c] = (i == 0 ? 1.0 / ny : 0.0) - (i == nx - 1 ? 1.0 / ny : 0.0);
        }
        b.lu[c] = b.ju[c];
        b.lv[c] = b.jv[c];
        b.lp[c] = b.jp[c];
    }
    ADJ_LOOP(q, NU) b.luf[q] = 0.0;
    ADJ_LOOP(q, NV) b.lvf[q] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.scal[3] = 0.0;
        b.scal[4] = 0.0;
    }
}

// J in FP64, one block, fixed summation order.
__global__ void k_adj_objective(Params<double> P, AdjBufs b)
{
    const int nx = P.g.nx, ny = P.g.ny;
    __shared__ double sh[32];
    double x = 0.0;
    for (int j = threadIdx.x; j < ny; j += blockDim.x) x += b.p[nx * j] - b.p[nx - 1 + nx * j];
    x = warp_sum(x);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) sh[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += sh[w];
        b.scal[5] = t / ny;
    }
}

// ---- corrections^T (kernels.cuh:583-843), gather form --------------------
// Forward: p += alpha_p p'; u_c += ru Ax/aC_c (p'_L(c) - p'_R(c)); interior
// faces uf += ru (1/aC_L + 1/aC_R) Ax (p'_L - p'_R); the neighbour L(c) / R(c)
// is the cell itself at a wall or inlet face and absent at an outlet.
__global__ void k_adj_corr(Params<double> P, AdjBufs b, AdjArgs A)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const double *aC = b.afold;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        double x = A.alpha_p * b.lp[c];
        if (i < nx - 1) x += A.ru * g.Ax / aC[c + 1] * b.lu[c + 1];
        if (i == 0 && g.closed[WEST]) x += A.ru * g.Ax / aC[c] * b.lu[c];
        if (i > 0) x -= A.ru * g.Ax / aC[c - 1] * b.lu[c - 1];
        if (i == nx - 1 && g.closed[EAST]) x -= A.ru * g.Ax / aC[c] * b.lu[c];
        if (j < ny - 1) x += A.rv * g.Ay / aC[c + nx] * b.lv[c + nx];
        if (j == 0 && g.closed[SOUTH]) x += A.rv * g.Ay / aC[c] * b.lv[c];
        if (j > 0) x -= A.rv * g.Ay / aC[c - nx] * b.lv[c - nx];
        if (j == ny - 1 && g.closed[NORTH]) x -= A.rv * g.Ay / aC[c] * b.lv[c];
        const int fu = i + (nx + 1) * j;
        if (i < nx - 1) x += A.ru * (1.0 / aC[c] + 1.0 / aC[c + 1]) * g.Ax * b.luf[fu + 1];
        if (i > 0) x -= A.ru * (1.0 / aC[c - 1] + 1.0 / aC[c]) * g.Ax * b.luf[fu];
        if (j < ny - 1) x += A.rv * (1.0 / aC[c] + 1.0 / aC[c + nx]) * g.Ay * b.lvf[c + nx];
        if (j > 0) x -= A.rv * (1.0 / aC[c - nx] + 1.0 / aC[c]) * g.Ay * b.lvf[c];
        b.lpc[0][c] = x;
        b.lus[0][c] = b.lu[c];
        b.lvs[0][c] = b.lv[c];
        b.op[c] = b.lp[c];
        b.lbp[c] = 0.0;
        b.lbu[c] = 0.0;
        b.lbv[c] = 0.0;
        for (int k = 0; k < 5; ++k) b.la[c + (size_t)N * k] = 0.0;
    }
    ADJ_LOOP(q, NU)
    {
        const int i = q % (nx + 1);
        b.lufs[q] = (i > 0 && i < nx) ? b.luf[q] : 0.0;
        b.lufa[q] = 0.0;
    }
    ADJ_LOOP(q, NV)
    {
        const int j = q / nx;
        b.lvfs[q] = (j > 0 && j < ny) ? b.lvf[q] : 0.0;
        b.lvfa[q] = 0.0;
    }
    ADJ_LOOP(q, ny) b.ltheta[q] = 0.0;
}

// p' mean removal^T: the adjoint loses its mean.
__global__ void k_adj_sum(const double *x, int N, Ctl *ctl, double *partials)
{
    double s[1] = {0.0};
    ADJ_LOOP(c, N) s[0] += x[c];
    __shared__ double tot[1];
    if (grid_reduce<1>(s, partials, ctl, tot) && threadIdx.x == 0) ctl->sq[SQ_PCSUM] = tot[0];
}

__global__ void k_adj_shift(double *x, int N, const Ctl *ctl)
{
    const double mean = ctl->sq[SQ_PCSUM] / (double)N;
    ADJ_LOOP(c, N) x[c] -= mean;
}

// One transposed red-black half sweep (colour h) of an equation with links a
// (5 planes, aC first) and relaxation alpha.  Forward, for X of colour h:
//   phi_X <- (1-alpha) phi_X + alpha (b_X - sum_nb a_X,nb phi_nb) / aC_X.
// Reverse: the colour-h cells accumulate the source adjoint alpha/aC_X l_X
// and keep (1 - alpha) of their adjoint; cells of the other colour gather
// -a_X,c alpha l_X / aC_X from their colour-h neighbours X.  With la set, the
// link adjoint of the colour-h cells is accumulated as well (phi = fixed point).
struct HalfT {
    const double *a;
    const double *in[2];
    double *out[2];
    double *lb[2];
    const double *phi[2];
    double alpha[2];
    int ncomp;
    int color;
    double *la;
};

__global__ void k_adj_half(Params<double> P, HalfT H)
{
    const int nx = P.g.nx, ny = P.g.ny, N = P.g.N;
    const double *a = H.a;
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        if (((i + j) & 1) == H.color) {
            const double aC = a[c];
            double dla[5] = {0, 0, 0, 0, 0};
            for (int m = 0; m < H.ncomp; ++m) {
                const double l = H.in[m][c];
                const double gm = H.alpha[m] / aC * l;
                H.lb[m][c] += gm;
                H.out[m][c] = (1.0 - H.alpha[m]) * l;
                if (H.la) {
                    const double *ph = H.phi[m];
                    if (i < nx - 1) dla[AE] += -ph[c + 1] * gm;
                    if (i > 0) dla[AW] += -ph[c - 1] * gm;
                    if (j < ny - 1) dla[AN] += -ph[c + nx] * gm;
                    if (j > 0) dla[AS] += -ph[c - nx] * gm;
                    dla[AC] += -ph[c] * gm;
                }
            }
            if (H.la)
                for (int k = 0; k < 5; ++k) H.la[c + (size_t)N * k] += dla[k];
        } else {
            for (int m = 0; m < H.ncomp; ++m) {
                const double *l = H.in[m];
                const double al = H.alpha[m];
                double x = l[c];
                if (i > 0) x += -a[c - 1 + (size_t)N * AE] * al * l[c - 1] / a[c - 1];
                if (i < nx - 1) x += -a[c + 1 + (size_t)N * AW] * al * l[c + 1] / a[c + 1];
                if (j > 0) x += -a[c - nx + (size_t)N * AN] * al * l[c - nx] / a[c - nx];
                if (j < ny - 1) x += -a[c + nx + (size_t)N * AS] * al * l[c + nx] / a[c + nx];
                H.out[m][c] = x;
            }
        }
    }
}

// ---- p' source^T on faces (kernels.cuh:558-563), inlet faces of u* -------
__global__ void k_adj_src_faces(Params<double> P, AdjBufs b)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    ADJ_LOOP(q, NU + NV)
    {
        if (q < NU) {
            const int i = q % (nx + 1), j = q / (nx + 1);
            double gsum = 0.0;
            if (i < nx) gsum += b.lbp[i + nx * j];
            if (i > 0) gsum -= b.lbp[i - 1 + nx * j];
            const double val = b.lufs[q] + g.rho * g.Ax * gsum;
            b.lufs[q] = val;
            if (i == 0 && g.bc[WEST] == INLET) b.ltheta[j] += val;
        } else {
            const int qq = q - NU, j = qq / nx, i = qq % nx;
            double gsum = 0.0;
            if (j < ny) gsum += b.lbp[i + nx * j];
            if (j > 0) gsum -= b.lbp[i + nx * (j - 1)];
            b.lvfs[qq] += g.rho * g.Ay * gsum;
        }
    }
}

// ---- Rhie-Chow^T (kernels.cuh:394-395, 497-498) and outlet faces^T ------
// Forward on interior face k between cells L = k-1 and R = k of a line:
//   f = 0.5 (phi_L + phi_R) + (p_R - p_LL) A/(4 aC_L) + (p_RR - p_L) A/(4 aC_R)
//       + 0.5 (1/aC_L + 1/aC_R) (p_L - p_R) A,
// LL/RR being the cell itself at a closed end and absent (0) at an outlet.
// Each cell gathers the terms of the up to four faces of its line it enters.
__device__ __forceinline__ void rc_face_adj(const double *pl, const double *al, int k, int n, int stride, double A,
                                            int clo, int chi, double l, int pos, double &lp, double &lac)
{
    const int L = k - 1, R = k;
    const double aL = al[(size_t)stride * L], aR = al[(size_t)stride * R];
    const double cL = A / (4.0 * aL), cR = A / (4.0 * aR), h = 0.5 * (1.0 / aL + 1.0 / aR) * A;
    const int LL = k >= 2 ? L - 1 : (clo ? L : -1);
    const int RR = k <= n - 2 ? R + 1 : (chi ? R : -1);
    const double pL = pl[(size_t)stride * L], pR = pl[(size_t)stride * R];
    const double pLL = LL >= 0 ? pl[(size_t)stride * LL] : 0.0, pRR = RR >= 0 ? pl[(size_t)stride * RR] : 0.0;
    if (pos == R) lp += (cL - h) * l;
    if (pos == LL) lp += -cL * l;
    if (pos == RR) lp += cR * l;
    if (pos == L) lp += (-cR + h) * l;
    if (pos == L) lac += (-(pR - pLL) * A / (4.0 * aL * aL) - 0.5 * (pL - pR) * A / (aL * aL)) * l;
    if (pos == R) lac += (-(pRR - pL) * A / (4.0 * aR * aR) - 0.5 * (pL - pR) * A / (aR * aR)) * l;
}

__global__ void k_adj_rc(Params<double> P, AdjBufs b, int buf)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const double *aC = b.afold;
    double *lus = b.lus[buf], *lvs = b.lvs[buf];
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        double lp = 0.0, lac = 0.0, lu = lus[c], lv = lvs[c];
        const int fu = i + (nx + 1) * j;
        for (int k = i - 1; k <= i + 2; ++k) {
            if (k < 1 || k > nx - 1) continue;
            const double l = b.lufs[k + (nx + 1) * j];
            if (l == 0.0) continue;
            rc_face_adj(b.p + (size_t)nx * j, aC + (size_t)nx * j, k, nx, 1, g.Ax, g.closed[WEST], g.closed[EAST], l,
                        i, lp, lac);
        }
        if (i >= 1) lu += 0.5 * b.lufs[fu];
        if (i <= nx - 2) lu += 0.5 * b.lufs[fu + 1];
        if (i == 0 && g.bc[WEST] == OUTLET) lu += b.lufs[fu];
        if (i == nx - 1 && g.bc[EAST] == OUTLET) lu += b.lufs[fu + 1];
        for (int k = j - 1; k <= j + 2; ++k) {
            if (k < 1 || k > ny - 1) continue;
            const double l = b.lvfs[i + nx * k];
            if (l == 0.0) continue;
            rc_face_adj(b.p + i, aC + i, k, ny, nx, g.Ay, g.closed[SOUTH], g.closed[NORTH], l, j, lp, lac);
        }
        if (j >= 1) lv += 0.5 * b.lvfs[c];
        if (j <= ny - 2) lv += 0.5 * b.lvfs[c + nx];
        if (j == 0 && g.bc[SOUTH] == OUTLET) lv += b.lvfs[c];
        if (j == ny - 1 && g.bc[NORTH] == OUTLET) lv += b.lvfs[c + nx];
        lus[c] = lu;
        lvs[c] = lv;
        b.op[c] += lp;
        b.la[c] += lac;  // adjoint of the folded diagonal
    }
}

// ---- fold-in^T per boundary cell (kernels.cuh:304-331): faces in the
// reverse of the forward order E W N S; then the link totals
// t_nb = la_nb - la_C of the raw links (aC = -sum a_nb).
__global__ void k_adj_fold(Params<double> P, AdjBufs b)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const double c83 = 8.0 / 3.0;
    double *la = b.la;
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        const int faces[4] = {SOUTH, NORTH, WEST, EAST};
        for (int q = 0; q < 4; ++q) {
            const int F = faces[q];
            const bool on = (F == SOUTH && j == 0) || (F == NORTH && j == ny - 1) || (F == WEST && i == 0) ||
                            (F == EAST && i == nx - 1);
            if (!on) continue;
            const int ex = F == EAST ? AE : F == WEST ? AW : F == NORTH ? AN : AS;
            const int in = F == EAST ? AW : F == WEST ? AE : F == NORTH ? AS : AN;
            if (g.bc[F] == OUTLET) {
                la[c + (size_t)N * ex] = la[c];
                continue;
            }
            const double exv = b.araw[c + (size_t)N * ex];
            double ubc = g.bcv[F][0];
            const double vbc = g.bcv[F][1];
            const bool prof = F == WEST && g.bc[WEST] == INLET;
            if (prof && g.inlet) ubc = g.inlet[j];
            la[c + (size_t)N * ex] = -2.0 * la[c] + la[c + (size_t)N * in] / 3.0 - c83 * ubc * b.lbu[c] -
                                     c83 * vbc * b.lbv[c];
            if (prof) b.ltheta[j] += -c83 * exv * b.lbu[c];
        }
        const double tC = la[c];
        for (int k = 1; k < 5; ++k) la[c + (size_t)N * k] -= tC;
    }
}

// ---- link coefficients^T per face (kernels.cuh:116-120) and face BCs^T ----
// a_E = rho min(u_e, 0) Ax - mu Ax/dx, a_W = rho min(-u_w, 0) Ax - mu Ax/dx.
__global__ void k_adj_links(Params<double> P, AdjBufs b)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    const double *t = b.la;
    ADJ_LOOP(q, NU + NV)
    {
        if (q < NU) {
            const int i = q % (nx + 1), j = q / (nx + 1);
            const double ufv = b.uf[q];
            double l = 0.0;
            if (i > 0 && ufv < 0.0) l += t[i - 1 + nx * j + (size_t)N * AE] * g.rho * g.Ax;
            if (i < nx && ufv > 0.0) l += -t[i + nx * j + (size_t)N * AW] * g.rho * g.Ax;
            b.ouf[q] = (i > 0 && i < nx) ? l : 0.0;
            if (i == 0) {
                if (g.bc[WEST] == INLET) b.ltheta[j] += l;
                if (g.bc[WEST] == OUTLET) b.lufa[q] = l;
            }
            if (i == nx && g.bc[EAST] == OUTLET) b.lufa[q] = l;
        } else {
            const int qq = q - NU, j = qq / nx, i = qq % nx;
            const double vfv = b.vf[qq];
            double l = 0.0;
            if (j > 0 && vfv < 0.0) l += t[i + nx * (j - 1) + (size_t)N * AN] * g.rho * g.Ay;
            if (j < ny && vfv > 0.0) l += -t[i + nx * j + (size_t)N * AS] * g.rho * g.Ay;
            b.ovf[qq] = (j > 0 && j < ny) ? l : 0.0;
            if ((j == 0 && g.bc[SOUTH] == OUTLET) || (j == ny && g.bc[NORTH] == OUTLET)) b.lvfa[qq] = l;
        }
    }
}

// ---- pressure source^T, outlet faces^T, mu^T, new iterate, convergence ---
// mode bit 0: set the loop condition; bit 1: count the pass as an iteration.
__global__ void k_adj_finish(Params<double> P, AdjBufs b, int buf, Ctl *ctl, double *partials,
                             cudaGraphConditionalHandle cond, int mode)
{
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    const double *t = b.la;
    double red[3] = {0.0, 0.0, 0.0};  // dJ/dmu, max |delta|, max |lambda|
    ADJ_LOOP(c, N)
    {
        const int i = c % nx, j = c / nx;
        double lp = b.op[c];
        // b_u = 0.5 (p_l - p_r) Ax, b_v = 0.5 (p_s - p_n) Ay with the boundary rule
        if (i < nx - 1) lp += 0.5 * g.Ax * b.lbu[c + 1];
        if (i == 0 && g.closed[WEST]) lp += 0.5 * g.Ax * b.lbu[c];
        if (i > 0) lp -= 0.5 * g.Ax * b.lbu[c - 1];
        if (i == nx - 1 && g.closed[EAST]) lp -= 0.5 * g.Ax * b.lbu[c];
        if (j < ny - 1) lp += 0.5 * g.Ay * b.lbv[c + nx];
        if (j == 0 && g.closed[SOUTH]) lp += 0.5 * g.Ay * b.lbv[c];
        if (j > 0) lp -= 0.5 * g.Ay * b.lbv[c - nx];
        if (j == ny - 1 && g.closed[NORTH]) lp -= 0.5 * g.Ay * b.lbv[c];
        double lu = b.lus[buf][c], lv = b.lvs[buf][c];
        if (i == 0 && g.bc[WEST] == OUTLET) lu += b.lufa[(nx + 1) * j];
        if (i == nx - 1 && g.bc[EAST] == OUTLET) lu += b.lufa[nx + (nx + 1) * j];
        if (j == 0 && g.bc[SOUTH] == OUTLET) lv += b.lvfa[i];
        if (j == ny - 1 && g.bc[NORTH] == OUTLET) lv += b.lvfa[i + nx * ny];
        red[0] += -(t[c + (size_t)N * AE] + t[c + (size_t)N * AW]) * g.Ax / g.dx -
                  (t[c + (size_t)N * AN] + t[c + (size_t)N * AS]) * g.Ay / g.dy;
        const double nu = lu + b.ju[c], nv = lv + b.jv[c], np = lp + b.jp[c];
        red[1] = fmax(red[1], fmax(fabs(nu - b.lu[c]), fmax(fabs(nv - b.lv[c]), fabs(np - b.lp[c]))));
        red[2] = fmax(red[2], fmax(fabs(nu), fmax(fabs(nv), fabs(np))));
        b.ou[c] = nu;
        b.ov[c] = nv;
        b.op[c] = np;
    }
    ADJ_LOOP(q, NU)
    {
        red[1] = fmax(red[1], fabs(b.ouf[q] - b.luf[q]));
        red[2] = fmax(red[2], fabs(b.ouf[q]));
    }
    ADJ_LOOP(q, NV)
    {
        red[1] = fmax(red[1], fabs(b.ovf[q] - b.lvf[q]));
        red[2] = fmax(red[2], fabs(b.ovf[q]));
    }
    // block: sum for dJ/dmu, max for the others; then the last block combines
    // the per-block partials in block order (deterministic).
    __shared__ double sh[3][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    double s0 = warp_sum(red[0]);
    double m1 = red[1], m2 = red[2];
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
    }
    if (lane == 0) {
        sh[0][warp] = s0;
        sh[1][warp] = m1;
        sh[2][warp] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int w = 0; w < nw; ++w) {
            a0 += sh[0][w];
            a1 = fmax(a1, sh[1][w]);
            a2 = fmax(a2, sh[2][w]);
        }
        partials[blockIdx.x] = a0;
        partials[gridDim.x + blockIdx.x] = a1;
        partials[2 * gridDim.x + blockIdx.x] = a2;
        __threadfence();
        last = atomicAdd(&ctl->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int k = 0; k < (int)gridDim.x; ++k) {
        a0 += __ldcg(&partials[k]);
        a1 = fmax(a1, __ldcg(&partials[gridDim.x + k]));
        a2 = fmax(a2, __ldcg(&partials[2 * gridDim.x + k]));
    }
    ctl->counter = 0;
    b.scal[0] = a0;
    b.scal[1] = a1;
    b.scal[2] = a2;
    const double it = b.scal[3] + ((mode & 2) ? 1.0 : 0.0);
    b.scal[3] = it;
    const bool conv = a1 <= b.scal[6] * a2;
    b.scal[4] = conv ? 1.0 : 0.0;
    if (mode & 1) cudaGraphSetConditional(cond, (conv || it >= b.scal[7]) ? 0u : 1u);
}

// The new iterate becomes the current one (kept apart so that the
// convergence measure compares old and new).
__global__ void k_adj_copy(Params<double> P, AdjBufs b)
{
    const int nx = P.g.nx, ny = P.g.ny, N = P.g.N;
    const int NU = (nx + 1) * ny, NV = nx * (ny + 1);
    ADJ_LOOP(q, N)
    {
        b.lu[q] = b.ou[q];
        b.lv[q] = b.ov[q];
        b.lp[q] = b.op[q];
    }
    ADJ_LOOP(q, NU) b.luf[q] = b.ouf[q];
    ADJ_LOOP(q, NV) b.lvf[q] = b.ovf[q];
}

#undef ADJ_LOOP

}  // namespace ifc
