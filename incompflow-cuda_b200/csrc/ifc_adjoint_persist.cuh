// ifc_adjoint_persist.cuh -- the whole adjoint fixed-point solve of
// ifc_adjoint2d.cuh in one cooperative launch.
//
// Every CTA owns one TX x TY tile for the whole solve.  The linearisation is
// frozen, so the CTA stages the transposed-sweep weights of its tile plus a
// halo of H = 2*KS cells (a_nb/aC and 1/aC of the momentum and p' links) in
// shared memory once and keeps them there.  One reverse pass is:
//   P1  corrections^T per cell (+ block sums for the p' mean removal)
//   P2  transposed p' sweeps, KS per pass, temporally blocked in shared memory
//   P3  p' source^T + Rhie-Chow^T + face BCs^T per cell
//   P4  transposed u/v sweeps, KS per pass, temporally blocked
//   P5a boundary fold-in^T per cell: link adjoints t_nb = la_nb - la_C, where
//       la_nb = -(u_nb lb_u + v_nb lb_v) (the sweeps' link adjoint is the
//       source adjoint times the neighbour value, since phi is the fixed point)
//   P5b link coefficients^T, face BCs^T, pressure source^T, new iterate and
//       the FP64 convergence measure
// separated by grid barriers (bounded waits, as in the primal's single-launch
// solve).  A transposed half sweep of colour h makes the cells of the other
// colour gather -alpha a_X->c / aC_X lambda_X from their colour-h neighbours
// X and the colour-h cells add alpha/aC_X lambda_X to their source adjoint;
// the colour-h cells' own factor (1 - alpha) is applied when they gather in
// the next half sweep (or at write-back after the last), so a half sweep
// updates in place with one __syncthreads.  After a pass of 2*ns half sweeps
// every tile cell holds exactly what ns global transposed sweeps give (each
// half sweep moves information one cell; halo cells farther than the
// remaining reach are skipped).  All values FP64.
#pragma once

#include "ifc_adjoint2d.cuh"
#include "ifc_persist2d.cuh"

namespace ifc {

struct AdjPArgs {
    int n_iter[3];     // u, v, p' sweeps per outer iteration
    int pin;
    double alpha[3];   // u, v, p' relaxation
    double ru, rv;     // relax_u*0.5, relax_v*0.5
    int max_iter;
    double tol;
    int single;        // 1: one reverse pass of the given lambda, no fixed-point loop
};

struct AdjLam {
    double *u, *v, *p, *uf, *vf;
};

__device__ __forceinline__ AdjLam lam_buf(const AdjBufs &b, int k)
{
    AdjLam L;
    L.u = k == 0 ? b.lu : b.ou;
    L.v = k == 0 ? b.lv : b.ov;
    L.p = k == 0 ? b.lp : b.op;
    L.uf = k == 0 ? b.luf : b.ouf;
    L.vf = k == 0 ? b.lvf : b.ovf;
    return L;
}

// Per-CTA partials of (sum, max, max) in warp order, and their grid totals in
// a fixed order (identical in every CTA).
template <int NT>
__device__ __forceinline__ void smm_partials(double s, double m1, double m2, double *partials, int G)
{
    __shared__ double red[NT / 32][3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    s = warp_sum(s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_down_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_down_sync(0xffffffffu, m2, o));
    }
    if (lane == 0) {
        red[warp][0] = s;
        red[warp][1] = m1;
        red[warp][2] = m2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int w = 0; w < NT / 32; ++w) {
            a0 += red[w][0];
            a1 = fmax(a1, red[w][1]);
            a2 = fmax(a2, red[w][2]);
        }
        partials[blockIdx.x] = a0;
        partials[G + blockIdx.x] = a1;
        partials[2 * G + blockIdx.x] = a2;
    }
}

template <int NT>
__device__ __forceinline__ void smm_reduce(const double *partials, int G, double *out)
{
    // warp 0: sum of column 0; warps 1, 2: max of columns 1, 2 (lane-strided,
    // then one shuffle tree: a fixed order, identical in every CTA)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (warp < 3) {
        const double *col = partials + (size_t)warp * G;
        double x = 0.0;
        for (int b = lane; b < G; b += 32) {
            const double y = __ldcg(&col[b]);
            x = warp == 0 ? x + y : fmax(x, y);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double y = __shfl_down_sync(0xffffffffu, x, o);
            x = warp == 0 ? x + y : fmax(x, y);
        }
        if (lane == 0) out[warp] = x;
    }
    __syncthreads();
}

// Adjoint of an x face k (0..nx) of row j after the p' source^T: the interior
// seed plus rho Ax (lb_p(right cell) - lb_p(left cell)).
__device__ __forceinline__ double lufs_x(const Params<double> &P, const AdjBufs &b, const double *luf, int k, int j)
{
    const int nx = P.g.nx;
    const double v = (k > 0 && k < nx) ? luf[k + (nx + 1) * j] : 0.0;
    double gs = 0.0;
    if (k < nx) gs += b.lbp[k + nx * j];
    if (k > 0) gs -= b.lbp[k - 1 + nx * j];
    return v + P.g.rho * P.g.Ax * gs;
}

__device__ __forceinline__ double lufs_y(const Params<double> &P, const AdjBufs &b, const double *lvf, int i, int k)
{
    const int nx = P.g.nx, ny = P.g.ny;
    const double v = (k > 0 && k < ny) ? lvf[i + nx * k] : 0.0;
    double gs = 0.0;
    if (k < ny) gs += b.lbp[i + nx * k];
    if (k > 0) gs -= b.lbp[i + nx * (k - 1)];
    return v + P.g.rho * P.g.Ay * gs;
}

// NC transposed red-black sweeps' worth of half sweeps (ns[m] sweeps of
// component m) on the staged region.  lb: this thread's source-adjoint
// accumulators of its own tile cells.  w: 4 planes (E W N S) of a_nb/aC, ra:
// 1/aC of every staged cell (0 outside the domain).
template <int NC, int W, int CPT, int KS>
__device__ __forceinline__ void tsweeps(double *const (&l)[NC], const double *w, const double *ra, int NR,
                                        const int (&ns)[NC], const double (&alpha)[NC], const int (&cq)[2][CPT],
                                        const int (&dq)[2][CPT], const bool (&own)[2][CPT],
                                        double (&lb)[NC][2][CPT])
{
    const double *wE = w, *wW = w + NR, *wN = w + 2 * NR, *wS = w + 3 * NR;
    int nmax = 0;
#pragma unroll
    for (int m = 0; m < NC; ++m) nmax = ns[m] > nmax ? ns[m] : nmax;
#pragma unroll 1
    for (int s = 0; s < nmax; ++s) {
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const int h = 1 - hh;       // active colour: 1, then 0
            const int oc = hh;          // gathering colour
            const int k = 2 * s + hh;   // half sweep within the pass
#pragma unroll
            for (int kk = 0; kk < CPT; ++kk) {
                const int q = cq[oc][kk];
                if (q < 0) continue;
                const double we = wE[q - 1], ww = wW[q + 1], wn = wN[q - W], wsv = wS[q + W];
#pragma unroll
                for (int m = 0; m < NC; ++m) {
                    if (s >= ns[m] || dq[oc][kk] > 2 * ns[m] - 1 - k) continue;
                    const double *L = l[m];
                    const double sc = k > 0 ? 1.0 - alpha[m] : 1.0;
                    const double g = we * L[q - 1] + ww * L[q + 1] + wn * L[q - W] + wsv * L[q + W];
                    l[m][q] = sc * L[q] - alpha[m] * g;
                }
            }
#pragma unroll
            for (int kk = 0; kk < CPT; ++kk) {
                const int q = cq[h][kk];
                if (q < 0 || !own[h][kk]) continue;
#pragma unroll
                for (int m = 0; m < NC; ++m)
                    if (s < ns[m]) lb[m][h][kk] += alpha[m] * ra[q] * l[m][q];
            }
            __syncthreads();
        }
    }
}

template <int TX, int TY, int KS, int NT>
__global__ void __launch_bounds__(NT, 1) k_adjoint2d(Params<double> P, AdjBufs b, AdjPArgs pa, double *partials,
                                                    GridBarrier *bar)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    const Geo<double> &g = P.g;
    const int nx = g.nx, ny = g.ny, N = g.N;
    const int G = gridDim.x;
    const int tid = threadIdx.x;
    const int tiles_x = (nx + TX - 1) / TX;
    const int x0 = (blockIdx.x % tiles_x) * TX, y0 = (blockIdx.x / tiles_x) * TY;
    const int gx0 = x0 - H, gy0 = y0 - H;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sl0 = reinterpret_cast<double *>(smem_raw);
    double *sl1 = sl0 + NR;
    double *mw = sl1 + NR;   // 4 planes
    double *mra = mw + 4 * NR;
    double *pw = mra + NR;   // 4 planes
    double *pra = pw + 4 * NR;
    __shared__ double tot[4];

    // Frozen weights of the staged region.
    for (int q = tid; q < NR; q += NT) {
        const int gi = gx0 + q % W, gj = gy0 + q / W;
        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
        const size_t id = (size_t)gi + (size_t)nx * gj;
        const double r = in ? 1.0 / b.afold[id] : 0.0;
        const double rp = in ? 1.0 / b.ap[id] : 0.0;
        mra[q] = r;
        pra[q] = rp;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            mw[k * NR + q] = in ? b.afold[id + (size_t)N * (AE + k)] * r : 0.0;
            pw[k * NR + q] = in ? b.ap[id + (size_t)N * (AE + k)] * rp : 0.0;
        }
    }
    int cq[2][CPT], dq[2][CPT];
    bool own[2][CPT];
    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < CPT; ++k) {
            dq[c][k] = tile_distance<W, H, TX, TY>(cq[c][k]);
            const int q = cq[c][k];
            own[c][k] = q >= 0 && q % W >= H && q % W < H + TX && q / W >= H && q / W < H + TY;
        }
    __syncthreads();

    const int npass_p = (pa.n_iter[2] + KS - 1) / KS;
    const int npass_m = (max(pa.n_iter[0], pa.n_iter[1]) + KS - 1) / KS;
    const double c83 = 8.0 / 3.0;
    unsigned int epoch = 0;
    bool failed = false;
    bool final = pa.single != 0;
    int cur = 0, it = 0;

    for (;;) {
        const AdjLam in = lam_buf(b, cur), out = lam_buf(b, 1 - cur);
        // ---------------- P1: corrections^T ----------------
        double pinsum = 0.0;
        for (int q = tid; q < TX * TY; q += NT) {
            const int i = x0 + q % TX, j = y0 + q / TX;
            if (i >= nx || j >= ny) continue;
            const int c = i + nx * j;
            const double *aC = b.afold;
            double x = pa.alpha[2] * in.p[c];
            if (i < nx - 1) x += pa.ru * g.Ax / aC[c + 1] * in.u[c + 1];
            if (i == 0 && g.closed[WEST]) x += pa.ru * g.Ax / aC[c] * in.u[c];
            if (i > 0) x -= pa.ru * g.Ax / aC[c - 1] * in.u[c - 1];
            if (i == nx - 1 && g.closed[EAST]) x -= pa.ru * g.Ax / aC[c] * in.u[c];
            if (j < ny - 1) x += pa.rv * g.Ay / aC[c + nx] * in.v[c + nx];
            if (j == 0 && g.closed[SOUTH]) x += pa.rv * g.Ay / aC[c] * in.v[c];
            if (j > 0) x -= pa.rv * g.Ay / aC[c - nx] * in.v[c - nx];
            if (j == ny - 1 && g.closed[NORTH]) x -= pa.rv * g.Ay / aC[c] * in.v[c];
            const int fu = i + (nx + 1) * j;
            if (i < nx - 1) x += pa.ru * (1.0 / aC[c] + 1.0 / aC[c + 1]) * g.Ax * in.uf[fu + 1];
            if (i > 0) x -= pa.ru * (1.0 / aC[c - 1] + 1.0 / aC[c]) * g.Ax * in.uf[fu];
            if (j < ny - 1) x += pa.rv * (1.0 / aC[c] + 1.0 / aC[c + nx]) * g.Ay * in.vf[c + nx];
            if (j > 0) x -= pa.rv * (1.0 / aC[c - nx] + 1.0 / aC[c]) * g.Ay * in.vf[c];
            b.lpc[0][c] = x;
            out.p[c] = in.p[c];
            pinsum += x;
            if (i == 0) b.ltheta[j] = 0.0;
        }
        if (pa.pin) smm_partials<NT>(pinsum, 0.0, 0.0, partials + 3 * (size_t)G, G);
        if (!grid_sync(bar, G, epoch)) { failed = true; break; }
        double mean = 0.0;
        if (pa.pin) {
            smm_reduce<NT>(partials + 3 * (size_t)G, G, tot);
            mean = tot[0] / (double)N;
        }

        // ---------------- P2: transposed p' sweeps ----------------
        {
            double lbp[1][2][CPT];
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int k = 0; k < CPT; ++k) lbp[0][c][k] = 0.0;
            for (int pass = 0; pass < npass_p; ++pass) {
                const int nsw[1] = {clamp_sweeps(pa.n_iter[2], pass, KS)};
                const double *src = b.lpc[pass & 1];
                double *dst = b.lpc[(pass + 1) & 1];
                const double shift = pass == 0 ? mean : 0.0;
                for (int q = tid; q < NR; q += NT) {
                    const int gi = gx0 + q % W, gj = gy0 + q / W;
                    const bool inr = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
                    sl0[q] = inr ? src[gi + nx * gj] - shift : 0.0;
                }
                __syncthreads();
                double *const ls[1] = {sl0};
                const double al[1] = {pa.alpha[2]};
                tsweeps<1, W, CPT, KS>(ls, pw, pra, NR, nsw, al, cq, dq, own, lbp);
                const double sc = 1.0 - pa.alpha[2];
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        const int q = cq[c][k];
                        if (q < 0 || !own[c][k]) continue;
                        const int id = gx0 + q % W + nx * (gy0 + q / W);
                        dst[id] = c == 0 && nsw[0] > 0 ? sc * sl0[q] : sl0[q];
                        if (pass == npass_p - 1) b.lbp[id] = lbp[0][c][k];
                    }
                if (!grid_sync(bar, G, epoch)) { failed = true; break; }
            }
            if (failed) break;
            if (npass_p == 0) {
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = x0 + q % TX, j = y0 + q / TX;
                    if (i < nx && j < ny) b.lbp[i + nx * j] = 0.0;
                }
                if (!grid_sync(bar, G, epoch)) { failed = true; break; }
            }
        }

        // ---------------- P3: p' source^T, Rhie-Chow^T, face BCs^T ----------------
        for (int q = tid; q < TX * TY; q += NT) {
            const int i = x0 + q % TX, j = y0 + q / TX;
            if (i >= nx || j >= ny) continue;
            const int c = i + nx * j;
            double lu = in.u[c], lv = in.v[c], lp = 0.0, lac = 0.0;
            for (int k = i - 1; k <= i + 2; ++k) {
                if (k < 1 || k > nx - 1) continue;
                const double l = lufs_x(P, b, in.uf, k, j);
                if (l == 0.0) continue;
                rc_face_adj(b.p + (size_t)nx * j, b.afold + (size_t)nx * j, k, nx, 1, g.Ax, g.closed[WEST],
                            g.closed[EAST], l, i, lp, lac);
            }
            if (i >= 1) lu += 0.5 * lufs_x(P, b, in.uf, i, j);
            if (i <= nx - 2) lu += 0.5 * lufs_x(P, b, in.uf, i + 1, j);
            if (i == 0 && g.bc[WEST] == OUTLET) lu += lufs_x(P, b, in.uf, 0, j);
            if (i == nx - 1 && g.bc[EAST] == OUTLET) lu += lufs_x(P, b, in.uf, nx, j);
            if (i == 0 && g.bc[WEST] == INLET) b.ltheta[j] += lufs_x(P, b, in.uf, 0, j);
            for (int k = j - 1; k <= j + 2; ++k) {
                if (k < 1 || k > ny - 1) continue;
                const double l = lufs_y(P, b, in.vf, i, k);
                if (l == 0.0) continue;
                rc_face_adj(b.p + i, b.afold + i, k, ny, nx, g.Ay, g.closed[SOUTH], g.closed[NORTH], l, j, lp, lac);
            }
            if (j >= 1) lv += 0.5 * lufs_y(P, b, in.vf, i, j);
            if (j <= ny - 2) lv += 0.5 * lufs_y(P, b, in.vf, i, j + 1);
            if (j == 0 && g.bc[SOUTH] == OUTLET) lv += lufs_y(P, b, in.vf, i, 0);
            if (j == ny - 1 && g.bc[NORTH] == OUTLET) lv += lufs_y(P, b, in.vf, i, ny);
            b.lus[0][c] = lu;
            b.lvs[0][c] = lv;
            out.p[c] += lp;
            b.la[c] = lac;
        }
        if (!grid_sync(bar, G, epoch)) { failed = true; break; }

        // ---------------- P4: transposed momentum sweeps ----------------
        {
            double lbm[2][2][CPT];
#pragma unroll
            for (int m = 0; m < 2; ++m)
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int k = 0; k < CPT; ++k) lbm[m][c][k] = 0.0;
            for (int pass = 0; pass < npass_m; ++pass) {
                const int nsw[2] = {clamp_sweeps(pa.n_iter[0], pass, KS), clamp_sweeps(pa.n_iter[1], pass, KS)};
                const double *su = b.lus[pass & 1], *sv = b.lvs[pass & 1];
                double *du = b.lus[(pass + 1) & 1], *dv = b.lvs[(pass + 1) & 1];
                for (int q = tid; q < NR; q += NT) {
                    const int gi = gx0 + q % W, gj = gy0 + q / W;
                    const bool inr = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
                    const int id = gi + nx * gj;
                    sl0[q] = inr ? su[id] : 0.0;
                    sl1[q] = inr ? sv[id] : 0.0;
                }
                __syncthreads();
                double *const ls[2] = {sl0, sl1};
                const double al[2] = {pa.alpha[0], pa.alpha[1]};
                tsweeps<2, W, CPT, KS>(ls, mw, mra, NR, nsw, al, cq, dq, own, lbm);
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int k = 0; k < CPT; ++k) {
                        const int q = cq[c][k];
                        if (q < 0 || !own[c][k]) continue;
                        const int id = gx0 + q % W + nx * (gy0 + q / W);
                        du[id] = c == 0 && nsw[0] > 0 ? (1.0 - pa.alpha[0]) * sl0[q] : sl0[q];
                        dv[id] = c == 0 && nsw[1] > 0 ? (1.0 - pa.alpha[1]) * sl1[q] : sl1[q];
                        if (pass == npass_m - 1) {
                            b.lbu[id] = lbm[0][c][k];
                            b.lbv[id] = lbm[1][c][k];
                        }
                    }
                if (pass < npass_m - 1) {
                    if (!grid_sync(bar, G, epoch)) { failed = true; break; }
                } else {
                    __syncthreads();
                }
            }
            if (failed) break;
            if (npass_m == 0) {
                for (int q = tid; q < TX * TY; q += NT) {
                    const int i = x0 + q % TX, j = y0 + q / TX;
                    if (i < nx && j < ny) {
                        b.lbu[i + nx * j] = 0.0;
                        b.lbv[i + nx * j] = 0.0;
                    }
                }
                __syncthreads();
            }
        }
        const double *lus_f = b.lus[npass_m & 1], *lvs_f = b.lvs[npass_m & 1];

        // ---------------- P5a: fold-in^T, link adjoints ----------------
        double dmu = 0.0;
        for (int q = tid; q < TX * TY; q += NT) {
            const int i = x0 + q % TX, j = y0 + q / TX;
            if (i >= nx || j >= ny) continue;
            const int c = i + nx * j;
            const double lbu = b.lbu[c], lbv = b.lbv[c];
            double la[5];
            la[AC] = b.la[c] - (b.u[c] * lbu + b.v[c] * lbv);
            la[AE] = i < nx - 1 ? -(b.u[c + 1] * lbu + b.v[c + 1] * lbv) : 0.0;
            la[AW] = i > 0 ? -(b.u[c - 1] * lbu + b.v[c - 1] * lbv) : 0.0;
            la[AN] = j < ny - 1 ? -(b.u[c + nx] * lbu + b.v[c + nx] * lbv) : 0.0;
            la[AS] = j > 0 ? -(b.u[c - nx] * lbu + b.v[c - nx] * lbv) : 0.0;
            const int faces[4] = {SOUTH, NORTH, WEST, EAST};
#pragma unroll
            for (int fq = 0; fq < 4; ++fq) {
                const int F = faces[fq];
                const bool on = (F == SOUTH && j == 0) || (F == NORTH && j == ny - 1) || (F == WEST && i == 0) ||
                                (F == EAST && i == nx - 1);
                if (!on) continue;
                const int ex = F == EAST ? AE : F == WEST ? AW : F == NORTH ? AN : AS;
                const int inl = F == EAST ? AW : F == WEST ? AE : F == NORTH ? AS : AN;
                if (g.bc[F] == OUTLET) {
                    la[ex] = la[AC];
                    continue;
                }
                double ubc = g.bcv[F][0];
                const double vbc = g.bcv[F][1];
                const bool prof = F == WEST && g.bc[WEST] == INLET;
                if (prof && g.inlet) ubc = g.inlet[j];
                la[ex] = -2.0 * la[AC] + la[inl] / 3.0 - c83 * ubc * lbu - c83 * vbc * lbv;
                if (prof) b.ltheta[j] += -c83 * b.araw[c + (size_t)N * ex] * lbu;
            }
            const double tE = la[AE] - la[AC], tW = la[AW] - la[AC], tN = la[AN] - la[AC], tS = la[AS] - la[AC];
            b.la[c + (size_t)N * AE] = tE;
            b.la[c + (size_t)N * AW] = tW;
            b.la[c + (size_t)N * AN] = tN;
            b.la[c + (size_t)N * AS] = tS;
            dmu += -(tE + tW) * g.Ax / g.dx - (tN + tS) * g.Ay / g.dy;
        }
        if (!grid_sync(bar, G, epoch)) { failed = true; break; }

        // ---------------- P5b: links^T, face BCs^T, pressure source^T, new iterate ----------------
        double mdel = 0.0, mabs = 0.0;
        {
            const double *t = b.la;
            const double rAx = g.rho * g.Ax, rAy = g.rho * g.Ay;
            for (int q = tid; q < TX * TY; q += NT) {
                const int i = x0 + q % TX, j = y0 + q / TX;
                if (i >= nx || j >= ny) continue;
                const int c = i + nx * j;
                double lu = lus_f[c], lv = lvs_f[c];
                // west face of the cell
                const int fw = i + (nx + 1) * j;
                {
                    const double ufv = b.uf[fw];
                    double l = 0.0;
                    if (i > 0 && ufv < 0.0) l += t[c - 1 + (size_t)N * AE] * rAx;
                    if (ufv > 0.0) l += -t[c + (size_t)N * AW] * rAx;
                    if (i > 0) {
                        out.uf[fw] = l;
                        mdel = fmax(mdel, fabs(l - in.uf[fw]));
                        mabs = fmax(mabs, fabs(l));
                    } else {
                        out.uf[fw] = 0.0;
                        if (g.bc[WEST] == INLET) b.ltheta[j] += l;
                        if (g.bc[WEST] == OUTLET) lu += l;
                    }
                }
                if (i == nx - 1) {
                    const double ufv = b.uf[fw + 1];
                    const double l = ufv < 0.0 ? t[c + (size_t)N * AE] * rAx : 0.0;
                    out.uf[fw + 1] = 0.0;
                    if (g.bc[EAST] == OUTLET) lu += l;
                }
                {
                    const double vfv = b.vf[c];
                    double l = 0.0;
                    if (j > 0 && vfv < 0.0) l += t[c - nx + (size_t)N * AN] * rAy;
                    if (vfv > 0.0) l += -t[c + (size_t)N * AS] * rAy;
                    if (j > 0) {
                        out.vf[c] = l;
                        mdel = fmax(mdel, fabs(l - in.vf[c]));
                        mabs = fmax(mabs, fabs(l));
                    } else {
                        out.vf[c] = 0.0;
                        if (g.bc[SOUTH] == OUTLET) lv += l;
                    }
                }
                if (j == ny - 1) {
                    const double vfv = b.vf[c + nx];
                    const double l = vfv < 0.0 ? t[c + (size_t)N * AN] * rAy : 0.0;
                    out.vf[c + nx] = 0.0;
                    if (g.bc[NORTH] == OUTLET) lv += l;
                }
                double lp = out.p[c];
                if (i < nx - 1) lp += 0.5 * g.Ax * b.lbu[c + 1];
                if (i == 0 && g.closed[WEST]) lp += 0.5 * g.Ax * b.lbu[c];
                if (i > 0) lp -= 0.5 * g.Ax * b.lbu[c - 1];
                if (i == nx - 1 && g.closed[EAST]) lp -= 0.5 * g.Ax * b.lbu[c];
                if (j < ny - 1) lp += 0.5 * g.Ay * b.lbv[c + nx];
                if (j == 0 && g.closed[SOUTH]) lp += 0.5 * g.Ay * b.lbv[c];
                if (j > 0) lp -= 0.5 * g.Ay * b.lbv[c - nx];
                if (j == ny - 1 && g.closed[NORTH]) lp -= 0.5 * g.Ay * b.lbv[c];
                const double nu = lu + b.ju[c], nv = lv + b.jv[c], np = lp + b.jp[c];
                mdel = fmax(mdel, fmax(fabs(nu - in.u[c]), fmax(fabs(nv - in.v[c]), fabs(np - in.p[c]))));
                mabs = fmax(mabs, fmax(fabs(nu), fmax(fabs(nv), fabs(np))));
                out.u[c] = nu;
                out.v[c] = nv;
                out.p[c] = np;
            }
        }
        smm_partials<NT>(dmu, mdel, mabs, partials, G);
        if (!grid_sync(bar, G, epoch)) { failed = true; break; }
        smm_reduce<NT>(partials, G, tot);
        if (final) {
            if (blockIdx.x == 0 && tid == 0) b.scal[0] = tot[0];
            break;
        }
        ++it;
        const bool conv = tot[1] <= pa.tol * tot[2];
        if (blockIdx.x == 0 && tid == 0) {
            b.scal[1] = tot[1];
            b.scal[2] = tot[2];
            b.scal[3] = (double)it;
            b.scal[4] = conv ? 1.0 : 0.0;
        }
        if (conv || it >= pa.max_iter) final = true;
        cur ^= 1;
    }
    if (tid == 0 && (failed || bar->err)) atomicExch(&bar->err, 1);
}

}  // namespace ifc
