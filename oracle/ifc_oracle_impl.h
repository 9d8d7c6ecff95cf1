/*
 * ifc_oracle_impl.h -- body of the CPU oracle, instantiated twice by
 * ifc_oracle.c with T = float / double and S = f / d.  TEST INFRASTRUCTURE ONLY.
 *
 * Every function names the reference code it restates
 * (WanZijun271/IncompFlow-CUDA, paths relative to that project).
 * Casts to (double) mark the places where the reference's double literals
 * (0.5, -0.5, 1e-20) promote a float expression to FP64 (defect D13 in the
 * reference review); results are rounded back to T where the reference stores
 * them into a `scalar` array.  In the double build the casts are no-ops.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define ST CAT(orc_state_, S)
#define FN(name) CAT(CAT(orc_, name), CAT(_, S))

struct CAT(orc_state_, S) {
    orc_config cfg;
    int dim, nx, ny, nz;
    size_t N;
    T dx, dy, dz, Ax, Ay, Az, rho, mu;
    T relax[4], tol[4];
    T *f[ORC_F_COUNT];
    size_t len[ORC_F_COUNT];
    T *tmp;
    int it;
    double max_p, max_u, max_v, max_w, max_uf, max_vf, max_wf;
    double rmax[4];             /* running maxima of the u, v, w residuals and the mass imbalance */
};

#define CID(s, i, j, k) ((size_t)(i) + (size_t)(s)->nx * ((size_t)(j) + (size_t)(s)->ny * (size_t)(k)))
#define UFID(s, i, j, k) ((size_t)(i) + (size_t)((s)->nx + 1) * ((size_t)(j) + (size_t)(s)->ny * (size_t)(k)))
#define VFID(s, i, j, k) ((size_t)(i) + (size_t)(s)->nx * ((size_t)(j) + (size_t)((s)->ny + 1) * (size_t)(k)))
#define WFID(s, i, j, k) ((size_t)(i) + (size_t)(s)->nx * ((size_t)(j) + (size_t)(s)->ny * (size_t)(k)))

static inline T CAT(min0_, S)(T x) { return x < (T)0 ? x : (T)0; }
#define MIN0 CAT(min0_, S)

/* OpenMP build (make -C oracle oracle_omp, for the all-cores CPU baseline
 * only): the per-cell loops of the sweeps, the link coefficients and
 * Rhie-Chow run over rows in parallel.  Each cell is computed as in the
 * serial build; only the FP64 sums of the sweeps are added in another order. */
#ifndef ORC_PAR_ROWS
#ifdef ORC_OMP
#define ORC_PAR_ROWS _Pragma("omp parallel for collapse(2) schedule(static)")
#define ORC_PAR_ROWS_SUM _Pragma("omp parallel for collapse(2) schedule(static) reduction(+ : sq)")
#else
#define ORC_PAR_ROWS
#define ORC_PAR_ROWS_SUM
#endif
#endif

ST *FN(create)(const orc_config *cfg)
{
    ST *s = (ST *)calloc(1, sizeof(ST));
    if (!s) return NULL;
    s->cfg = *cfg;
    s->dim = cfg->dim;
    s->nx = cfg->nx;
    s->ny = cfg->ny;
    s->nz = cfg->dim == 2 ? 1 : cfg->nz;
    s->N = (size_t)s->nx * s->ny * s->nz;
    /* include/constants.h:22-28: derived constants are evaluated in `scalar`. */
    {
        T xmax = (T)cfg->xmax, xmin = (T)cfg->xmin, ymax = (T)cfg->ymax, ymin = (T)cfg->ymin;
        T zmax = (T)cfg->zmax, zmin = (T)cfg->zmin;
        s->dx = (xmax - xmin) / (T)s->nx;
        const int sy = (cfg->slab_axis_cells > 0 && s->dim == 2) ? cfg->slab_axis_cells : s->ny;
        const int sz = (cfg->slab_axis_cells > 0 && s->dim == 3) ? cfg->slab_axis_cells : s->nz;
        s->dy = (ymax - ymin) / (T)sy;
        s->dz = (zmax - zmin) / (T)sz;
        s->Ax = s->dy * s->dz;
        s->Ay = s->dz * s->dx;
        s->Az = s->dx * s->dy;
    }
    s->rho = (T)cfg->density;
    s->mu = (T)cfg->viscosity;
    for (int q = 0; q < 4; ++q) {
        s->relax[q] = (T)cfg->relax[q];
        s->tol[q] = (T)cfg->tol[q];
    }
    size_t N = s->N, nc = (size_t)(2 * s->dim + 1);
    s->len[ORC_F_U] = s->len[ORC_F_V] = s->len[ORC_F_W] = s->len[ORC_F_P] = s->len[ORC_F_PC] = N;
    s->len[ORC_F_SRC_U] = s->len[ORC_F_SRC_V] = s->len[ORC_F_SRC_W] = s->len[ORC_F_SRC_P] = N;
    s->len[ORC_F_UF] = (size_t)(s->nx + 1) * s->ny * s->nz;
    s->len[ORC_F_VF] = (size_t)s->nx * (s->ny + 1) * s->nz;
    s->len[ORC_F_WF] = (size_t)s->nx * s->ny * (s->nz + 1);
    s->len[ORC_F_MCOEF] = s->len[ORC_F_PCOEF] = N * nc;
    for (int q = 0; q < ORC_F_COUNT; ++q) {
        s->f[q] = (T *)calloc(s->len[q], sizeof(T));
        if (!s->f[q]) return NULL;
    }
    s->tmp = (T *)calloc(N, sizeof(T));
    return s;
}

void FN(destroy)(ST *s)
{
    if (!s) return;
    for (int q = 0; q < ORC_F_COUNT; ++q) free(s->f[q]);
    free(s->tmp);
    free(s);
}

T *FN(field)(ST *s, int field) { return (field >= 0 && field < ORC_F_COUNT) ? s->f[field] : NULL; }
size_t FN(field_len)(const ST *s, int field) { return (field >= 0 && field < ORC_F_COUNT) ? s->len[field] : 0; }
int FN(iteration_count)(const ST *s) { return s->it; }

/* include/kernels.cuh:10-45 (initFaceVelKernel): interior faces take the mean of
 * the two neighbouring cells.  Only on the first outer iteration
 * (src/Solver.cu:162-164). */
void FN(init_face_vel)(ST *s)
{
    const T *u = s->f[ORC_F_U], *v = s->f[ORC_F_V], *w = s->f[ORC_F_W];
    T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 1; i < s->nx; ++i)
                uf[UFID(s, i, j, k)] = (u[CID(s, i - 1, j, k)] + u[CID(s, i, j, k)]) / (T)2;
    for (int k = 0; k < s->nz; ++k)
        for (int j = 1; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i)
                vf[VFID(s, i, j, k)] = (v[CID(s, i, j - 1, k)] + v[CID(s, i, j, k)]) / (T)2;
    if (s->dim == 3)
        for (int k = 1; k < s->nz; ++k)
            for (int j = 0; j < s->ny; ++j)
                for (int i = 0; i < s->nx; ++i)
                    wf[WFID(s, i, j, k)] = (w[CID(s, i, j, k - 1)] + w[CID(s, i, j, k)]) / (T)2;
}

static T CAT(west_inlet_, S)(const ST *s, int j, int k)
{
    if (s->cfg.inlet_profile && s->cfg.bc_type[ORC_WEST] == ORC_INLET)
        return (T)s->cfg.inlet_profile[(size_t)j + (size_t)s->ny * k];
    return (T)s->cfg.bc_val[ORC_WEST][0];
}

/* include/kernels.cuh:47-95 (applyBCsToFaceVelKernel), launched per face by
 * src/Solver.cu:410-465: wall -> 0, inlet -> prescribed normal component,
 * outlet -> velocity of the adjacent cell. */
void FN(bc_face_vel)(ST *s)
{
    const orc_config *c = &s->cfg;
    const T *u = s->f[ORC_F_U], *v = s->f[ORC_F_V], *w = s->f[ORC_F_W];
    T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j) {
            int t = c->bc_type[ORC_WEST];
            uf[UFID(s, 0, j, k)] = t == ORC_WALL ? (T)0 : t == ORC_INLET ? CAT(west_inlet_, S)(s, j, k) : u[CID(s, 0, j, k)];
            t = c->bc_type[ORC_EAST];
            uf[UFID(s, s->nx, j, k)] = t == ORC_WALL ? (T)0 : t == ORC_INLET ? (T)c->bc_val[ORC_EAST][0] : u[CID(s, s->nx - 1, j, k)];
        }
    for (int k = 0; k < s->nz; ++k)
        for (int i = 0; i < s->nx; ++i) {
            int t = c->bc_type[ORC_SOUTH];
            vf[VFID(s, i, 0, k)] = t == ORC_WALL ? (T)0 : t == ORC_INLET ? (T)c->bc_val[ORC_SOUTH][1] : v[CID(s, i, 0, k)];
            t = c->bc_type[ORC_NORTH];
            vf[VFID(s, i, s->ny, k)] = t == ORC_WALL ? (T)0 : t == ORC_INLET ? (T)c->bc_val[ORC_NORTH][1] : v[CID(s, i, s->ny - 1, k)];
        }
    if (s->dim == 3)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                int t = c->bc_type[ORC_BOTTOM];
                wf[WFID(s, i, j, 0)] = t == ORC_WALL ? (T)0 : t == ORC_INLET ? (T)c->bc_val[ORC_BOTTOM][2] : w[CID(s, i, j, 0)];
                t = c->bc_type[ORC_TOP];
                wf[WFID(s, i, j, s->nz)] = t == ORC_WALL ? (T)0 : t == ORC_INLET ? (T)c->bc_val[ORC_TOP][2] : w[CID(s, i, j, s->nz - 1)];
            }
}

/* include/kernels.cuh:97-134 (calcMomLinkCoefKernel): first-order upwind
 * convection plus central diffusion; aC = -sum(a_nb).  One coefficient set
 * serves u, v and w (the reference copies it, src/Solver.cu:167-171). */
void FN(mom_link_coef)(ST *s)
{
    const T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    T *a = s->f[ORC_F_MCOEF];
    const size_t N = s->N;
    const T rho = s->rho, mu = s->mu, Ax = s->Ax, Ay = s->Ay, Az = s->Az;
    ORC_PAR_ROWS
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t id = CID(s, i, j, k);
                T ue = uf[UFID(s, i + 1, j, k)], uw = uf[UFID(s, i, j, k)];
                T vn = vf[VFID(s, i, j + 1, k)], vs = vf[VFID(s, i, j, k)];
                T aE = (rho * MIN0(ue) * Ax) - mu * Ax / s->dx;
                T aW = (rho * MIN0(-uw) * Ax) - mu * Ax / s->dx;
                T aN = (rho * MIN0(vn) * Ay) - mu * Ay / s->dy;
                T aS = (rho * MIN0(-vs) * Ay) - mu * Ay / s->dy;
                T aC = -(aE + aW + aN + aS);
                a[id + N * ORC_AE] = aE;
                a[id + N * ORC_AW] = aW;
                a[id + N * ORC_AN] = aN;
                a[id + N * ORC_AS] = aS;
                if (s->dim == 3) {
                    T wt = wf[WFID(s, i, j, k + 1)], wb = wf[WFID(s, i, j, k)];
                    T aT = (rho * MIN0(wt) * Az) - mu * Az / s->dz;
                    T aB = (rho * MIN0(-wb) * Az) - mu * Az / s->dz;
                    a[id + N * ORC_AT] = aT;
                    a[id + N * ORC_AB] = aB;
                    aC += -(aT + aB);
                }
                a[id + N * ORC_AC] = aC;
            }
}

static int CAT(closed_face_, S)(const ST *s, int face) { return s->cfg.bc_type[face] != ORC_OUTLET; }

/* include/kernels.cuh:136-250 (calcInteriorMomSrcTermKernel and
 * calcBCMomSrcTermKernel): b = 0.5 (p_L - p_R) A.  At a wall or inlet face the
 * face pressure is the cell pressure; at an outlet face it is 0. */
void FN(mom_src)(ST *s)
{
    const T *p = s->f[ORC_F_P];
    T *su = s->f[ORC_F_SRC_U], *sv = s->f[ORC_F_SRC_V], *sw = s->f[ORC_F_SRC_W];
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t id = CID(s, i, j, k);
                T pC = p[id], pL, pR;
                pL = i > 0 ? p[id - 1] : (CAT(closed_face_, S)(s, ORC_WEST) ? pC : (T)0);
                pR = i < s->nx - 1 ? p[id + 1] : (CAT(closed_face_, S)(s, ORC_EAST) ? pC : (T)0);
                su[id] = (T)(0.5 * (double)(T)(pL - pR) * (double)s->Ax);
                pL = j > 0 ? p[id - s->nx] : (CAT(closed_face_, S)(s, ORC_SOUTH) ? pC : (T)0);
                pR = j < s->ny - 1 ? p[id + s->nx] : (CAT(closed_face_, S)(s, ORC_NORTH) ? pC : (T)0);
                sv[id] = (T)(0.5 * (double)(T)(pL - pR) * (double)s->Ay);
                if (s->dim == 3) {
                    size_t pl = (size_t)s->nx * s->ny;
                    pL = k > 0 ? p[id - pl] : (CAT(closed_face_, S)(s, ORC_BOTTOM) ? pC : (T)0);
                    pR = k < s->nz - 1 ? p[id + pl] : (CAT(closed_face_, S)(s, ORC_TOP) ? pC : (T)0);
                    sw[id] = (T)(0.5 * (double)(T)(pL - pR) * (double)s->Az);
                }
            }
}

/* include/kernels.cuh:252-334 (applyBCsToMomEqKernel), faces in the launch
 * order of src/Solver.cu:583-608 (east, west, north, south, top, bottom).
 * Wall/inlet: aC -= 2 aEx; aIn += aEx/3; b -= 8/3 aEx phi_BC; aEx = 0.
 * Outlet: aC += aEx; aEx = 0. */
static void CAT(bc_mom_cell_, S)(ST *s, int face, size_t id, int slot_ex, int slot_in, T ubc, T vbc, T wbc)
{
    T *a = s->f[ORC_F_MCOEF];
    const size_t N = s->N;
    T ex = a[id + N * slot_ex];
    if (s->cfg.bc_type[face] == ORC_OUTLET) {
        a[id + N * ORC_AC] += ex;
        a[id + N * slot_ex] = 0;
        return;
    }
    const T c83 = (T)8 / (T)3;
    a[id + N * ORC_AC] -= (T)2 * ex;
    a[id + N * slot_in] += ex / (T)3;
    s->f[ORC_F_SRC_U][id] -= c83 * ex * ubc;
    s->f[ORC_F_SRC_V][id] -= c83 * ex * vbc;
    if (s->dim == 3) s->f[ORC_F_SRC_W][id] -= c83 * ex * wbc;
    a[id + N * slot_ex] = 0;
}

void FN(bc_mom)(ST *s)
{
    const orc_config *c = &s->cfg;
#define BCV(face, comp) ((T)c->bc_val[face][comp])
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            CAT(bc_mom_cell_, S)(s, ORC_EAST, CID(s, s->nx - 1, j, k), ORC_AE, ORC_AW, BCV(ORC_EAST, 0), BCV(ORC_EAST, 1), BCV(ORC_EAST, 2));
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            CAT(bc_mom_cell_, S)(s, ORC_WEST, CID(s, 0, j, k), ORC_AW, ORC_AE, CAT(west_inlet_, S)(s, j, k), BCV(ORC_WEST, 1), BCV(ORC_WEST, 2));
    for (int k = 0; k < s->nz; ++k)
        for (int i = 0; i < s->nx; ++i)
            CAT(bc_mom_cell_, S)(s, ORC_NORTH, CID(s, i, s->ny - 1, k), ORC_AN, ORC_AS, BCV(ORC_NORTH, 0), BCV(ORC_NORTH, 1), BCV(ORC_NORTH, 2));
    for (int k = 0; k < s->nz; ++k)
        for (int i = 0; i < s->nx; ++i)
            CAT(bc_mom_cell_, S)(s, ORC_SOUTH, CID(s, i, 0, k), ORC_AS, ORC_AN, BCV(ORC_SOUTH, 0), BCV(ORC_SOUTH, 1), BCV(ORC_SOUTH, 2));
    if (s->dim == 3) {
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i)
                CAT(bc_mom_cell_, S)(s, ORC_TOP, CID(s, i, j, s->nz - 1), ORC_AT, ORC_AB, BCV(ORC_TOP, 0), BCV(ORC_TOP, 1), BCV(ORC_TOP, 2));
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i)
                CAT(bc_mom_cell_, S)(s, ORC_BOTTOM, CID(s, i, j, 0), ORC_AB, ORC_AT, BCV(ORC_BOTTOM, 0), BCV(ORC_BOTTOM, 1), BCV(ORC_BOTTOM, 2));
    }
#undef BCV
}

/* Higher-order convection by deferred correction (Khosla & Rubin 1974).  Not in
 * the reference, whose convection is first-order upwind only
 * (include/kernels.cuh:97-134; README.md:412 lists higher-order schemes as
 * planned).  The links stay upwind; the difference between a higher-order face
 * value and the upwind one, times the face's mass flux, enters the source,
 * evaluated with the fields at the start of the outer iteration:
 *   b_C += sum over faces f of -F_f,out (phi_f - phi_U,f).
 * With phi_U the upwind cell, phi_D the downwind cell and phi_UU the cell
 * beyond phi_U, dd = phi_D - phi_U and du = phi_U - phi_UU, the face value is
 * phi_f = phi_U + 0.5 L(du, dd):
 *   central                 L = dd
 *   second-order upwind     L = du
 *   QUICK (Leonard 1979)    L = (3 dd + du) / 4
 *   minmod (Roe 1986)       L = du or dd, the smaller in magnitude, if du dd > 0, else 0
 *   van Leer (1974)         L = 2 du dd / (du + dd) if du dd > 0, else 0
 * Boundary faces, and faces whose far-upwind cell lies outside the domain,
 * keep the upwind value.  Face quantity Q = (rho u_f A) * (0.5 L); a cell's
 * correction is (Q_w - Q_e) + (Q_s - Q_n) [+ (Q_b - Q_t)], added to its source
 * after the boundary fold-in. */
static inline T CAT(dc_limit_, S)(int scheme, T du, T dd)
{
    switch (scheme) {
    case ORC_CONV_CENTRAL: return dd;
    case ORC_CONV_SOU: return du;
    case ORC_CONV_QUICK: return ((T)3 * dd + du) / (T)4;
    case ORC_CONV_MINMOD:
        if (!(du * dd > (T)0)) return (T)0;
        return fabs((double)du) < fabs((double)dd) ? du : dd;
    case ORC_CONV_VAN_LEER:
        if (!(du * dd > (T)0)) return (T)0;
        return (T)2 * du * dd / (du + dd);
    default: return (T)0;
    }
}

/* Q of one interior face between cells L and R along one axis; ll / rr are the
 * cells beyond L and R (has_ll / has_rr: inside the domain). */
static inline T CAT(dc_face_, S)(int scheme, T rho, T uf, T A, T pll, T pl, T pr, T prr, int has_ll, int has_rr)
{
    const T F = rho * uf * A;
    T U, D, UU;
    if (F > (T)0) {
        if (!has_ll) return (T)0;
        U = pl; D = pr; UU = pll;
    } else if (F < (T)0) {
        if (!has_rr) return (T)0;
        U = pr; D = pl; UU = prr;
    } else {
        return (T)0;
    }
    return F * ((T)0.5 * CAT(dc_limit_, S)(scheme, U - UU, D - U));
}

static T CAT(dc_cell_, S)(const ST *s, const T *phi, int i, int j, int k)
{
    const int sc = s->cfg.convection, nx = s->nx, ny = s->ny, nz = s->nz;
    const T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    const T rho = s->rho;
#define PH(a, b, c) phi[CID(s, a, b, c)]
    T qw = (T)0, qe = (T)0, qs = (T)0, qn = (T)0, qb = (T)0, qt = (T)0;
    if (i > 0)
        qw = CAT(dc_face_, S)(sc, rho, uf[UFID(s, i, j, k)], s->Ax, i > 1 ? PH(i - 2, j, k) : (T)0, PH(i - 1, j, k),
                              PH(i, j, k), i < nx - 1 ? PH(i + 1, j, k) : (T)0, i > 1, i < nx - 1);
    if (i < nx - 1)
        qe = CAT(dc_face_, S)(sc, rho, uf[UFID(s, i + 1, j, k)], s->Ax, i > 0 ? PH(i - 1, j, k) : (T)0, PH(i, j, k),
                              PH(i + 1, j, k), i < nx - 2 ? PH(i + 2, j, k) : (T)0, i > 0, i < nx - 2);
    if (j > 0)
        qs = CAT(dc_face_, S)(sc, rho, vf[VFID(s, i, j, k)], s->Ay, j > 1 ? PH(i, j - 2, k) : (T)0, PH(i, j - 1, k),
                              PH(i, j, k), j < ny - 1 ? PH(i, j + 1, k) : (T)0, j > 1, j < ny - 1);
    if (j < ny - 1)
        qn = CAT(dc_face_, S)(sc, rho, vf[VFID(s, i, j + 1, k)], s->Ay, j > 0 ? PH(i, j - 1, k) : (T)0, PH(i, j, k),
                              PH(i, j + 1, k), j < ny - 2 ? PH(i, j + 2, k) : (T)0, j > 0, j < ny - 2);
    T dc = (qw - qe) + (qs - qn);
    if (s->dim == 3) {
        if (k > 0)
            qb = CAT(dc_face_, S)(sc, rho, wf[WFID(s, i, j, k)], s->Az, k > 1 ? PH(i, j, k - 2) : (T)0,
                                  PH(i, j, k - 1), PH(i, j, k), k < nz - 1 ? PH(i, j, k + 1) : (T)0, k > 1, k < nz - 1);
        if (k < nz - 1)
            qt = CAT(dc_face_, S)(sc, rho, wf[WFID(s, i, j, k + 1)], s->Az, k > 0 ? PH(i, j, k - 1) : (T)0,
                                  PH(i, j, k), PH(i, j, k + 1), k < nz - 2 ? PH(i, j, k + 2) : (T)0, k > 0, k < nz - 2);
        dc = dc + (qb - qt);
    }
#undef PH
    return dc;
}

/* Adds the deferred-correction source of every momentum component (u, v, w
 * all at the start-of-iteration fields) to src_u, src_v, src_w. */
void FN(dc_source)(ST *s)
{
    if (s->cfg.convection == ORC_CONV_UPWIND) return;
    const int nc = s->dim;
    const int fphi[3] = {ORC_F_U, ORC_F_V, ORC_F_W}, fsrc[3] = {ORC_F_SRC_U, ORC_F_SRC_V, ORC_F_SRC_W};
    for (int c = 0; c < nc; ++c) {
        T *b = s->f[fsrc[c]];
        for (int k = 0; k < s->nz; ++k)
            for (int j = 0; j < s->ny; ++j)
                for (int i = 0; i < s->nx; ++i) s->tmp[CID(s, i, j, k)] = CAT(dc_cell_, S)(s, s->f[fphi[c]], i, j, k);
        for (size_t id = 0; id < s->N; ++id) b[id] = b[id] + s->tmp[id];
    }
}

/* One relaxed point update, include/kernels.cuh:935-988 (GaussSeidelIterateKernel)
 * and :854-907 (pointJacobiIterateKernel): out-of-domain neighbours are 0,
 * phi_new = (b - sum a_nb phi_nb) / aC, phi += relax (phi_new - phi). */
static inline double CAT(point_update_, S)(const ST *s, const T *src_phi, T *dst_phi, const T *a, const T *b,
                                           int i, int j, int k, T relax)
{
    const size_t N = s->N, id = CID(s, i, j, k), pl = (size_t)s->nx * s->ny;
    T pc = src_phi[id];
    T pE = i != s->nx - 1 ? src_phi[id + 1] : (T)0;
    T pW = i != 0 ? src_phi[id - 1] : (T)0;
    T pN = j != s->ny - 1 ? src_phi[id + s->nx] : (T)0;
    T pS = j != 0 ? src_phi[id - s->nx] : (T)0;
    T np = b[id] - a[id + N * ORC_AE] * pE - a[id + N * ORC_AW] * pW - a[id + N * ORC_AN] * pN - a[id + N * ORC_AS] * pS;
    if (s->dim == 3) {
        T pT = k != s->nz - 1 ? src_phi[id + pl] : (T)0;
        T pB = k != 0 ? src_phi[id - pl] : (T)0;
        np -= a[id + N * ORC_AT] * pT + a[id + N * ORC_AB] * pB;
    }
    np /= a[id + N * ORC_AC];
    T d = relax * (np - pc);
    dst_phi[id] = pc + d;
    return (double)d * (double)d;
}

static void CAT(eq_arrays_, S)(ST *s, int eq, T **phi, T **a, T **b)
{
    switch (eq) {
    case ORC_EQ_U: *phi = s->f[ORC_F_U]; *a = s->f[ORC_F_MCOEF]; *b = s->f[ORC_F_SRC_U]; break;
    case ORC_EQ_V: *phi = s->f[ORC_F_V]; *a = s->f[ORC_F_MCOEF]; *b = s->f[ORC_F_SRC_V]; break;
    case ORC_EQ_W: *phi = s->f[ORC_F_W]; *a = s->f[ORC_F_MCOEF]; *b = s->f[ORC_F_SRC_W]; break;
    default: *phi = s->f[ORC_F_PC]; *a = s->f[ORC_F_PCOEF]; *b = s->f[ORC_F_SRC_P]; break;
    }
}

/* One sweep over all cells in the given ordering; returns sum (d phi)^2 in FP64. */
double FN(sweep)(ST *s, int eq, int mode)
{
    T *phi, *a, *b;
    CAT(eq_arrays_, S)(s, eq, &phi, &a, &b);
    const T relax = s->relax[eq];
    double sq = 0.0;
    if (mode == ORC_JACOBI) {
        memcpy(s->tmp, phi, s->N * sizeof(T));
        for (int k = 0; k < s->nz; ++k)
            for (int j = 0; j < s->ny; ++j)
                for (int i = 0; i < s->nx; ++i)
                    sq += CAT(point_update_, S)(s, s->tmp, phi, a, b, i, j, k, relax);
    } else if (mode == ORC_GS_REDBLACK) {
        for (int color = 0; color < 2; ++color) {
            ORC_PAR_ROWS_SUM
            for (int k = 0; k < s->nz; ++k)
                for (int j = 0; j < s->ny; ++j)
                    for (int i = (color + j + k) & 1; i < s->nx; i += 2)
                        sq += CAT(point_update_, S)(s, phi, phi, a, b, i, j, k, relax);
        }
    } else {
        for (int k = 0; k < s->nz; ++k)
            for (int j = 0; j < s->ny; ++j)
                for (int i = 0; i < s->nx; ++i)
                    sq += CAT(point_update_, S)(s, phi, phi, a, b, i, j, k, relax);
    }
    return sq;
}

/* src/Solver.cu:922-966 (GaussSeidelIterate) and :868-920 (pointJacobiIterate):
 * up to nIter sweeps; after each sweep the RMS change is compared with the
 * largest RMS change of this call and the loop stops once the ratio falls
 * below tol.  check_every > 1 evaluates that rule after blocks of sweeps, the
 * granularity of the temporally blocked device sweeps.  Returns the number of
 * sweeps done; sweep_norms (optional) receives sum (d phi)^2 per sweep. */
int FN(linear_solve)(ST *s, int eq, double *sweep_norms)
{
    const int n = s->cfg.n_iter[eq];
    const int g = s->cfg.check_every > 0 ? s->cfg.check_every : 1;
    double max_norm = -1e20;
    int done = 0, stop = 0;
    while (done < n && !stop) {
        int chunk = n - done < g ? n - done : g;
        for (int c = 0; c < chunk; ++c) {
            double sq = FN(sweep)(s, eq, s->cfg.sweep_mode);
            if (sweep_norms) sweep_norms[done + c] = sq;
            if (stop) continue;
            double nrm = sqrt(sq / (double)s->N);
            if (nrm > max_norm) max_norm = nrm;
            double rel = nrm / (max_norm + 1e-20);
            if (rel < (double)s->tol[eq]) stop = 1;
        }
        done += chunk;
    }
    return done;
}

/* include/kernels.cuh:336-500 (interiorRhieChowInterpolateKernel and
 * bcRhieChowInterpolateKernel): face velocity = linear mean + the
 * pressure-smoothing term.  Faces next to the boundary replace the missing
 * far pressure by the cell pressure (wall/inlet) or 0 (outlet).  Boundary faces
 * themselves are left for the face boundary conditions. */
static T CAT(rc_face_, S)(T uL, T uR, T aCL, T aCR, T pLL, T pL, T pR, T pRR, T A)
{
    double t0 = 0.5 * (double)(T)(uL + uR);
    T t1 = (pR - pLL) * A / ((T)4 * aCL);
    T t2 = (pRR - pL) * A / ((T)4 * aCR);
    T sr = (T)1 / aCL + (T)1 / aCR;
    double t3 = 0.5 * (double)sr * (double)(T)(pL - pR) * (double)A;
    return (T)(t0 + (double)t1 + (double)t2 + t3);
}

void FN(rhie_chow)(ST *s)
{
    const T *u = s->f[ORC_F_U], *v = s->f[ORC_F_V], *w = s->f[ORC_F_W], *p = s->f[ORC_F_P];
    const T *a = s->f[ORC_F_MCOEF]; /* slot aC is the first plane */
    T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    const int cw = CAT(closed_face_, S)(s, ORC_WEST), ce = CAT(closed_face_, S)(s, ORC_EAST);
    const int cs = CAT(closed_face_, S)(s, ORC_SOUTH), cn = CAT(closed_face_, S)(s, ORC_NORTH);
    const int cb = CAT(closed_face_, S)(s, ORC_BOTTOM), ct = CAT(closed_face_, S)(s, ORC_TOP);
    ORC_PAR_ROWS
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 1; i < s->nx; ++i) {
                size_t L = CID(s, i - 1, j, k), R = CID(s, i, j, k);
                T pL = p[L], pR = p[R];
                T pLL = i >= 2 ? p[L - 1] : (cw ? pL : (T)0);
                T pRR = i <= s->nx - 2 ? p[R + 1] : (ce ? pR : (T)0);
                uf[UFID(s, i, j, k)] = CAT(rc_face_, S)(u[L], u[R], a[L], a[R], pLL, pL, pR, pRR, s->Ax);
            }
    ORC_PAR_ROWS
    for (int k = 0; k < s->nz; ++k)
        for (int j = 1; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t L = CID(s, i, j - 1, k), R = CID(s, i, j, k);
                T pL = p[L], pR = p[R];
                T pLL = j >= 2 ? p[L - s->nx] : (cs ? pL : (T)0);
                T pRR = j <= s->ny - 2 ? p[R + s->nx] : (cn ? pR : (T)0);
                vf[VFID(s, i, j, k)] = CAT(rc_face_, S)(v[L], v[R], a[L], a[R], pLL, pL, pR, pRR, s->Ay);
            }
    if (s->dim == 3) {
        size_t pl = (size_t)s->nx * s->ny;
        ORC_PAR_ROWS
        for (int k = 1; k < s->nz; ++k)
            for (int j = 0; j < s->ny; ++j)
                for (int i = 0; i < s->nx; ++i) {
                    size_t L = CID(s, i, j, k - 1), R = CID(s, i, j, k);
                    T pL = p[L], pR = p[R];
                    T pLL = k >= 2 ? p[L - pl] : (cb ? pL : (T)0);
                    T pRR = k <= s->nz - 2 ? p[R + pl] : (ct ? pR : (T)0);
                    wf[WFID(s, i, j, k)] = CAT(rc_face_, S)(w[L], w[R], a[L], a[R], pLL, pL, pR, pRR, s->Az);
                }
    }
}

/* include/kernels.cuh:502-540 (calcPresCorrLinkCoefKernel):
 * a_nb = -0.5 rho A^2 (1/aC_C + 1/aC_nb) on interior faces; boundary links stay
 * 0 (the reference never writes them after the constructor's memset,
 * src/Solver.cu:81), i.e. zero-gradient p' on every boundary. */
void FN(pcorr_link_coef)(ST *s)
{
    const T *m = s->f[ORC_F_MCOEF];
    T *a = s->f[ORC_F_PCOEF];
    const size_t N = s->N, pl = (size_t)s->nx * s->ny;
    const double rho = (double)s->rho;
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t id = CID(s, i, j, k);
                T c = m[id];
                if (i < s->nx - 1) a[id + N * ORC_AE] = (T)(-0.5 * rho * (double)s->Ax * (double)s->Ax * (double)(T)((T)1 / c + (T)1 / m[id + 1]));
                if (i > 0) a[id + N * ORC_AW] = (T)(-0.5 * rho * (double)s->Ax * (double)s->Ax * (double)(T)((T)1 / c + (T)1 / m[id - 1]));
                if (j < s->ny - 1) a[id + N * ORC_AN] = (T)(-0.5 * rho * (double)s->Ay * (double)s->Ay * (double)(T)((T)1 / c + (T)1 / m[id + s->nx]));
                if (j > 0) a[id + N * ORC_AS] = (T)(-0.5 * rho * (double)s->Ay * (double)s->Ay * (double)(T)((T)1 / c + (T)1 / m[id - s->nx]));
                T aC = -(a[id + N * ORC_AE] + a[id + N * ORC_AW] + a[id + N * ORC_AN] + a[id + N * ORC_AS]);
                if (s->dim == 3) {
                    if (k < s->nz - 1) a[id + N * ORC_AT] = (T)(-0.5 * rho * (double)s->Az * (double)s->Az * (double)(T)((T)1 / c + (T)1 / m[id + pl]));
                    if (k > 0) a[id + N * ORC_AB] = (T)(-0.5 * rho * (double)s->Az * (double)s->Az * (double)(T)((T)1 / c + (T)1 / m[id - pl]));
                    aC += -(a[id + N * ORC_AT] + a[id + N * ORC_AB]);
                }
                a[id + N * ORC_AC] = aC;
            }
}

/* include/kernels.cuh:542-581 (calcPresCorrSrcTermKernel): mass imbalance
 * b = rho (Ax (uf_w - uf_e) + Ay (vf_s - vf_n) [+ Az (wf_b - wf_t)]).
 * Returns sum b^2 in FP64 (the reference accumulates it in float). */
double FN(pcorr_src)(ST *s)
{
    const T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    T *b = s->f[ORC_F_SRC_P];
    double sq = 0.0;
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t id = CID(s, i, j, k);
                T bb = s->rho * (s->Ax * (uf[UFID(s, i, j, k)] - uf[UFID(s, i + 1, j, k)]) +
                                 s->Ay * (vf[VFID(s, i, j, k)] - vf[VFID(s, i, j + 1, k)]));
                if (s->dim == 3) bb += s->rho * s->Az * (wf[WFID(s, i, j, k)] - wf[WFID(s, i, j, k + 1)]);
                b[id] = bb;
                sq += (double)bb * (double)bb;
            }
    return sq;
}

/* Pressure-reference pinning (new-build addition for closed domains): remove
 * the FP64 mean of p' so that the pure-Neumann p' problem cannot drift. */
void FN(pin_pcorr)(ST *s)
{
    T *pc = s->f[ORC_F_PC];
    double sum = 0.0;
    for (size_t q = 0; q < s->N; ++q) sum += (double)pc[q];
    double mean = sum / (double)s->N;
    for (size_t q = 0; q < s->N; ++q) pc[q] = (T)((double)pc[q] - mean);
}

/* include/kernels.cuh:583-843 (updateInteriorVelKernel, updateBCVelKernel,
 * updateFaceVelKernel, updatePresKernel) as launched by src/Solver.cu:739-866:
 * p += relax_p p'; u += relax_u 0.5 (p'_L - p'_R) A / aC; interior faces
 * uf += relax_u 0.5 (1/aC_L + 1/aC_R) (p'_L - p'_R) A.  Sums of squared
 * changes go to out (FP64). */
void FN(update_field)(ST *s, orc_norms *out)
{
    const T *pc = s->f[ORC_F_PC], *m = s->f[ORC_F_MCOEF];
    T *p = s->f[ORC_F_P], *u = s->f[ORC_F_U], *v = s->f[ORC_F_V], *w = s->f[ORC_F_W];
    T *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF], *wf = s->f[ORC_F_WF];
    const size_t pl = (size_t)s->nx * s->ny;
    double sp = 0, su = 0, sv = 0, sw = 0, suf = 0, svf = 0, swf = 0;
    const int cw = CAT(closed_face_, S)(s, ORC_WEST), ce = CAT(closed_face_, S)(s, ORC_EAST);
    const int cs = CAT(closed_face_, S)(s, ORC_SOUTH), cn = CAT(closed_face_, S)(s, ORC_NORTH);
    const int cb = CAT(closed_face_, S)(s, ORC_BOTTOM), ct = CAT(closed_face_, S)(s, ORC_TOP);
    const double ru = (double)s->relax[ORC_EQ_U] * 0.5, rv = (double)s->relax[ORC_EQ_V] * 0.5;
    const double rw = (double)s->relax[ORC_EQ_W] * 0.5;
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t id = CID(s, i, j, k);
                T dp = s->relax[ORC_EQ_P] * pc[id];
                p[id] += dp;
                sp += (double)dp * (double)dp;
                T c = pc[id], aC = m[id], L, R, d;
                L = i > 0 ? pc[id - 1] : (cw ? c : (T)0);
                R = i < s->nx - 1 ? pc[id + 1] : (ce ? c : (T)0);
                d = (T)(ru * (double)(T)(L - R) * (double)s->Ax / (double)aC);
                u[id] += d;
                su += (double)d * (double)d;
                L = j > 0 ? pc[id - s->nx] : (cs ? c : (T)0);
                R = j < s->ny - 1 ? pc[id + s->nx] : (cn ? c : (T)0);
                d = (T)(rv * (double)(T)(L - R) * (double)s->Ay / (double)aC);
                v[id] += d;
                sv += (double)d * (double)d;
                if (s->dim == 3) {
                    L = k > 0 ? pc[id - pl] : (cb ? c : (T)0);
                    R = k < s->nz - 1 ? pc[id + pl] : (ct ? c : (T)0);
                    d = (T)(rw * (double)(T)(L - R) * (double)s->Az / (double)aC);
                    w[id] += d;
                    sw += (double)d * (double)d;
                }
            }
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 1; i < s->nx; ++i) {
                size_t L = CID(s, i - 1, j, k), R = CID(s, i, j, k);
                T sr = (T)1 / m[L] + (T)1 / m[R];
                T d = (T)(ru * (double)sr * (double)(T)(pc[L] - pc[R]) * (double)s->Ax);
                uf[UFID(s, i, j, k)] += d;
                suf += (double)d * (double)d;
            }
    for (int k = 0; k < s->nz; ++k)
        for (int j = 1; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                size_t L = CID(s, i, j - 1, k), R = CID(s, i, j, k);
                T sr = (T)1 / m[L] + (T)1 / m[R];
                T d = (T)(rv * (double)sr * (double)(T)(pc[L] - pc[R]) * (double)s->Ay);
                vf[VFID(s, i, j, k)] += d;
                svf += (double)d * (double)d;
            }
    if (s->dim == 3)
        for (int k = 1; k < s->nz; ++k)
            for (int j = 0; j < s->ny; ++j)
                for (int i = 0; i < s->nx; ++i) {
                    size_t L = CID(s, i, j, k - 1), R = CID(s, i, j, k);
                    T sr = (T)1 / m[L] + (T)1 / m[R];
                    T d = (T)(rw * (double)sr * (double)(T)(pc[L] - pc[R]) * (double)s->Az);
                    wf[WFID(s, i, j, k)] += d;
                    swf += (double)d * (double)d;
                }
    if (out) {
        out->p = sp; out->u = su; out->v = sv; out->w = sw;
        out->uf = suf; out->vf = svf; out->wf = swf;
    }
}

/* Sum of squares, in FP64, of the residual b - aC phi - sum a_nb phi_nb of
 * the assembled momentum equation of component `eq` at the current field
 * (out-of-domain neighbours enter as 0, as in the sweeps).  A library
 * addition: the reference measures convergence by its corrections only. */
static double FN(mom_residual_sq)(ST *s, int eq)
{
    const T *a = s->f[ORC_F_MCOEF];
    const T *b = s->f[eq == ORC_EQ_U ? ORC_F_SRC_U : eq == ORC_EQ_V ? ORC_F_SRC_V : ORC_F_SRC_W];
    const T *x = s->f[eq == ORC_EQ_U ? ORC_F_U : eq == ORC_EQ_V ? ORC_F_V : ORC_F_W];
    const size_t N = s->N;
    double sum = 0.0;
    for (int k = 0; k < s->nz; ++k)
        for (int j = 0; j < s->ny; ++j)
            for (int i = 0; i < s->nx; ++i) {
                const size_t c = CID(s, i, j, k);
                double r = (double)b[c] - (double)a[c + N * ORC_AC] * (double)x[c];
                if (i < s->nx - 1) r -= (double)a[c + N * ORC_AE] * (double)x[c + 1];
                if (i > 0) r -= (double)a[c + N * ORC_AW] * (double)x[c - 1];
                if (j < s->ny - 1) r -= (double)a[c + N * ORC_AN] * (double)x[c + s->nx];
                if (j > 0) r -= (double)a[c + N * ORC_AS] * (double)x[c - s->nx];
                if (s->dim == 3) {
                    const size_t pl = (size_t)s->nx * s->ny;
                    if (k < s->nz - 1) r -= (double)a[c + N * ORC_AT] * (double)x[c + pl];
                    if (k > 0) r -= (double)a[c + N * ORC_AB] * (double)x[c - pl];
                }
                sum += r * r;
            }
    return sum;
}

/* One SIMPLE outer iteration, src/Solver.cu:160-289, followed by the norms and
 * the convergence test.  Returns 1 when converged. */
int FN(outer_iteration)(ST *s, orc_norms *out)
{
    orc_norms nm;
    memset(&nm, 0, sizeof(nm));
    if (s->it == 0) FN(init_face_vel)(s);
    FN(bc_face_vel)(s);
    FN(mom_link_coef)(s);
    FN(mom_src)(s);
    FN(bc_mom)(s);
    FN(dc_source)(s);
    if (s->cfg.criterion == ORC_CRIT_RESIDUAL) {
        nm.res_u = sqrt(FN(mom_residual_sq)(s, ORC_EQ_U) / (double)s->N);
        nm.res_v = sqrt(FN(mom_residual_sq)(s, ORC_EQ_V) / (double)s->N);
        if (s->dim == 3) nm.res_w = sqrt(FN(mom_residual_sq)(s, ORC_EQ_W) / (double)s->N);
    }
    nm.sweeps[ORC_EQ_U] = FN(linear_solve)(s, ORC_EQ_U, NULL);
    nm.sweeps[ORC_EQ_V] = FN(linear_solve)(s, ORC_EQ_V, NULL);
    if (s->dim == 3) nm.sweeps[ORC_EQ_W] = FN(linear_solve)(s, ORC_EQ_W, NULL);
    FN(rhie_chow)(s);
    FN(bc_face_vel)(s);
    FN(pcorr_link_coef)(s);
    double mass = FN(pcorr_src)(s);
    memset(s->f[ORC_F_PC], 0, s->N * sizeof(T));
    nm.sweeps[ORC_EQ_P] = FN(linear_solve)(s, ORC_EQ_P, NULL);
    if (s->cfg.pin_pressure) FN(pin_pcorr)(s);
    FN(update_field)(s, &nm);

    /* src/Solver.cu:226-235 */
    const double N = (double)s->N;
    nm.p = sqrt(nm.p / N);
    nm.u = sqrt(nm.u / N);
    nm.v = sqrt(nm.v / N);
    nm.uf = sqrt(nm.uf / ((double)(s->nx - 1) * s->ny * s->nz));
    nm.vf = sqrt(nm.vf / ((double)s->nx * (s->ny - 1) * s->nz));
    nm.mass = sqrt(mass / N);
    if (s->dim == 3) {
        nm.w = sqrt(nm.w / N);
        nm.wf = sqrt(nm.wf / ((double)s->nx * s->ny * (s->nz - 1)));
    }
    if (s->cfg.criterion == ORC_CRIT_REFERENCE) {
        /* src/Solver.cu:237-256: every relative norm is divided by the running
         * maximum of the pressure norm (defect D6, kept for parity). */
        if (nm.p > s->max_p) s->max_p = nm.p;
        double mx = s->max_p;
        nm.rel_p = nm.p / mx; nm.rel_u = nm.u / mx; nm.rel_v = nm.v / mx;
        nm.rel_uf = nm.uf / mx; nm.rel_vf = nm.vf / mx;
        nm.rel_w = nm.w / mx; nm.rel_wf = nm.wf / mx;
    } else if (s->cfg.criterion == ORC_CRIT_PER_FIELD) {
#define RELF(x) do { if (nm.x > s->max_##x) s->max_##x = nm.x; nm.rel_##x = s->max_##x > 0 ? nm.x / s->max_##x : 0.0; } while (0)
        RELF(p); RELF(u); RELF(v); RELF(uf); RELF(vf);
        if (s->dim == 3) { RELF(w); RELF(wf); }
#undef RELF
    } else {
        /* Per field on the FP64 residuals: u, v, w by their momentum residual,
         * p by the mass imbalance, each over its own running maximum; the
         * face velocities follow from u and p and are not tested. */
        const double r[4] = {nm.res_u, nm.res_v, nm.res_w, nm.mass};
        double rel[4];
        for (int q = 0; q < 4; ++q) {
            if (r[q] > s->rmax[q]) s->rmax[q] = r[q];
            rel[q] = s->rmax[q] > 0 ? r[q] / s->rmax[q] : 0.0;
        }
        nm.rel_u = rel[0]; nm.rel_v = rel[1]; nm.rel_w = s->dim == 3 ? rel[2] : 0.0; nm.rel_p = rel[3];
        nm.rel_uf = nm.rel_vf = nm.rel_wf = 0.0;
    }
    /* src/Solver.cu:258-268 */
    int conv = nm.rel_p < (double)s->tol[ORC_EQ_P] && nm.rel_u < (double)s->tol[ORC_EQ_U] &&
               nm.rel_v < (double)s->tol[ORC_EQ_V] && nm.rel_uf < (double)s->tol[ORC_EQ_U] &&
               nm.rel_vf < (double)s->tol[ORC_EQ_V];
    if (s->dim == 3) conv = conv && nm.rel_w < (double)s->tol[ORC_EQ_W] && nm.rel_wf < (double)s->tol[ORC_EQ_W];
    conv = conv || nm.mass < (double)(T)s->cfg.tol_mass;
    nm.converged = conv;
    s->it++;
    if (out) *out = nm;
    return conv;
}

/* src/Solver.cu:153-299 (Solver::solve) without the final host copies: up to
 * max_outer further outer iterations (num_outer_iter when max_outer <= 0),
 * stopping at convergence.  Returns the iterations done by this call. */
int FN(solve)(ST *s, int max_outer, orc_norms *last)
{
    int n = max_outer > 0 ? max_outer : s->cfg.num_outer_iter;
    orc_norms nm;
    memset(&nm, 0, sizeof(nm));
    int done = 0;
    for (; done < n;) {
        int conv = FN(outer_iteration)(s, &nm);
        ++done;
        if (conv) break;
    }
    if (last) *last = nm;
    return done;
}

#undef MIN0
#undef ST
#undef FN
#undef CAT
#undef CAT_
