/*
 * ifc_adjoint_impl.h -- reverse pass of one SIMPLE outer iteration at its
 * fixed point, FP64, 2D (TEST INFRASTRUCTURE ONLY; included by ifc_oracle.c
 * after the double instantiation).
 *
 * The persistent state of an outer iteration is x = (u, v, p, interior uf,
 * interior vf); one iteration is x -> G(x, theta, mu) (src/Solver.cu:160-198
 * with the corrections of :739-866), theta being the west-inlet velocity of
 * each boundary row.  At a fixed point every Gauss-Seidel iterate of the
 * momentum solve equals the converged field and p' is 0 in every p' sweep, so
 * the transposed steps need no stored history:
 *   corrections^T -> [p' mean removal]^T -> p' sweeps^T (red-black order
 *   reversed) -> p' source^T -> Rhie-Chow + face BCs^T -> momentum sweeps^T
 *   (accumulating the adjoint of the shared coefficients and sources) ->
 *   boundary fold-in^T (faces in reverse launch order) -> pressure source^T ->
 *   link coefficients^T (upwind derivative [u_f < 0], viscosity) -> face
 *   BCs^T.
 * orc_adjoint_apply_d returns G_x^T lambda, G_theta^T lambda and G_mu^T lambda
 * for a seed lambda on G's outputs.  The inner early exit of the sweeps is
 * taken as not firing (full sweep counts), which holds at convergence.
 */

#define AD(s, i, j) ((size_t)(i) + (size_t)(s)->nx * (size_t)(j))

typedef orc_state_d AS;

/* One transposed red-black half sweep over the cells of `color`.
 * forward: phi_X <- (1-alpha) phi_X + alpha (b_X - sum_nb a_X,nb phi_nb) / aC_X
 * reverse: lb_X += alpha/aC_X l_X; l_nb += -alpha a_X,nb/aC_X l_X;
 *          la_X,nb += -alpha phi_nb/aC_X l_X; la_X,C += -alpha phi_X/aC_X l_X;
 *          l_X <- (1-alpha) l_X, with l_X the adjoint of the half sweep's output. */
static void adj_half(const AS *s, int color, const double *a, double alpha, const double *phi, double *lam,
                     double *lb, double *la)
{
    const size_t N = s->N;
    const int nx = s->nx, ny = s->ny;
    for (int j = 0; j < ny; ++j)
        for (int i = (color + j) & 1; i < nx; i += 2) {
            const size_t c = AD(s, i, j);
            const double l = lam[c];
            const double aC = a[c + N * ORC_AC];
            const double g = alpha / aC * l;
            if (lb) lb[c] += g;
            const int nb_ok[4] = {i < nx - 1, i > 0, j < ny - 1, j > 0};
            const long off[4] = {1, -1, nx, -nx};
            const int slot[4] = {ORC_AE, ORC_AW, ORC_AN, ORC_AS};
            for (int q = 0; q < 4; ++q) {
                if (!nb_ok[q]) continue;
                const size_t nb = (size_t)((long)c + off[q]);
                lam[nb] += -a[c + N * slot[q]] * g;
                if (la && phi) la[c + N * slot[q]] += -phi[nb] * g;
            }
            if (la && phi) la[c + N * ORC_AC] += -phi[c] * g;
            lam[c] = (1.0 - alpha) * l;
        }
}

/* Cell index of a pressure-like neighbour with the reference's boundary rule
 * (kernels.cuh:232-246): inside the domain the neighbour, at a wall or inlet
 * face the cell itself, at an outlet face nothing (value 0). */
static long nb_or_self(const AS *s, long c, int inside, long nb, int closed)
{
    (void)s;
    if (inside) return nb;
    return closed ? c : -1;
}

static void add_if(double *x, long idx, double v)
{
    if (idx >= 0) x[idx] += v;
}

int orc_adjoint_apply_d(AS *s, const double *lu_in, const double *lv_in, const double *lp_in, const double *luf_in,
                        const double *lvf_in, double *lu_out, double *lv_out, double *lp_out, double *luf_out,
                        double *lvf_out, double *ltheta, double *lmu)
{
    if (s->dim != 2) return -1;
    const int nx = s->nx, ny = s->ny;
    const size_t N = s->N, NU = (size_t)(nx + 1) * ny, NV = (size_t)nx * (ny + 1);
    const orc_config *cf = &s->cfg;
    const int cw = cf->bc_type[ORC_WEST] != ORC_OUTLET, ce = cf->bc_type[ORC_EAST] != ORC_OUTLET;
    const int cs = cf->bc_type[ORC_SOUTH] != ORC_OUTLET, cn = cf->bc_type[ORC_NORTH] != ORC_OUTLET;
    const double Ax = s->Ax, Ay = s->Ay, rho = s->rho;
    const double *u = s->f[ORC_F_U], *v = s->f[ORC_F_V], *p = s->f[ORC_F_P];

    /* Intermediate quantities of the forward iteration at this state. */
    orc_bc_face_vel_d(s);
    orc_mom_link_coef_d(s);
    double *a_raw = (double *)malloc(N * 5 * sizeof(double));
    memcpy(a_raw, s->f[ORC_F_MCOEF], N * 5 * sizeof(double));
    orc_mom_src_d(s);
    orc_bc_mom_d(s);
    const double *a = s->f[ORC_F_MCOEF];
    orc_pcorr_link_coef_d(s);
    const double *ap = s->f[ORC_F_PCOEF];
    const double *uf = s->f[ORC_F_UF], *vf = s->f[ORC_F_VF];

    double *lpc = calloc(N, sizeof(double)), *lbp = calloc(N, sizeof(double));
    double *lus = calloc(N, sizeof(double)), *lvs = calloc(N, sizeof(double));
    double *lufs = calloc(NU, sizeof(double)), *lvfs = calloc(NV, sizeof(double));
    double *la = calloc(N * 5, sizeof(double)), *lbu = calloc(N, sizeof(double)), *lbv = calloc(N, sizeof(double));
    double *lufa = calloc(NU, sizeof(double)), *lvfa = calloc(NV, sizeof(double));
    for (int j = 0; j < ny; ++j) ltheta[j] = 0.0;
    *lmu = 0.0;
    memset(lu_out, 0, N * sizeof(double));
    memset(lv_out, 0, N * sizeof(double));
    memset(lp_out, 0, N * sizeof(double));
    memset(luf_out, 0, NU * sizeof(double));
    memset(lvf_out, 0, NV * sizeof(double));

    /* corrections^T (kernels.cuh:583-843) */
    const double ru = (double)cf->relax[ORC_EQ_U] * 0.5, rv = (double)cf->relax[ORC_EQ_V] * 0.5;
    const double ap_ = cf->relax[ORC_EQ_P];
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const long c = (long)AD(s, i, j);
            lp_out[c] += lp_in[c];
            lpc[c] += ap_ * lp_in[c];
            lus[c] += lu_in[c];
            lvs[c] += lv_in[c];
            const double aC = a[c];
            const double ku = ru * Ax / aC, kv = rv * Ay / aC;
            add_if(lpc, nb_or_self(s, c, i > 0, c - 1, cw), ku * lu_in[c]);
            add_if(lpc, nb_or_self(s, c, i < nx - 1, c + 1, ce), -ku * lu_in[c]);
            add_if(lpc, nb_or_self(s, c, j > 0, c - nx, cs), kv * lv_in[c]);
            add_if(lpc, nb_or_self(s, c, j < ny - 1, c + nx, cn), -kv * lv_in[c]);
        }
    for (int j = 0; j < ny; ++j)
        for (int i = 1; i < nx; ++i) {
            const size_t f = (size_t)i + (size_t)(nx + 1) * j, L = AD(s, i - 1, j), R = AD(s, i, j);
            lufs[f] += luf_in[f];
            const double m = ru * (1.0 / a[L] + 1.0 / a[R]) * Ax;
            lpc[L] += m * luf_in[f];
            lpc[R] -= m * luf_in[f];
        }
    for (int j = 1; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t f = AD(s, i, j), L = AD(s, i, j - 1), R = AD(s, i, j);
            lvfs[f] += lvf_in[f];
            const double m = rv * (1.0 / a[L] + 1.0 / a[R]) * Ay;
            lpc[L] += m * lvf_in[f];
            lpc[R] -= m * lvf_in[f];
        }
    /* p' mean removal^T */
    if (cf->pin_pressure) {
        double sum = 0.0;
        for (size_t q = 0; q < N; ++q) sum += lpc[q];
        for (size_t q = 0; q < N; ++q) lpc[q] -= sum / (double)N;
    }
    /* p' sweeps^T (p' = 0 throughout at the fixed point) */
    for (int sw = cf->n_iter[ORC_EQ_P] - 1; sw >= 0; --sw) {
        adj_half(s, 1, ap, ap_, NULL, lpc, lbp, NULL);
        adj_half(s, 0, ap, ap_, NULL, lpc, lbp, NULL);
    }
    /* p' source^T (kernels.cuh:558-563) */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) {
            const size_t f = (size_t)i + (size_t)(nx + 1) * j;
            double g = 0.0;
            if (i < nx) g += lbp[AD(s, i, j)];
            if (i > 0) g -= lbp[AD(s, i - 1, j)];
            lufs[f] += rho * Ax * g;
        }
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t f = AD(s, i, j);
            double g = 0.0;
            if (j < ny) g += lbp[AD(s, i, j)];
            if (j > 0) g -= lbp[AD(s, i, j - 1)];
            lvfs[f] += rho * Ay * g;
        }
    /* face BCs on u*, v*^T (kernels.cuh:87-93) */
    double *lac = calloc(N, sizeof(double));
    for (int j = 0; j < ny; ++j) {
        const size_t f0 = (size_t)(nx + 1) * j, f1 = f0 + nx;
        if (cf->bc_type[ORC_WEST] == ORC_INLET && cf->inlet_profile) ltheta[j] += lufs[f0];
        if (cf->bc_type[ORC_WEST] == ORC_OUTLET) lus[AD(s, 0, j)] += lufs[f0];
        if (cf->bc_type[ORC_EAST] == ORC_OUTLET) lus[AD(s, nx - 1, j)] += lufs[f1];
    }
    for (int i = 0; i < nx; ++i) {
        if (cf->bc_type[ORC_SOUTH] == ORC_OUTLET) lvs[AD(s, i, 0)] += lvfs[AD(s, i, 0)];
        if (cf->bc_type[ORC_NORTH] == ORC_OUTLET) lvs[AD(s, i, ny - 1)] += lvfs[AD(s, i, ny)];
    }
    /* Rhie-Chow^T on interior faces (kernels.cuh:394-395, 497-498) */
    for (int dir = 0; dir < 2; ++dir) {
        const int nfi = dir == 0 ? nx : ny;       /* faces 1..nfi-1 along the direction */
        const int nfo = dir == 0 ? ny : nx;       /* rows across */
        const double A = dir == 0 ? Ax : Ay;
        const int clo = dir == 0 ? cw : cs, chi = dir == 0 ? ce : cn;
        const long step = dir == 0 ? 1 : nx;
        for (int o = 0; o < nfo; ++o)
            for (int k = 1; k < nfi; ++k) {
                long L, R;
                double l;
                if (dir == 0) {
                    L = (long)AD(s, k - 1, o);
                    R = (long)AD(s, k, o);
                    l = lufs[(size_t)k + (size_t)(nx + 1) * o];
                } else {
                    L = (long)AD(s, o, k - 1);
                    R = (long)AD(s, o, k);
                    l = lvfs[AD(s, o, k)];
                }
                if (l == 0.0) continue;
                const double aL = a[L], aR = a[R];
                const double cL = A / (4.0 * aL), cR = A / (4.0 * aR), h = 0.5 * (1.0 / aL + 1.0 / aR) * A;
                const long LL = nb_or_self(s, L, k >= 2, L - step, clo);
                const long RR = nb_or_self(s, R, k <= nfi - 2, R + step, chi);
                double *lph = dir == 0 ? lus : lvs;
                lph[L] += 0.5 * l;
                lph[R] += 0.5 * l;
                const double pL = p[L], pR = p[R];
                const double pLL = LL >= 0 ? p[LL] : 0.0, pRR = RR >= 0 ? p[RR] : 0.0;
                lp_out[R] += (cL - h) * l;
                add_if(lp_out, LL, -cL * l);
                add_if(lp_out, RR, cR * l);
                lp_out[L] += (-cR + h) * l;
                lac[L] += (-(pR - pLL) * A / (4.0 * aL * aL) - 0.5 * (pL - pR) * A / (aL * aL)) * l;
                lac[R] += (-(pRR - pL) * A / (4.0 * aR * aR) - 0.5 * (pL - pR) * A / (aR * aR)) * l;
            }
    }
    /* momentum sweeps^T: u then v share the coefficients (kernels.cuh:926-1005) */
    for (int sw = cf->n_iter[ORC_EQ_U] - 1; sw >= 0; --sw) {
        adj_half(s, 1, a, cf->relax[ORC_EQ_U], u, lus, lbu, la);
        adj_half(s, 0, a, cf->relax[ORC_EQ_U], u, lus, lbu, la);
    }
    for (int sw = cf->n_iter[ORC_EQ_V] - 1; sw >= 0; --sw) {
        adj_half(s, 1, a, cf->relax[ORC_EQ_V], v, lvs, lbv, la);
        adj_half(s, 0, a, cf->relax[ORC_EQ_V], v, lvs, lbv, la);
    }
    for (size_t c = 0; c < N; ++c) {
        lu_out[c] += lus[c];
        lv_out[c] += lvs[c];
        la[c + N * ORC_AC] += lac[c];
    }
    /* boundary fold-in^T, faces in reverse launch order (kernels.cuh:304-331) */
    const int faces[4] = {ORC_SOUTH, ORC_NORTH, ORC_WEST, ORC_EAST};
    const double c83 = 8.0 / 3.0;
    for (int q = 0; q < 4; ++q) {
        const int F = faces[q];
        const int ex = F == ORC_EAST ? ORC_AE : F == ORC_WEST ? ORC_AW : F == ORC_NORTH ? ORC_AN : ORC_AS;
        const int in = F == ORC_EAST ? ORC_AW : F == ORC_WEST ? ORC_AE : F == ORC_NORTH ? ORC_AS : ORC_AN;
        const int cnt = (F == ORC_EAST || F == ORC_WEST) ? ny : nx;
        for (int t = 0; t < cnt; ++t) {
            const size_t c = F == ORC_EAST ? AD(s, nx - 1, t) : F == ORC_WEST ? AD(s, 0, t)
                                                                              : F == ORC_NORTH ? AD(s, t, ny - 1)
                                                                                               : AD(s, t, 0);
            const double exv = a_raw[c + N * ex];
            if (cf->bc_type[F] == ORC_OUTLET) {
                la[c + N * ex] = la[c + N * ORC_AC];
                continue;
            }
            double ubc = cf->bc_val[F][0], vbc = cf->bc_val[F][1];
            const int prof = F == ORC_WEST && cf->bc_type[F] == ORC_INLET && cf->inlet_profile;
            if (prof) ubc = cf->inlet_profile[t];
            la[c + N * ex] = -2.0 * la[c + N * ORC_AC] + la[c + N * in] / 3.0 - c83 * ubc * lbu[c] - c83 * vbc * lbv[c];
            if (prof) ltheta[t] += -c83 * exv * lbu[c];
        }
    }
    /* pressure source^T (kernels.cuh:136-250) */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const long c = (long)AD(s, i, j);
            add_if(lp_out, nb_or_self(s, c, i > 0, c - 1, cw), 0.5 * Ax * lbu[c]);
            add_if(lp_out, nb_or_self(s, c, i < nx - 1, c + 1, ce), -0.5 * Ax * lbu[c]);
            add_if(lp_out, nb_or_self(s, c, j > 0, c - nx, cs), 0.5 * Ay * lbv[c]);
            add_if(lp_out, nb_or_self(s, c, j < ny - 1, c + nx, cn), -0.5 * Ay * lbv[c]);
        }
    /* link coefficients^T (kernels.cuh:116-120) */
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const size_t c = AD(s, i, j);
            const double tC = la[c + N * ORC_AC];
            const double tE = la[c + N * ORC_AE] - tC, tW = la[c + N * ORC_AW] - tC;
            const double tN = la[c + N * ORC_AN] - tC, tS = la[c + N * ORC_AS] - tC;
            const size_t fe = (size_t)(i + 1) + (size_t)(nx + 1) * j, fw = fe - 1;
            const size_t fn = AD(s, i, j + 1), fs = AD(s, i, j);
            if (uf[fe] < 0) lufa[fe] += tE * rho * Ax;
            if (uf[fw] > 0) lufa[fw] += -tW * rho * Ax;
            if (vf[fn] < 0) lvfa[fn] += tN * rho * Ay;
            if (vf[fs] > 0) lvfa[fs] += -tS * rho * Ay;
            *lmu += -(tE + tW) * Ax / s->dx - (tN + tS) * Ay / s->dy;
        }
    /* face BCs at the start of the iteration^T */
    for (int j = 0; j < ny; ++j) {
        const size_t f0 = (size_t)(nx + 1) * j, f1 = f0 + nx;
        if (cf->bc_type[ORC_WEST] == ORC_INLET && cf->inlet_profile) ltheta[j] += lufa[f0];
        if (cf->bc_type[ORC_WEST] == ORC_OUTLET) lu_out[AD(s, 0, j)] += lufa[f0];
        if (cf->bc_type[ORC_EAST] == ORC_OUTLET) lu_out[AD(s, nx - 1, j)] += lufa[f1];
        for (int i = 1; i < nx; ++i) luf_out[(size_t)i + (size_t)(nx + 1) * j] += lufa[(size_t)i + (size_t)(nx + 1) * j];
    }
    for (int i = 0; i < nx; ++i) {
        if (cf->bc_type[ORC_SOUTH] == ORC_OUTLET) lv_out[AD(s, i, 0)] += lvfa[AD(s, i, 0)];
        if (cf->bc_type[ORC_NORTH] == ORC_OUTLET) lv_out[AD(s, i, ny - 1)] += lvfa[AD(s, i, ny)];
        for (int j = 1; j < ny; ++j) lvf_out[AD(s, i, j)] += lvfa[AD(s, i, j)];
    }
    free(a_raw); free(lpc); free(lbp); free(lus); free(lvs); free(lufs); free(lvfs);
    free(la); free(lbu); free(lbv); free(lufa); free(lvfa); free(lac);
    return 0;
}

#undef AD
