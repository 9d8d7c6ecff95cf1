// ifc_batch_tb.cuh -- temporally blocked form of the batched kernel (included
// by ifc_batch.cu inside its anonymous namespace, after the case queue, loop
// state and cluster-reduction helpers).
//
// A cluster of kCL CTAs solves one case at a time, as k_batch2d does, but the
// linear sweeps run as temporally blocked passes, the same passes as the
// single-case solve (ifc_persist2d.cuh): the case is cut into TX x TY tiles,
// the cluster's CTAs take the tiles in turn, and each tile is staged with a
// halo of 2*KS cells in shared memory, swept KS times there (momentum: u and v
// together, coefficients rebuilt on the fly; p': links from 1/aC) and written
// back -- to the other buffer of a ping-pong pair, so no tile reads a
// neighbour tile's values of the same pass.  Cluster barriers separate the
// passes and phases; every norm is reduced per CTA in warp order and across
// the cluster through distributed shared memory in rank order, so each CTA
// takes the same early-exit and convergence decisions.  Tile shape and sweeps
// per pass are template parameters; the batch autotuner picks them per size
// class.

template <typename T>
struct TBPools {
    T *tu, *tv, *tpc;  // ping-pong partners of u, v and p' (same offsets as the pools)
};

template <int NV, int NT>
__device__ __forceinline__ void tb_block_sum(const double (&v)[NV], double *part)
{
    __shared__ double red[NT / 32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < NV; ++r) {
        const double t = warp_sum(v[r]);
        if (lane == 0) red[warp][r] = t;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = 0.0;
        for (int w = 0; w < NT / 32; ++w) t += red[w][threadIdx.x];
        part[threadIdx.x] = t;
    }
}

// Inner early-exit rule (src/Solver.cu:955-962) after a pass of ns sweeps with
// per-sweep sums sq[0..ns).
__device__ __forceinline__ void tb_pass_done(CaseLoop &L, int e, const double *sq, int ns, int N, double tol)
{
    double mx = L.inner_max[e];
    bool stop_now = false;
    for (int s = 0; s < ns && !stop_now; ++s) {
        const double rms = sqrt(sq[s] / (double)N);
        if (rms > mx) mx = rms;
        if (rms / (mx + 1e-20) < tol) stop_now = true;
    }
    L.inner_max[e] = mx;
    L.sweeps[e] += ns;
    if (stop_now) L.stop[e] = 1;
}

template <typename T, int TX, int TY, int KS, int NT>
__global__ void __cluster_dims__(kCL, 1, 1) __launch_bounds__(NT)
    k_batch_tb(const BCase<T> *cases, BState *states, BPools<T> pool, TBPools<T> tp, int ncases, BQueue *q,
               int chunk, cudaGraphConditionalHandle cond, int use_cond)
{
    constexpr int H = 2 * KS;
    using R = Region<TX, TY, H>;
    constexpr int W = R::W, NR = R::NR;
    constexpr int CPT = (R::NHALF + NT - 1) / NT;
    constexpr int NP = 2 * KS + 8;  // partial-sum slots per set
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int tid = threadIdx.x, lane = tid & 31;
    const int gw = (int)rank * (NT / 32) + (tid >> 5);  // warp index within the cluster
    constexpr int TW = kCL * NT / 32;                   // warps per cluster

    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *s0 = reinterpret_cast<T *>(smem_raw);
    T *s1 = s0 + NR;
    T *s2 = s1 + NR;
    __shared__ int s_case;
    __shared__ BCase<T> C;
    __shared__ CaseLoop L;
    __shared__ BState S;
    // Two sets of this CTA's partial sums, used alternately: a set is rewritten
    // only after a later cluster barrier that every CTA reaches after reading it.
    __shared__ double part[2][NP];
    __shared__ double tot[NP];
    int rs = 0;

    for (;;) {
        if (rank == 0 && tid == 0) s_case = (int)atomicAdd(&q->next, 1u);
        cl.sync();
        const int cid = *cl.map_shared_rank(&s_case, 0);
        if (cid >= ncases) break;
        if (tid == 0) {
            C = cases[cid];
            S = states[cid];
        }
        cl.sync();
        if (S.done) continue;

        const Params<T> &P = C.P;
        const Geo<T> &g = P.g;
        const int nx = g.nx, ny = g.ny, N = g.N;
        const int tiles_x = (nx + TX - 1) / TX, ntiles = tiles_x * ((ny + TY - 1) / TY);
        T *u = pool.u + C.off_c, *v = pool.v + C.off_c, *p = pool.p + C.off_c, *pc = pool.pc + C.off_c;
        T *ac = pool.ac + C.off_c, *rac = pool.rac + C.off_c, *sp = pool.sp + C.off_c;
        T *uf = pool.uf + C.off_uf, *vf = pool.vf + C.off_vf;
        T *bu[2] = {u, tp.tu + C.off_c}, *bv[2] = {v, tp.tv + C.off_c}, *bp[2] = {pc, tp.tpc + C.off_c};

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

        for (int it = 0; it < chunk && !S.done; ++it) {
            if (tid == 0)
                for (int e = 0; e < 4; ++e) {
                    L.stop[e] = 0;
                    L.inner_max[e] = -1e20;
                    L.sweeps[e] = 0;
                }
            __syncthreads();
            int mcur = 0, pcur = 0;

            // ---------------- momentum passes ----------------
            const int nu = C.n_iter[0], nv = C.n_iter[1];
            const int npass_m = (max(nu, nv) + KS - 1) / KS;
            for (int pass = 0; pass < (npass_m > 0 ? npass_m : 1); ++pass) {
                const int ns0 = clamp_sweeps(nu, pass, KS), ns1 = clamp_sweeps(nv, pass, KS);
                const bool au = ns0 > 0 && !L.stop[EQ_U];
                const bool av = ns1 > 0 && !L.stop[EQ_V];
                if (!au && !av && pass > 0) continue;  // the same in every CTA
                double acc[2 * KS];
#pragma unroll
                for (int s = 0; s < 2 * KS; ++s) acc[s] = 0.0;
                for (int t = (int)rank; t < ntiles; t += kCL) {
                    const int x0 = (t % tiles_x) * TX, y0 = (t / tiles_x) * TY;
                    const int gx0 = x0 - H, gy0 = y0 - H;
                    for (int q2 = tid; q2 < NR; q2 += NT) {
                        const int gi = gx0 + q2 % W, gj = gy0 + q2 / W;
                        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
                        const int id = gi + nx * gj;
                        s0[q2] = in ? bu[mcur][id] : (T)0;
                        s1[q2] = in ? bv[mcur][id] : (T)0;
                        s2[q2] = in ? p[id] : (T)0;
                    }
                    int cq[2][CPT], dq[2][CPT];
                    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
                    __syncthreads();
                    T cE[2][CPT], cW[2][CPT], cN[2][CPT], cS[2][CPT], cC[2][CPT], cbu[2][CPT], cbv[2][CPT];
                    bool own[2][CPT];
#pragma unroll
                    for (int c = 0; c < 2; ++c)
#pragma unroll
                        for (int k = 0; k < CPT; ++k) {
                            const int q2 = cq[c][k];
                            dq[c][k] = tile_distance<W, H, TX, TY>(q2);
                            own[c][k] = false;
                            cE[c][k] = cW[c][k] = cN[c][k] = cS[c][k] = cbu[c][k] = cbv[c][k] = (T)0;
                            cC[c][k] = (T)1;
                            if (q2 < 0) continue;
                            const int a = q2 % W, b = q2 / W;
                            const int gi = gx0 + a, gj = gy0 + b;
                            const int fu = gi + (nx + 1) * gj, fv = gi + nx * gj;
                            T a7[7], b3[3];
                            mom_cell<T, 2>(P, gi, gj, 0, uf[fu], uf[fu + 1], vf[fv], vf[fv + nx], (T)0, (T)0, s2[q2],
                                           s2[q2 - 1], s2[q2 + 1], s2[q2 - W], s2[q2 + W], (T)0, (T)0, a7, b3);
                            cE[c][k] = a7[AE];
                            cW[c][k] = a7[AW];
                            cN[c][k] = a7[AN];
                            cS[c][k] = a7[AS];
                            cC[c][k] = a7[AC];
                            cbu[c][k] = b3[0];
                            cbv[c][k] = b3[1];
                            own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
                            if (pass == 0 && own[c][k]) ac[gi + nx * gj] = a7[AC];
                        }
                    const T ru = g.relax[EQ_U], rv = g.relax[EQ_V];
#pragma unroll 1
                    for (int s = 0; s < KS; ++s) {
                        const bool du = au && s < ns0;
                        const bool dv = av && s < ns1;
                        if (!du && !dv) break;
#pragma unroll
                        for (int color = 0; color < 2; ++color) {
                            const int hs = 2 * s + color;
#pragma unroll
                            for (int k = 0; k < CPT; ++k) {
                                const int q2 = cq[color][k];
                                if (q2 < 0) continue;
                                T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k],
                                           (T)0, (T)0};
                                T d;
                                if (du && dq[color][k] <= 2 * ns0 - 1 - hs) {
                                    s0[q2] = point_update<T, 2>(a7, cbu[color][k], s0[q2], s0[q2 + 1], s0[q2 - 1],
                                                                s0[q2 + W], s0[q2 - W], (T)0, (T)0, ru, d);
                                    if (own[color][k]) acc[s] += (double)d * (double)d;
                                }
                                if (dv && dq[color][k] <= 2 * ns1 - 1 - hs) {
                                    s1[q2] = point_update<T, 2>(a7, cbv[color][k], s1[q2], s1[q2 + 1], s1[q2 - 1],
                                                                s1[q2 + W], s1[q2 - W], (T)0, (T)0, rv, d);
                                    if (own[color][k]) acc[KS + s] += (double)d * (double)d;
                                }
                            }
                            __syncthreads();
                        }
                    }
                    for (int q2 = tid; q2 < TX * TY; q2 += NT) {
                        const int a = H + q2 % TX, b = H + q2 / TX;
                        const int gi = gx0 + a, gj = gy0 + b;
                        if (gi >= nx || gj >= ny) continue;
                        const int id = gi + nx * gj;
                        bu[mcur ^ 1][id] = s0[b * W + a];
                        bv[mcur ^ 1][id] = s1[b * W + a];
                    }
                    __syncthreads();  // the next tile restages the shared arrays
                }
                tb_block_sum<2 * KS, NT>(acc, part[rs]);
                cl.sync();
                cluster_total<2 * KS>(cl, part[rs], tot);
                rs ^= 1;
                if (tid == 0) {
                    if (au) tb_pass_done(L, EQ_U, tot, ns0, N, g.tol[EQ_U]);
                    if (av) tb_pass_done(L, EQ_V, tot + KS, ns1, N, g.tol[EQ_V]);
                }
                __syncthreads();
                mcur ^= 1;
            }
            T *const cu = bu[mcur], *const cv = bv[mcur];

            // ---- Rhie-Chow faces, face BCs, p' source, 1/aC (kernels.cuh:336-581)
            double mass_sq;
            {
                double m[1] = {0.0};
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) {
                        const int c = i + nx * j;
                        const T uw = i == 0 ? face_bc(g, WEST, 0, cu[c], j) : rcx(g, cu, ac, p, i, j);
                        const T ue = i == nx - 1 ? face_bc(g, EAST, 0, cu[c], j) : rcx(g, cu, ac, p, i + 1, j);
                        const T vs = j == 0 ? face_bc(g, SOUTH, 1, cv[c], 0) : rcy(g, cv, ac, p, i, j);
                        const T vn = j == ny - 1 ? face_bc(g, NORTH, 1, cv[c], 0) : rcy(g, cv, ac, p, i, j + 1);
                        const T bb = mass_imbalance<T, 2>(g, uw, ue, vs, vn, (T)0, (T)0);
                        uf[i + (nx + 1) * j] = uw;
                        if (i == nx - 1) uf[nx + (nx + 1) * j] = ue;
                        vf[c] = vs;
                        if (j == ny - 1) vf[c + nx] = vn;
                        sp[c] = bb;
                        rac[c] = (T)1 / ac[c];
                        m[0] += (double)bb * (double)bb;
                    }
                tb_block_sum<1, NT>(m, part[rs]);
                cl.sync();
                cluster_total<1>(cl, part[rs], tot);
                rs ^= 1;
                mass_sq = tot[0];
            }

            // ---------------- p' passes from p' = 0 ----------------
            const int np = C.n_iter[3];
            const int npass_p = (np + KS - 1) / KS;
            for (int pass = 0; pass < npass_p; ++pass) {
                const int ns = clamp_sweeps(np, pass, KS);
                if (ns <= 0 || L.stop[EQ_P]) continue;  // the same in every CTA
                double acc[KS];
#pragma unroll
                for (int s = 0; s < KS; ++s) acc[s] = 0.0;
                for (int t = (int)rank; t < ntiles; t += kCL) {
                    const int x0 = (t % tiles_x) * TX, y0 = (t / tiles_x) * TY;
                    const int gx0 = x0 - H, gy0 = y0 - H;
                    for (int q2 = tid; q2 < NR; q2 += NT) {
                        const int gi = gx0 + q2 % W, gj = gy0 + q2 / W;
                        const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
                        const int id = gi + nx * gj;
                        s0[q2] = (in && pass > 0) ? bp[pcur][id] : (T)0;
                        s1[q2] = in ? rac[id] : (T)0;
                    }
                    int cq[2][CPT], dq[2][CPT];
                    own_cells<W, R::HH, R::NHALF, NT, CPT>(tid, gx0, gy0, nx, ny, cq);
                    __syncthreads();
                    T cE[2][CPT], cW[2][CPT], cN[2][CPT], cS[2][CPT], cC[2][CPT], cb[2][CPT];
                    bool own[2][CPT];
#pragma unroll
                    for (int c = 0; c < 2; ++c)
#pragma unroll
                        for (int k = 0; k < CPT; ++k) {
                            const int q2 = cq[c][k];
                            dq[c][k] = tile_distance<W, H, TX, TY>(q2);
                            own[c][k] = false;
                            cE[c][k] = cW[c][k] = cN[c][k] = cS[c][k] = cb[c][k] = (T)0;
                            cC[c][k] = (T)1;
                            if (q2 < 0) continue;
                            const int a = q2 % W, b = q2 / W;
                            const int gi = gx0 + a, gj = gy0 + b;
                            const T r = s1[q2];
                            const T e = gi < nx - 1 ? (T)(P.d.Kx * (double)(T)(r + s1[q2 + 1])) : (T)0;
                            const T w = gi > 0 ? (T)(P.d.Kx * (double)(T)(r + s1[q2 - 1])) : (T)0;
                            const T n = gj < ny - 1 ? (T)(P.d.Ky * (double)(T)(r + s1[q2 + W])) : (T)0;
                            const T so = gj > 0 ? (T)(P.d.Ky * (double)(T)(r + s1[q2 - W])) : (T)0;
                            cE[c][k] = e;
                            cW[c][k] = w;
                            cN[c][k] = n;
                            cS[c][k] = so;
                            cC[c][k] = -(e + w + n + so);
                            cb[c][k] = sp[gi + nx * gj];
                            own[c][k] = a >= H && a < H + TX && b >= H && b < H + TY;
                        }
                    const T relax = g.relax[EQ_P];
#pragma unroll 1
                    for (int s = 0; s < KS; ++s) {
                        if (s >= ns) break;
#pragma unroll
                        for (int color = 0; color < 2; ++color) {
                            const int reach = 2 * ns - 1 - (2 * s + color);
#pragma unroll
                            for (int k = 0; k < CPT; ++k) {
                                const int q2 = cq[color][k];
                                if (q2 < 0 || dq[color][k] > reach) continue;
                                T a7[7] = {cC[color][k], cE[color][k], cW[color][k], cN[color][k], cS[color][k],
                                           (T)0, (T)0};
                                T d;
                                s0[q2] = point_update<T, 2>(a7, cb[color][k], s0[q2], s0[q2 + 1], s0[q2 - 1],
                                                            s0[q2 + W], s0[q2 - W], (T)0, (T)0, relax, d);
                                if (own[color][k]) acc[s] += (double)d * (double)d;
                            }
                            __syncthreads();
                        }
                    }
                    for (int q2 = tid; q2 < TX * TY; q2 += NT) {
                        const int a = H + q2 % TX, b = H + q2 / TX;
                        const int gi = gx0 + a, gj = gy0 + b;
                        if (gi >= nx || gj >= ny) continue;
                        bp[pcur ^ 1][gi + nx * gj] = s0[b * W + a];
                    }
                    __syncthreads();
                }
                tb_block_sum<KS, NT>(acc, part[rs]);
                cl.sync();
                cluster_total<KS>(cl, part[rs], tot);
                rs ^= 1;
                if (tid == 0) tb_pass_done(L, EQ_P, tot, ns, N, g.tol[EQ_P]);
                __syncthreads();
                pcur ^= 1;
            }
            T *const pcc = bp[pcur];
            if (npass_p == 0) {
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) pcc[i + nx * j] = (T)0;
                cl.sync();
            }

            // ---- FP64 removal of the p' mean (closed cavities)
            if (C.pin) {
                double m[1] = {0.0};
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) m[0] += (double)pcc[i + nx * j];
                tb_block_sum<1, NT>(m, part[rs]);
                cl.sync();
                cluster_total<1>(cl, part[rs], tot);
                rs ^= 1;
                const double mean = tot[0] / (double)N;
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) pcc[i + nx * j] = (T)((double)pcc[i + nx * j] - mean);
                cl.sync();
            }

            // ---- corrections + next iteration's boundary faces (kernels.cuh:583-843)
            {
                double sq[5] = {0, 0, 0, 0, 0};
                for (int j = gw; j < ny; j += TW)
                    for (int i = lane; i < nx; i += 32) {
                        const int c = i + nx * j, fu = i + (nx + 1) * j;
                        const T x = pcc[c], aC = ac[c];
                        const T xW = i > 0 ? pcc[c - 1] : (T)0, xE = i < nx - 1 ? pcc[c + 1] : (T)0;
                        const T xS = j > 0 ? pcc[c - nx] : (T)0, xN = j < ny - 1 ? pcc[c + nx] : (T)0;
                        const T aW = i > 0 ? ac[c - 1] : (T)1, aS = j > 0 ? ac[c - nx] : (T)1;
                        const T p0 = p[c], u0 = cu[c], v0 = cv[c];
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
                tb_block_sum<5, NT>(sq, part[rs]);
                cl.sync();
                cluster_total<5>(cl, part[rs], tot);
                rs ^= 1;
            }

            // ---- norms and convergence test (src/Solver.cu:226-268)
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
        cl.sync();
    }
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
