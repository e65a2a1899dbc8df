/*
 * ORACLE (test infrastructure only): per-level LBM phases, written once for
 * the reference's ufloat_t and included twice (R = float, R = double).
 * Expression order follows the cited reference lines; the file is compiled
 * with -ffp-contract=off so every operation rounds as written.
 */
#ifndef R
#error "define R and FN before including orc_lbm_impl.h"
#endif

static inline R FN(bc_hook)(const orc_case *c, int nbr_id, R f, R rho, R u, R v, R w,
                            R wp, R cxp, R cyp, R czp)
{
    /* Cu_ImposeBC presets of inc/custom.h:79-122; u_ref replaces the literal 0.05. */
    const R U = (R)c->P.u_ref;
    switch (c->P.bc_preset) {
    case AGAL_BC_LDC2D:
        if (nbr_id == -4) { R cdotu = (R)3.0 * (cxp * U); return f - (R)2.0 * wp * cdotu; }
        break;
    case AGAL_BC_LDC3D:
        if (nbr_id == -6) { R cdotu = (R)3.0 * (cxp * U); return f - (R)2.0 * wp * cdotu; }
        break;
    case AGAL_BC_FPSC2D:
    case AGAL_BC_FPSC3D: {
        int inflow = (nbr_id == -1 || nbr_id == -3 || nbr_id == -4);
        if (c->P.bc_preset == AGAL_BC_FPSC3D) inflow = inflow || nbr_id == -5 || nbr_id == -6;
        if (inflow) { R cdotu = (R)3.0 * (cxp * U); return f - (R)2.0 * wp * cdotu; }
        if (nbr_id == -2) {
            R cdotu = cxp * u + cyp * v + czp * w;
            cdotu = (R)1.0 + (R)4.5 * cdotu * cdotu - (R)1.5 * (u * u + v * v + w * w);
            return -f + (R)2.0 * wp * cdotu;
        }
        break;
    }
    default:
        break;
    }
    return f;
}

static inline R FN(feq)(R w, R rho, R cu, R udotu)
{
    return w * rho * ((R)1.0 + (R)3.0 * cu + (R)4.5 * cu * cu - (R)1.5 * udotu);
}

/* Deterministic IC noise in [-1, 1) from integer lattice coordinates. */
static inline double FN(noise)(uint64_t seed, int L, long ix, long iy, long iz, int comp)
{
    uint64_t z = seed ^ ((uint64_t)(unsigned)L << 56) ^ ((uint64_t)(ix & 0xFFFFF) << 36)
               ^ ((uint64_t)(iy & 0xFFFFF) << 16) ^ ((uint64_t)(iz & 0xFFFF)) ^ ((uint64_t)comp << 60);
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

static int FN(set_ic)(orc_case *c, int L)
{
    /* solver_lbm_kernels.cu:15-77 */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const R dxL = c->fp64 ? (R)c->dxf_d[L] : (R)c->dxf[L];
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
            R rho = (R)1.0, u = (R)0.0, v = (R)0.0, w = (R)0.0;
            if (c->P.ic_preset == AGAL_IC_UNIFORM) {
                u = (R)c->P.u_ref;
                if (c->P.ic_noise != 0.0) {
                    double a = c->P.ic_noise * c->P.u_ref;
                    long ix = lrint((double)c->cblock_f_X[b] / (double)dxL) + I;
                    long iy = lrint((double)c->cblock_f_X[b + nmb] / (double)dxL) + J;
                    long iz = (dim == 3) ? lrint((double)c->cblock_f_X[b + 2 * nmb] / (double)dxL) + K : 0;
                    u = (R)(c->P.u_ref + a * FN(noise)(c->P.seed, L, ix, iy, iz, 0));
                    v = (R)(a * FN(noise)(c->P.seed, L, ix, iy, iz, 1));
                    if (dim == 3) w = (R)(a * FN(noise)(c->P.seed, L, ix, iy, iz, 2));
                }
            }
            R udotu = u * u + v * v + w * w;
            int valid_mask = c->cells_ID_mask[(int64_t)b * MC + t];
            for (int p = 0; p < Q; p++) {
                R cdotu = (R)c->cx[p] * u + (R)c->cy[p] * v + (R)c->cz[p] * w;
                R f_p = (R)(-1.0);
                if (valid_mask != ORC_CELL_SOLID)
                    f_p = rho * (R)c->w[p] * ((R)1.0 + (R)3.0 * cdotu + (R)4.5 * cdotu * cdotu - (R)1.5 * udotu);
                F[(int64_t)b * MC + t + (int64_t)c->pb[p] * nmc] = f_p;
            }
            F[(int64_t)b * MC + t + (int64_t)(Q + 0) * nmc] = rho;
            F[(int64_t)b * MC + t + (int64_t)(Q + 1) * nmc] = u;
            F[(int64_t)b * MC + t + (int64_t)(Q + 2) * nmc] = v;
            if (dim == 3) F[(int64_t)b * MC + t + (int64_t)(Q + 3) * nmc] = w;
        }
    }
    return 0;
}

static int FN(refresh)(orc_case *c, int L)
{
    /* solver_lbm_kernels.cu:112-159 */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        for (int t = 0; t < MC; t++) {
            int64_t o = (int64_t)b * MC + t;
            R rho = 0, u = 0, v = 0, w = 0;
            for (int p = 0; p < Q; p++) {
                R f = F[o + (int64_t)c->pb[p] * nmc];
                rho += f;
                u += c->cx[p] * f;
                v += c->cy[p] * f;
                if (dim == 3) w += c->cz[p] * f;
            }
            u /= rho;
            v /= rho;
            if (dim == 3) w /= rho;
            F[o + (int64_t)(Q + 0) * nmc] = rho;
            F[o + (int64_t)(Q + 1) * nmc] = u;
            F[o + (int64_t)(Q + 2) * nmc] = v;
            if (dim == 3) F[o + (int64_t)(Q + 3) * nmc] = w;
        }
    }
    return 0;
}

/* D3Q19 MRT (no live kernel in the reference; the moment basis of the
   legacy solver_old/solver_lbm_collide_mrt_d3q19.cu, whose inverse transform
   is the transpose scaled by the row norms, with its equilibria :131-148 and
   the e equilibrium read as 19 rho |u|^2).  Basis rows as polynomials of c. */
static int FN(mrt_row)(int i, int cx, int cy, int cz)
{
    int c2 = cx * cx + cy * cy + cz * cz;
    switch (i) {
    case 0: return 1;
    case 1: return 19 * c2 - 30;
    case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
    case 3: return cx;
    case 4: return (5 * c2 - 9) * cx;
    case 5: return cy;
    case 6: return (5 * c2 - 9) * cy;
    case 7: return cz;
    case 8: return (5 * c2 - 9) * cz;
    case 9: return 3 * cx * cx - c2;
    case 10: return (3 * c2 - 5) * (3 * cx * cx - c2);
    case 11: return cy * cy - cz * cz;
    case 12: return (3 * c2 - 5) * (cy * cy - cz * cz);
    case 13: return cx * cy;
    case 14: return cy * cz;
    case 15: return cx * cz;
    case 16: return (cy * cy - cz * cz) * cx;
    case 17: return (cz * cz - cx * cx) * cy;
    default: return (cx * cx - cy * cy) * cz;
    }
}

static void FN(mrt)(const orc_case *c, const R *f, R rho, R u, R v, R w, R omeg, R *out)
{
    R m[19];
    int n[19];
    for (int i = 0; i < 19; i++) {
        R acc = 0;
        n[i] = 0;
        for (int p = 0; p < 19; p++) {
            int k = FN(mrt_row)(i, c->cx[p], c->cy[p], c->cz[p]);
            acc += (R)k * f[p];
            n[i] += k * k;
        }
        m[i] = acc;
    }
    const R s1 = (R)c->P.s1, s2 = (R)c->P.s2, s3 = (R)c->P.s3, s5 = (R)c->P.s5, s6 = (R)c->P.s6;
    const R usq = u * u + v * v + w * w;
    R eq[19] = {0};
    eq[1] = (R)(-11.0) * rho + (R)19.0 * rho * usq;
    eq[2] = (R)3.0 * rho - (R)5.5 * rho * usq;
    eq[4] = (R)(-2.0 / 3.0) * rho * u;
    eq[6] = (R)(-2.0 / 3.0) * rho * v;
    eq[8] = (R)(-2.0 / 3.0) * rho * w;
    eq[9] = (R)2.0 * rho * u * u - rho * (v * v + w * w);
    eq[10] = (R)(-0.5) * eq[9];
    eq[11] = rho * (v * v - w * w);
    eq[12] = (R)(-0.5) * eq[11];
    eq[13] = rho * u * v;
    eq[14] = rho * v * w;
    eq[15] = rho * u * w;
    const R rate[19] = {0, s1, s2, 0, s3, 0, s3, 0, s3, omeg, s5, omeg, s5, omeg, omeg, omeg, s6, s6, s6};
    for (int i = 0; i < 19; i++) m[i] = m[i] - rate[i] * (m[i] - eq[i]);
    for (int p = 0; p < 19; p++) {
        R acc = 0;
        for (int i = 0; i < 19; i++) {
            int k = FN(mrt_row)(i, c->cx[p], c->cy[p], c->cz[p]);
            if (k) acc += (R)((double)k / (double)n[i]) * m[i];
        }
        out[p] = acc;
    }
}

static int FN(collide)(orc_case *c, int L)
{
    /* Cu_Collide, solver_lbm_kernels.cu:206-289 */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const R dxL = c->fp64 ? (R)c->dxf_d[L] : (R)c->dxf[L];
    const R tauL = (R)c->tau[L];
    const R omeg = dxL / tauL;
    const R omegp = (R)1.0 - omeg;
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        if (!(c->cblock_ID_nbr_child[b] < 0 || c->cblock_ID_mask[b] != ORC_BLOCK_SOLID)) continue;
        for (int t = 0; t < MC; t++) {
            int64_t o = (int64_t)b * MC + t;
            int valid_mask = c->cells_ID_mask[o];
            R rho = 0, u = 0, v = 0, w = 0;
            R f_p[27];
            for (int p = 0; p < Q; p++) {
                R f = F[o + (int64_t)c->pb[p] * nmc];
                rho += f;
                u += c->cx[p] * f;
                v += c->cy[p] * f;
                if (dim == 3) w += c->cz[p] * f;
                f_p[p] = f;
            }
            u /= rho;
            v /= rho;
            if (dim == 3) w /= rho;
            R udotu = u * u + v * v + w * w;
            F[o + (int64_t)(Q + 0) * nmc] = rho;
            F[o + (int64_t)(Q + 1) * nmc] = u;
            F[o + (int64_t)(Q + 2) * nmc] = v;
            if (dim == 3) F[o + (int64_t)(Q + 3) * nmc] = w;
            if (Q == 19 && c->P.collision == AGAL_MRT) {
                R fn[19];
                FN(mrt)(c, f_p, rho, u, v, w, omeg, fn);
                for (int p = 0; p < Q; p++)
                    if (valid_mask != ORC_CELL_SOLID) F[o + (int64_t)p * nmc] = fn[p];
                continue;
            }
            for (int p = 0; p < Q; p++) {
                R cdotu = (R)c->cx[p] * u + (R)c->cy[p] * v + (R)c->cz[p] * w;
                R fn = f_p[p] * omegp + ((R)c->w[p] * rho * ((R)1.0 + (R)3.0 * cdotu + (R)4.5 * cdotu * cdotu - (R)1.5 * udotu)) * omeg;
                if (valid_mask != ORC_CELL_SOLID) F[o + (int64_t)p * nmc] = fn;
            }
        }
    }
    return 0;
}

/* Interpolated bounce-back of one link (solver_lbm_kernels.cu:816-824):
   f is the post-collision value leaving the boundary cell towards the wall,
   f_m the one of the cell behind it, f_o the opposite population of the
   boundary cell; dQ the link length in cell units. */
static inline R FN(bouzidi)(R f, R f_m, R f_o, float dQf)
{
    const R dQ = (R)dQf;
    if (dQf > 0 && dQf < 0.5f) return (R)2.0 * dQ * f + ((R)1.0 - (R)2.0 * dQ) * f_m;
    if (dQf >= 0.5f) return ((R)1.0 / ((R)2.0 * dQ)) * f + (((R)2.0 * dQ - (R)1.0) / ((R)2.0 * dQ)) * f_o;
    return f;
}

static int FN(impose_bc)(orc_case *c, int L)
{
    /* Cu_ImposeBC, solver_lbm_kernels.cu:693-887: the boundary hook on domain
       faces, then with S_BC_TYPE=1 the interpolated bounce-back of boundary
       cells of wall blocks, in the order p-hook, p-wall, pb-hook, pb-wall of
       each pair.  The wall update reads the post-collision value of the
       cell behind the boundary cell; the reference reads it while other
       blocks rewrite their own pairs, so here every block reads the values
       before this phase and the results are written afterwards. */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb, ncb = c->n_maxcells_b;
    const int Q = c->Q, MC = c->MC, dim = c->dim, Qmax = c->Qmax;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const int wall = c->geometry_init && c->P.S_BC_TYPE > 0 && c->X_b;
    R *out = (R *)malloc(sizeof(R) * (size_t)(n > 0 ? n : 1) * MC * Q);
    if (!out) return AGAL_ERR_OOM;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        if (c->cblock_ID_onb[b] != 1) continue;
        const int bm = c->geometry_init ? c->onb_solid[b] : -1;
        int s_nbr[27];
        for (int S = 0; S < Qmax; S++) s_nbr[S] = c->cblock_ID_nbr[b + (int64_t)c->map[S] * nmb];
        R *ob = &out[(int64_t)kap * MC * Q];
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
            int64_t o = (int64_t)b * MC + t;
            int valid_mask = c->cells_ID_mask[o];
            R rho = F[o + (int64_t)(Q + 0) * nmc];
            R u = F[o + (int64_t)(Q + 1) * nmc];
            R v = F[o + (int64_t)(Q + 2) * nmc];
            R w = (dim == 3) ? F[o + (int64_t)(Q + 3) * nmc] : (R)0.0;
            const int bz = wall && valid_mask == ORC_CELL_BOUNDARY && bm > -1;
            for (int p = 0; p < Q; p++) ob[p * MC + t] = F[o + (int64_t)p * nmc];
            for (int p = 1; p < Q; p++) {
                if (!orc_half(dim, p)) continue;
                int q = c->pb[p];
                R f_p = F[o + (int64_t)p * nmc];
                R f_q = F[o + (int64_t)q * nmc];
                int nb = s_nbr[orc_nbrslot(dim, I + c->cx[p], J + c->cy[p], K + c->cz[p])];
                if (nb < 0 && nb != ORC_N_SKIPID)
                    f_p = FN(bc_hook)(c, nb, f_p, rho, u, v, w, (R)c->w[p], (R)c->cx[p], (R)c->cy[p], (R)c->cz[p]);
                if (bz) {
                    const int Ib = I + c->cx[q], Jb = J + c->cy[q], Kb = K + c->cz[q];
                    const int nbh = s_nbr[orc_nbrslot(dim, Ib, Jb, Kb)];
                    if (nbh < 0) { bad = 1; continue; }
                    const R f_m = F[(int64_t)nbh * MC + orc_nbrcell(dim, Ib, Jb, Kb) + (int64_t)p * nmc];
                    f_p = FN(bouzidi)(f_p, f_m, f_q, c->X_b[(int64_t)bm * MC + t + (int64_t)p * ncb]);
                }
                nb = s_nbr[orc_nbrslot(dim, I + c->cx[q], J + c->cy[q], K + c->cz[q])];
                if (nb < 0 && nb != ORC_N_SKIPID)
                    f_q = FN(bc_hook)(c, nb, f_q, rho, u, v, w, (R)c->w[q], (R)c->cx[q], (R)c->cy[q], (R)c->cz[q]);
                if (bz) {
                    const int Ib = I + c->cx[p], Jb = J + c->cy[p], Kb = K + c->cz[p];
                    const int nbh = s_nbr[orc_nbrslot(dim, Ib, Jb, Kb)];
                    if (nbh < 0) { bad = 1; continue; }
                    const R f_m = F[(int64_t)nbh * MC + orc_nbrcell(dim, Ib, Jb, Kb) + (int64_t)q * nmc];
                    f_q = FN(bouzidi)(f_q, f_m, f_p, c->X_b[(int64_t)bm * MC + t + (int64_t)q * ncb]);
                }
                if (valid_mask != ORC_CELL_SOLID) {
                    ob[p * MC + t] = f_p;
                    ob[q * MC + t] = f_q;
                }
            }
        }
    }
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        if (c->cblock_ID_onb[b] != 1) continue;
        const R *ob = &out[(int64_t)kap * MC * Q];
        for (int p = 0; p < Q; p++)
            for (int t = 0; t < MC; t++) F[(int64_t)b * MC + t + (int64_t)p * nmc] = ob[p * MC + t];
    }
    free(out);
    /* A wall link whose cell behind has no block: the reference reads
       outside its arrays there. */
    return bad ? AGAL_ERR_STATE : 0;
}

/* Cu_ComputeForcesMEA (solver_lbm_kernels_forces.cu:324-537): momentum
   exchange over the wall links of boundary cells, summed per block into
   cblock_f_Ff (post = 0 stores, post = 1 adds). */
static int FN(forces_mea)(orc_case *c, int L, int post)
{
    if (!c->geometry_init || !c->X_b || L != c->max_levels - 1 || c->n_ids[L] <= 0) return 0;
    R *F = (R *)c->F;
    R *Ff = (R *)c->Ff;
    const int64_t nmc = c->nmc, nmb = c->nmb, ncb = c->n_maxcells_b;
    const int Q = c->Q, MC = c->MC, dim = c->dim, Qmax = c->Qmax;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const R dxL = c->fp64 ? (R)c->dxf_d[L] : (R)c->dxf[L];
    R dvL = (R)1.0;
    for (int d = 0; d < dim; d++) dvL *= dxL;
    const int order = c->P.S_FORCE_ORDER;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int kap = 0; kap < n; kap++) {
        const int b = ids[kap];
        const int bm = c->onb_solid[b];
        if (bm < 0) continue;
        int s_nbr[27];
        for (int S = 0; S < Qmax; S++) s_nbr[S] = c->cblock_ID_nbr[b + (int64_t)c->map[S] * nmb];
        R s[64][3];
        for (int t = 0; t < MC; t++) {
            s[t][0] = s[t][1] = s[t][2] = (R)0.0;
            const int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
            const int64_t o = (int64_t)b * MC + t;
            if (c->cells_ID_mask[o] != ORC_CELL_BOUNDARY) continue;
            for (int p = 1; p < Q; p++) {
                if (!orc_half(dim, p)) continue;
                const int q = c->pb[p];
                const R f_p = F[o + (int64_t)p * nmc];
                const R f_q = F[o + (int64_t)q * nmc];
                for (int side = 0; side < 2; side++) {
                    const int a = side ? q : p;      /* link direction */
                    const int e = side ? p : q;      /* towards the cell behind */
                    const R f_a = side ? f_q : f_p;
                    const float dist = c->X_b[(int64_t)bm * MC + t + (int64_t)a * ncb];
                    if (!(dist > 0)) continue;
                    const int Ib = I + c->cx[e], Jb = J + c->cy[e], Kb = K + c->cz[e];
                    const int nbh = s_nbr[orc_nbrslot(dim, Ib, Jb, Kb)];
                    if (nbh < 0) { bad = 1; continue; }
                    const R f_m = F[(int64_t)nbh * MC + orc_nbrcell(dim, Ib, Jb, Kb) + (int64_t)a * nmc];
                    const int ca[3] = {c->cx[a], c->cy[a], c->cz[a]};
                    for (int d = 0; d < dim; d++) {
                        if (order == 1) {
                            s[t][d] += f_a * (R)ca[d];
                        } else {
                            /* 0.5 is a double literal there: the term is formed in double. */
                            const double term = ((0.5 + (double)(R)dist) * (double)f_a + (0.5 - (double)(R)dist) * (double)f_m) * (double)ca[d];
                            s[t][d] = (R)((double)s[t][d] + term);
                        }
                    }
                }
            }
        }
        for (int h = MC / 2; h > 0; h >>= 1)
            for (int t = 0; t < h; t++)
                for (int d = 0; d < dim; d++) s[t][d] = s[t][d] + s[t + h][d];
        for (int d = 0; d < dim; d++) {
            if (post == 0) {
                Ff[b + (int64_t)(2 * d + 0) * nmb] = s[0][d] * dvL;
                Ff[b + (int64_t)(2 * d + 1) * nmb] = (R)0.0;
            } else {
                Ff[b + (int64_t)(2 * d + 0) * nmb] += s[0][d] * dvL;
            }
        }
    }
    return bad ? AGAL_ERR_STATE : 0;
}

/* S_ReportForces sums (solver_lbm_compute.cu:166-201): the six rows of
   cblock_f_Ff over block IDs below id_max[MAX_LEVELS], in double. */
static void FN(forces_sum)(const orc_case *c, double *out)
{
    const R *Ff = (const R *)c->Ff;
    const int n = c->id_max[c->max_levels];
    for (int r = 0; r < 6; r++) {
        double s = 0.0;
        for (int b = 0; b < n; b++) s += (double)Ff[b + (int64_t)r * c->nmb];
        out[r] = s;
    }
}

static int FN(stream)(orc_case *c, int L)
{
    /* Cu_Stream, solver_lbm_kernels.cu:534-633: swap slot p of x with slot
       pb(p) of x + c_p.  Every (cell, slot) pair is touched by exactly one
       swap, so blocks can be processed in parallel. */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim, Qmax = c->Qmax;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        if (!(c->cblock_ID_nbr_child[b] < 0 || c->cblock_ID_mask[b] != ORC_BLOCK_SOLID)) continue;
        int s_nbr[27];
        for (int S = 0; S < Qmax; S++) s_nbr[S] = c->cblock_ID_nbr[b + (int64_t)c->map[S] * nmb];
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
            int64_t o = (int64_t)b * MC + t;
            int valid_mask = c->cells_ID_mask[o];
            for (int p = 1; p < Q; p++) {
                if (!orc_half(dim, p)) continue;
                R f_p = F[o + (int64_t)p * nmc];
                int Ip = I + c->cx[p], Jp = J + c->cy[p], Kp = K + c->cz[p];
                int nb = s_nbr[orc_nbrslot(dim, Ip, Jp, Kp)];
                int nc = orc_nbrcell(dim, Ip, Jp, Kp);
                R f_pb = (R)(-1.0);
                if (nb > -1) f_pb = F[(int64_t)nb * MC + nc + (int64_t)c->pb[p] * nmc];
                if (valid_mask != ORC_CELL_SOLID && f_pb > 0) {
                    F[(int64_t)nb * MC + nc + (int64_t)c->pb[p] * nmc] = f_p;
                    F[o + (int64_t)p * nmc] = f_pb;
                }
            }
        }
    }
    return 0;
}

static void FN(mass_momentum)(const orc_case *c, double *out)
{
    const R *F = (const R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim;
    double m = 0, mx = 0, my = 0, mz = 0;
    for (int L = 0; L < c->max_levels; L++) {
        const int *ids = &c->id_set[(int64_t)L * nmb];
        for (int kap = 0; kap < c->n_ids[L]; kap++) {
            int b = ids[kap];
            if (c->cblock_ID_nbr_child[b] >= 0) continue;   /* leaf blocks only */
            const double vol = ldexp(1.0, -L * dim);   /* (dx_L / dx_0)^dim */
            for (int t = 0; t < MC; t++) {
                int64_t o = (int64_t)b * MC + t;
                if (c->cells_ID_mask[o] == ORC_CELL_SOLID) continue;
                for (int p = 0; p < Q; p++) {
                    double f = (double)F[o + (int64_t)c->pb[p] * nmc];
                    m += f * vol;
                    mx += c->cx[p] * f * vol;
                    my += c->cy[p] * f * vol;
                    mz += c->cz[p] * f * vol;
                }
            }
        }
    }
    out[0] = m; out[1] = mx; out[2] = my;
    if (dim == 3) out[3] = mz;
}

/* ---------------------------------------------------------------------------
 * Level-interface transfers (solver_lbm_kernels_comm.cu) and the refinement
 * criterion (solver_lbm_criterion.cu).  They read the macros stored in slots
 * Q..Q+dim by the last refresh, as the reference does.
 */

/* Rescaled population g = feq + (f - feq) * ratio of slot pb(p) of cell o. */
static inline R FN(rescaled)(const orc_case *c, const R *F, int64_t o, int p, R ratio)
{
    const int64_t nmc = c->nmc;
    const int Q = c->Q;
    R rho = F[o + (int64_t)(Q + 0) * nmc];
    R u = F[o + (int64_t)(Q + 1) * nmc];
    R v = F[o + (int64_t)(Q + 2) * nmc];
    R w = (c->dim == 3) ? F[o + (int64_t)(Q + 3) * nmc] : (R)0.0;
    R udotu = u * u + v * v + w * w;
    R cdotu = (R)c->cx[p] * u + (R)c->cy[p] * v + (R)c->cz[p] * w;
    R feq = (R)c->w[p] * rho * ((R)1.0 + (R)3.0 * cdotu + (R)4.5 * cdotu * cdotu - (R)1.5 * udotu);
    R f = F[o + (int64_t)c->pb[p] * nmc];
    return feq + (f - feq) * ratio;
}

/* Lagrange weight of node a (nodes at 0, 1/3, 2/3, 1) at position x. */
static inline double FN(lag4)(int a, double x)
{
    static const double t[4] = {0.0, 1.0 / 3.0, 2.0 / 3.0, 1.0};
    double r = 1.0;
    for (int k = 0; k < 4; k++)
        if (k != a) r *= (x - t[k]) / (t[a] - t[k]);
    return r;
}

static int FN(interpolate)(orc_case *c, int L, int var)
{
    /* Cu_Interpolate_Linear (kernels_comm.cu:15-138) and Cu_Interpolate_Cubic
       (:406-640): parent cells rescaled by tau_{L+1}/tau_L, then bilinear /
       trilinear (offsets -0.25 + 0.5 I from parent cell 2ci) or tricubic
       Lagrange on the 4^d parent cells (children at -1/12 + m/6 in units where
       parent cell k sits at k/3) into the children's ghost cells (mask 2) or,
       for newly added children, into all their cells. */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim, NCH = c->NCH;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const R ratio = c->fp64 ? (R)(c->tau[L + 1] / c->tau[L]) : (R)((float)c->tau[L + 1] / (float)c->tau[L]);
    const int cubic = (c->P.interp_order == AGAL_INTERP_CUBIC);
    /* cubic weights: positions m = 0..7 along an axis */
    double W[4][8];
    for (int a = 0; a < 4; a++)
        for (int m = 0; m < 8; m++) W[a][m] = FN(lag4)(a, -1.0 / 12.0 + m / 6.0);
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        int bc = c->cblock_ID_nbr_child[b];
        int b1 = (var == AGAL_INTERP_INTERFACE) && (c->cblock_ID_mask[b] == ORC_BLOCK_INTERFACE);
        int b2 = (var == AGAL_INTERP_ADDED) && (c->cblock_ID_ref[b] == ORC_REF_MARK_REFINE);
        if (!(b1 || b2)) continue;
        R sF[64];
        for (int p = 0; p < Q; p++) {
            for (int t = 0; t < MC; t++) sF[t] = FN(rescaled)(c, F, (int64_t)b * MC + t, p, ratio);
            for (int ch = 0; ch < NCH; ch++) {
                int ci = ch & 1, cj = (ch >> 1) & 1, ck = (ch >> 2) & 1;
                int64_t cb = (int64_t)(bc + ch);
                for (int t = 0; t < MC; t++) {
                    if (var == AGAL_INTERP_INTERFACE && c->cells_ID_mask[cb * MC + t] != ORC_CELL_GHOST) continue;
                    int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
                    R val;
                    if (!cubic) {
                        int s = 2 * ci + 8 * cj + 32 * ck;
                        R Ix = (R)(-0.25) + (R)(0.5) * (R)I, Iy = (R)(-0.25) + (R)(0.5) * (R)J;
                        if (dim == 2) {
                            val = sF[0 + s] + (sF[1 + s] - sF[0 + s]) * Ix + (sF[4 + s] - sF[0 + s]) * Iy +
                                  (sF[5 + s] - sF[4 + s] - sF[1 + s] + sF[0 + s]) * Ix * Iy;
                        } else {
                            R Iz = (R)(-0.25) + (R)(0.5) * (R)K;
                            val = sF[0 + s] + (sF[1 + s] - sF[0 + s]) * Ix + (sF[4 + s] - sF[0 + s]) * Iy +
                                  (sF[16 + s] - sF[0 + s]) * Iz +
                                  (sF[5 + s] - sF[1 + s] - sF[4 + s] + sF[0 + s]) * Ix * Iy +
                                  (sF[17 + s] - sF[1 + s] - sF[16 + s] + sF[0 + s]) * Ix * Iz +
                                  (sF[20 + s] - sF[4 + s] - sF[16 + s] + sF[0 + s]) * Iy * Iz +
                                  (sF[21 + s] + sF[1 + s] + sF[4 + s] + sF[16 + s] - sF[5 + s] - sF[17 + s] -
                                   sF[20 + s] - sF[0 + s]) * Ix * Iy * Iz;
                        }
                    } else {
                        int mx = I + 4 * ci, my = J + 4 * cj, mz = K + 4 * ck;
                        double acc = 0.0;
                        if (dim == 2) {
                            for (int bj = 0; bj < 4; bj++)
                                for (int ai = 0; ai < 4; ai++) acc += W[ai][mx] * W[bj][my] * (double)sF[ai + 4 * bj];
                        } else {
                            for (int ck2 = 0; ck2 < 4; ck2++)
                                for (int bj = 0; bj < 4; bj++)
                                    for (int ai = 0; ai < 4; ai++)
                                        acc += W[ai][mx] * W[bj][my] * W[ck2][mz] * (double)sF[ai + 4 * bj + 16 * ck2];
                        }
                        val = (R)acc;
                    }
                    F[cb * MC + t + (int64_t)c->pb[p] * nmc] = val;
                }
            }
        }
    }
    return 0;
}

static int FN(average)(orc_case *c, int L, int var)
{
    /* Cu_Average (kernels_comm.cu:174-347): parent cell = mean of the 2^d child
       cells under it, rescaled by tau_L/tau_{L+1}, where the child cell at the
       quadrant's corner has mask 1 (INTERFACE) or mask < 2 (BLOCK, GRID). */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim, NCH = c->NCH;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const R ratio = c->fp64 ? (R)(c->tau[L] / c->tau[L + 1]) : (R)((float)c->tau[L] / (float)c->tau[L + 1]);
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        int bc = c->cblock_ID_nbr_child[b];
        if (!(bc > -1 && (var == AGAL_AVERAGE_GRID || c->cblock_ID_mask[b] == ORC_BLOCK_INTERFACE))) continue;
        for (int ch = 0; ch < NCH; ch++) {
            int ci = ch & 1, cj = (ch >> 1) & 1, ck = (ch >> 2) & 1;
            int64_t cb = (int64_t)(bc + ch);
            int mask[64];
            for (int t = 0; t < MC; t++) {
                mask[t] = c->cells_ID_mask[cb * MC + t];
                if (var > 0 && mask[t] < 2) mask[t] = 1;
            }
            R g[64];
            for (int p = 0; p < Q; p++) {
                for (int t = 0; t < MC; t++) g[t] = FN(rescaled)(c, F, cb * MC + t, p, ratio);
                for (int t = 0; t < MC; t++) {
                    int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
                    if (!(I >= 2 * ci && I < 2 + 2 * ci && J >= 2 * cj && J < 2 + 2 * cj)) continue;
                    if (dim == 3 && !(K >= 2 * ck && K < 2 + 2 * ck)) continue;
                    int c0 = 2 * (I % 2) + 4 * (2 * (J % 2)) + (dim == 3 ? 16 * (2 * (K % 2)) : 0);
                    if (mask[c0] != 1) continue;
                    R val;
                    if (dim == 2)
                        val = (R)0.25 * (g[c0 + 0] + g[c0 + 1] + g[c0 + 4] + g[c0 + 5]);
                    else
                        val = (R)0.125 * (g[c0 + 0] + g[c0 + 1] + g[c0 + 4] + g[c0 + 5] + g[c0 + 16] + g[c0 + 17] +
                                          g[c0 + 20] + g[c0 + 21]);
                    F[(int64_t)b * MC + t + (int64_t)c->pb[p] * nmc] = val;
                }
            }
        }
    }
    return 0;
}

static int FN(ref_criteria)(orc_case *c)
{
    /* Cu_ComputeRefCriteria (solver_lbm_criterion.cu:440-592), launched over
       every block ID below id_max[MAX_LEVELS] with the level-0 spacing (the
       reference passes dxf_vec[0], criterion.cu:604).  Halo by 4th-order
       extrapolation (util_math.h:56-116), central differences, floor(log2 |w|)
       (S_CRITERION 0) or of |Q| (1), ghost cells 0, block maximum. */
    const R *F = (const R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim, Qmax = c->Qmax;
    const int idm = c->id_max[c->max_levels];
    const R dxL = c->fp64 ? (R)c->dxf_d[0] : (R)c->dxf[0];
    const int MLI = c->P.MAX_LEVELS_INTERIOR;
    const R NRS = (R)c->P.N_REFINE_START, NRI = (R)c->P.N_REFINE_INC, NRM = (R)c->P.N_REFINE_MAX;
#pragma omp parallel for schedule(static)
    for (int b = 0; b < idm; b++) {
        if (c->cblock_ID_ref[b] == ORC_REF_INACTIVE) continue;
        R h[3][216];
        for (int comp = 0; comp < dim; comp++)
            for (int t = 0; t < MC; t++) {
                int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
                int hi = (I + 1) + 6 * (J + 1) + (dim == 3 ? 36 * (K + 1) : 0);
                h[comp][hi] = F[(int64_t)b * MC + t + (int64_t)(Q + 1 + comp) * nmc];
            }
        for (int comp = 0; comp < dim; comp++) {
            R *s = h[comp];
#define HI(i, j, k) (((i) + 1) + 6 * ((j) + 1) + (dim == 3 ? 36 * ((k) + 1) : 0))
            for (int t = 0; t < MC; t++) {
                int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
                if (I == 0) {
                    s[HI(-1, J, K)] = (R)4.0 * s[HI(0, J, K)] + (R)(-6.0) * s[HI(1, J, K)] + (R)4.0 * s[HI(2, J, K)] + (R)(-1.0) * s[HI(3, J, K)];
                    s[HI(4, J, K)] = (R)4.0 * s[HI(3, J, K)] + (R)(-6.0) * s[HI(2, J, K)] + (R)4.0 * s[HI(1, J, K)] + (R)(-1.0) * s[HI(0, J, K)];
                }
                if (J == 0) {
                    s[HI(I, -1, K)] = (R)4.0 * s[HI(I, 0, K)] + (R)(-6.0) * s[HI(I, 1, K)] + (R)4.0 * s[HI(I, 2, K)] + (R)(-1.0) * s[HI(I, 3, K)];
                    s[HI(I, 4, K)] = (R)4.0 * s[HI(I, 3, K)] + (R)(-6.0) * s[HI(I, 2, K)] + (R)4.0 * s[HI(I, 1, K)] + (R)(-1.0) * s[HI(I, 0, K)];
                }
                if (dim == 3 && K == 0) {
                    s[HI(I, J, -1)] = (R)4.0 * s[HI(I, J, 0)] + (R)(-6.0) * s[HI(I, J, 1)] + (R)4.0 * s[HI(I, J, 2)] + (R)(-1.0) * s[HI(I, J, 3)];
                    s[HI(I, J, 4)] = (R)4.0 * s[HI(I, J, 3)] + (R)(-6.0) * s[HI(I, J, 2)] + (R)4.0 * s[HI(I, J, 1)] + (R)(-1.0) * s[HI(I, J, 0)];
                }
            }
        }
        R Wmax = -INFINITY;
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
            R d[3][3] = {{0}};   /* d[comp][axis] */
            for (int comp = 0; comp < dim; comp++) {
                const R *s = h[comp];
                if (dim == 2) {
                    /* 2D divides by the double 2.0*dx_L (criterion.cu:502-505) */
                    d[comp][0] = (R)((double)(s[HI(I + 1, J, K)] - s[HI(I - 1, J, K)]) / (2.0 * (double)dxL));
                    d[comp][1] = (R)((double)(s[HI(I, J + 1, K)] - s[HI(I, J - 1, K)]) / (2.0 * (double)dxL));
                } else {
                    d[comp][0] = (s[HI(I + 1, J, K)] - s[HI(I - 1, J, K)]) / ((R)2 * dxL);
                    d[comp][1] = (s[HI(I, J + 1, K)] - s[HI(I, J - 1, K)]) / ((R)2 * dxL);
                    d[comp][2] = (s[HI(I, J, K + 1)] - s[HI(I, J, K - 1)]) / ((R)2 * dxL);
                }
            }
#undef HI
            R uX = d[0][0], uY = d[0][1], uZ = d[0][2], vX = d[1][0], vY = d[1][1], vZ = d[1][2];
            R wX = d[2][0], wY = d[2][1], wZ = d[2][2];
            R Wt = (R)0;
            if (c->P.S_CRITERION == 0)
                Wt = (R)floor(log2((double)(R)sqrt((double)((wY - vZ) * (wY - vZ) + (uZ - wX) * (uZ - wX) + (vX - uY) * (vX - uY)))));
            if (c->P.S_CRITERION == 1)
                Wt = (R)floor(log2((double)(R)fabs((double)((R)0.5 * (uX * uX + vY * vY + wZ * wZ + (R)2.0 * (uY * vX + uZ * wX + wY * vZ))))));
            if (c->cells_ID_mask[(int64_t)b * MC + t] == ORC_CELL_GHOST) Wt = (R)0;
            Wmax = (R)fmax((double)Wmax, (double)Wt);   /* BlockwiseMaximum with fmaxf (util.h:29, 787) */
        }
        if (Wmax > NRM) Wmax = NRM;
        int ref_kap = c->cblock_ID_ref[b], level_kap = c->cblock_level[b];
        int L_desired = MLI - 1;
        for (int p = 1; p <= MLI - 1; p++)
            if (Wmax < NRS - NRI * (R)p) L_desired = (MLI - 1) - p;
        int eligible = 1;
        for (int p = 0; p < Qmax; p++)
            if (c->cblock_ID_nbr[b + (int64_t)p * nmb] == ORC_N_SKIPID) eligible = 0;
        if (eligible && level_kap != MLI - 1 && ref_kap == ORC_REF_UNREFINED && L_desired > level_kap)
            c->cblock_ID_ref[b] = ORC_REF_MARK_REFINE;
        if (ref_kap == ORC_REF_REFINED && L_desired < level_kap + 1) c->cblock_ID_ref[b] = ORC_REF_MARK_COARSEN;
    }
    return 0;
}

/* ---------------------------------------------------------------------------
 * Percentile criterion (S_CRITERION = AGAL_CRITERION_PERCENTILE; the
 * reference has no counterpart).  Per block the maximum vorticity magnitude
 * over its non-ghost cells, from the macros of the last refresh, with the
 * halo of solver_lbm_criterion.cu (fourth-order extrapolation) and central
 * differences at the block's own spacing.  Every operation is written in the
 * order the CUDA kernel rounds it (this file is compiled without
 * contraction).  Leaf blocks above the ref_pct_hi quantile of all leaf
 * blocks are refined, refined blocks below the ref_pct_lo quantile coarsened.
 */
static R FN(xpol4)(R a, R b, R c4, R d)
{
    return (((R)4 * a + (R)(-6) * b) + (R)4 * c4) + (R)(-1) * d;
}

static R FN(block_wmax)(const orc_case *c, int b, R dxL)
{
    const R *F = (const R *)c->F;
    const int64_t nmc = c->nmc;
    const int Q = c->Q, MC = c->MC, dim = c->dim;
    R h[3][216];
#define HX(i, j, k) (((i) + 1) + 6 * ((j) + 1) + (dim == 3 ? 36 * ((k) + 1) : 0))
    for (int comp = 0; comp < dim; comp++) {
        R *s = h[comp];
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? t / 16 : 0;
            s[HX(I, J, K)] = F[(int64_t)b * MC + t + (int64_t)(Q + 1 + comp) * nmc];
        }
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? t / 16 : 0;
            if (I == 0) {
                s[HX(-1, J, K)] = FN(xpol4)(s[HX(0, J, K)], s[HX(1, J, K)], s[HX(2, J, K)], s[HX(3, J, K)]);
                s[HX(4, J, K)] = FN(xpol4)(s[HX(3, J, K)], s[HX(2, J, K)], s[HX(1, J, K)], s[HX(0, J, K)]);
            }
            if (J == 0) {
                s[HX(I, -1, K)] = FN(xpol4)(s[HX(I, 0, K)], s[HX(I, 1, K)], s[HX(I, 2, K)], s[HX(I, 3, K)]);
                s[HX(I, 4, K)] = FN(xpol4)(s[HX(I, 3, K)], s[HX(I, 2, K)], s[HX(I, 1, K)], s[HX(I, 0, K)]);
            }
            if (dim == 3 && K == 0) {
                s[HX(I, J, -1)] = FN(xpol4)(s[HX(I, J, 0)], s[HX(I, J, 1)], s[HX(I, J, 2)], s[HX(I, J, 3)]);
                s[HX(I, J, 4)] = FN(xpol4)(s[HX(I, J, 3)], s[HX(I, J, 2)], s[HX(I, J, 1)], s[HX(I, J, 0)]);
            }
        }
    }
    const R h2 = (R)2 * dxL;
    R wmax = (R)0;
    for (int t = 0; t < MC; t++) {
        if (c->cells_ID_mask[(int64_t)b * MC + t] == ORC_CELL_GHOST) continue;
        int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? t / 16 : 0;
        R g[3][3] = {{0}};
        for (int comp = 0; comp < dim; comp++) {
            const R *s = h[comp];
            g[comp][0] = (s[HX(I + 1, J, K)] - s[HX(I - 1, J, K)]) / h2;
            g[comp][1] = (s[HX(I, J + 1, K)] - s[HX(I, J - 1, K)]) / h2;
            if (dim == 3) g[comp][2] = (s[HX(I, J, K + 1)] - s[HX(I, J, K - 1)]) / h2;
        }
        R w;
        if (dim == 2) {
            w = (R)fabs((double)(g[1][0] - g[0][1]));
        } else {
            const R wx = g[2][1] - g[1][2], wy = g[0][2] - g[2][0], wz = g[1][0] - g[0][1];
            const R ss = (wx * wx + wy * wy) + wz * wz;
            w = (sizeof(R) == 4) ? (R)sqrtf((float)ss) : (R)sqrt((double)ss);
        }
        if (w > wmax) wmax = w;
    }
#undef HX
    return wmax;
}

static int FN(cmp_r)(const void *a, const void *b)
{
    const R x = *(const R *)a, y = *(const R *)b;
    return (x > y) - (x < y);
}

static int FN(ref_criteria_pct)(orc_case *c)
{
    const int64_t nmb = c->nmb;
    const int idm = c->id_max[c->max_levels], Qmax = c->Qmax;
    const int MLI = c->P.MAX_LEVELS_INTERIOR;
    R *w = (R *)malloc(sizeof(R) * (size_t)(idm > 0 ? idm : 1));
    R *pop = (R *)malloc(sizeof(R) * (size_t)(idm > 0 ? idm : 1));
    if (!w || !pop) { free(w); free(pop); return AGAL_ERR_OOM; }
    int n = 0;
    for (int b = 0; b < idm; b++) {
        w[b] = (R)-1;
        if (c->cblock_ID_ref[b] == ORC_REF_INACTIVE) continue;
        const int L = c->cblock_level[b];
        const R dxL = c->fp64 ? (R)c->dxf_d[L] : (R)c->dxf[L];
        w[b] = FN(block_wmax)(c, b, dxL);
        if (c->cblock_ID_nbr_child[b] < 0) pop[n++] = w[b];
    }
    if (n > 0) {
        qsort(pop, (size_t)n, sizeof(R), FN(cmp_r));
        const R thr_hi = pop[(int)floor(c->P.ref_pct_hi * (double)(n - 1))];
        const R thr_lo = pop[(int)floor(c->P.ref_pct_lo * (double)(n - 1))];
        for (int b = 0; b < idm; b++) {
            const int r = c->cblock_ID_ref[b];
            if (r == ORC_REF_INACTIVE) continue;
            int eligible = 1;
            for (int p = 0; p < Qmax; p++)
                if (c->cblock_ID_nbr[b + (int64_t)p * nmb] == ORC_N_SKIPID) eligible = 0;
            if (r == ORC_REF_UNREFINED && eligible && c->cblock_level[b] < MLI - 1 && w[b] > thr_hi)
                c->cblock_ID_ref[b] = ORC_REF_MARK_REFINE;
            if (r == ORC_REF_REFINED && w[b] < thr_lo) c->cblock_ID_ref[b] = ORC_REF_MARK_COARSEN;
        }
    }
    free(w);
    free(pop);
    return 0;
}
