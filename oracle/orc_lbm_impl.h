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
            for (int p = 0; p < Q; p++) {
                R cdotu = (R)c->cx[p] * u + (R)c->cy[p] * v + (R)c->cz[p] * w;
                R fn = f_p[p] * omegp + ((R)c->w[p] * rho * ((R)1.0 + (R)3.0 * cdotu + (R)4.5 * cdotu * cdotu - (R)1.5 * udotu)) * omeg;
                if (valid_mask != ORC_CELL_SOLID) F[o + (int64_t)p * nmc] = fn;
            }
        }
    }
    return 0;
}

static int FN(impose_bc)(orc_case *c, int L)
{
    /* Cu_ImposeBC, solver_lbm_kernels.cu:693-887 (simple bounce-back hook path;
       the interpolated bounce-back of S_BC_TYPE=1 needs link lengths). */
    R *F = (R *)c->F;
    const int64_t nmc = c->nmc, nmb = c->nmb;
    const int Q = c->Q, MC = c->MC, dim = c->dim, Qmax = c->Qmax;
    const int n = c->n_ids[L];
    const int *ids = &c->id_set[(int64_t)L * nmb];
#pragma omp parallel for schedule(static)
    for (int kap = 0; kap < n; kap++) {
        int b = ids[kap];
        if (c->cblock_ID_onb[b] != 1) continue;
        int s_nbr[27];
        for (int S = 0; S < Qmax; S++) s_nbr[S] = c->cblock_ID_nbr[b + (int64_t)c->map[S] * nmb];
        for (int t = 0; t < MC; t++) {
            int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
            int64_t o = (int64_t)b * MC + t;
            int valid_mask = c->cells_ID_mask[o];
            R rho = F[o + (int64_t)(Q + 0) * nmc];
            R u = F[o + (int64_t)(Q + 1) * nmc];
            R v = F[o + (int64_t)(Q + 2) * nmc];
            R w = (dim == 3) ? F[o + (int64_t)(Q + 3) * nmc] : (R)0.0;
            for (int p = 1; p < Q; p++) {
                if (!orc_half(dim, p)) continue;
                int q = c->pb[p];
                R f_p = F[o + (int64_t)p * nmc];
                R f_q = F[o + (int64_t)q * nmc];
                int nb = s_nbr[orc_nbrslot(dim, I + c->cx[p], J + c->cy[p], K + c->cz[p])];
                if (nb < 0 && nb != ORC_N_SKIPID)
                    f_p = FN(bc_hook)(c, nb, f_p, rho, u, v, w, (R)c->w[p], (R)c->cx[p], (R)c->cy[p], (R)c->cz[p]);
                nb = s_nbr[orc_nbrslot(dim, I + c->cx[q], J + c->cy[q], K + c->cz[q])];
                if (nb < 0 && nb != ORC_N_SKIPID)
                    f_q = FN(bc_hook)(c, nb, f_q, rho, u, v, w, (R)c->w[q], (R)c->cx[q], (R)c->cy[q], (R)c->cz[q]);
                if (valid_mask != ORC_CELL_SOLID) {
                    F[o + (int64_t)p * nmc] = f_p;
                    F[o + (int64_t)q * nmc] = f_q;
                }
            }
        }
    }
    return 0;
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
