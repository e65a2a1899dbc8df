/*
 * ORACLE (test infrastructure only) - see agal_oracle.h.
 *
 * Mesh construction and the level recursion of the reference, restated in C.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "orc_internal.h"

#define R float
#define FN(n) n##_f32
#include "orc_lbm_impl.h"
#undef R
#undef FN
#define R double
#define FN(n) n##_f64
#include "orc_lbm_impl.h"
#undef R
#undef FN

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* Padded root-grid value at (i, j, k), i in [0, bx+1] etc.  Boundaries are
   written z first, then y, then x (mesh_init.cu:406-460), so an x boundary
   wins over y and z at edges and corners; periodic faces copy the opposite
   interior layer. */
static int root_padded_id(const orc_case *c, int bx, int by, int bz, int i, int j, int k)
{
    if (i < 1 || i > bx) {
        if (!c->P.PERIODIC_X) return (i < 1) ? -1 : -2;
        i = (i < 1) ? bx : 1;
    }
    if (j < 1 || j > by) {
        if (!c->P.PERIODIC_Y) return (j < 1) ? -3 : -4;
        j = (j < 1) ? by : 1;
    }
    if (c->dim == 3 && (k < 1 || k > bz)) {
        if (!c->P.PERIODIC_Z) return (k < 1) ? -5 : -6;
        k = (k < 1) ? bz : 1;
    }
    if (c->dim == 2) k = 1;
    return (i - 1) + bx * ((j - 1) + by * (k - 1));
}

static void *xmalloc(size_t n)
{
    void *p = malloc(n ? n : 1);
    return p;
}

orc_case *orc_create(const agal_params *p, int64_t n_maxcblocks, int fp64)
{
    orc_case *c = (orc_case *)calloc(1, sizeof(orc_case));
    if (!c) return NULL;
    c->P = *p;
    c->fp64 = fp64 ? 1 : 0;
    switch (p->velocity_set) {
    case AGAL_D2Q9: c->dim = 2; c->Q = 9; break;
    case AGAL_D3Q19: c->dim = 3; c->Q = 19; break;
    case AGAL_D3Q27: c->dim = 3; c->Q = 27; break;
    default: free(c); return NULL;
    }
    c->Qmax = (c->dim == 2) ? 9 : 27;
    c->MC = (c->dim == 2) ? 16 : 64;
    c->NCH = (c->dim == 2) ? 4 : 8;
    if (c->dim == 2) {
        c->cx = ORC_C2[0]; c->cy = ORC_C2[1]; c->cz = ORC_C2[2];
        c->pb = ORC_PB2; c->w = ORC_W2; c->map = ORC_MAP2;
    } else {
        c->cx = ORC_C3[0]; c->cy = ORC_C3[1]; c->cz = ORC_C3[2];
        c->pb = ORC_PB3; c->w = (c->Q == 19) ? ORC_W19 : ORC_W27; c->map = ORC_MAP3;
    }

    /* mesh_init.cu:22-91 */
    float Lx = (float)p->L_c;
    float Ly = (float)(p->L_fy * Lx);
    float Lz = (float)(p->L_fz * Lx);
    c->Nx = p->Nx;
    c->Ny = (int)(c->Nx * (Ly / Lx));
    c->Nz = (int)(c->Nx * (Lz / Lx));
    if (c->dim == 2) c->Nz = 1;
    c->dx = Lx / (float)c->Nx;
    c->dx_cblock = 4.0f * c->dx;
    c->max_levels = p->MAX_LEVELS_WALL > p->MAX_LEVELS_INTERIOR ? p->MAX_LEVELS_WALL : p->MAX_LEVELS_INTERIOR;
    if (c->max_levels < 1 || c->max_levels > ORC_MAXL) { free(c); return NULL; }
    c->L0 = p->N_LEVEL_START;
    if (c->max_levels == 1) c->L0 = 0;
    if (c->L0 > c->max_levels - 1) c->L0 = c->max_levels - 1;
    for (int L = 0; L < c->max_levels; L++) {
        c->dxf[L] = (float)((double)c->dx / pow(2.0, (double)(float)L));
        c->dxf_d[L] = (double)c->dx / pow(2.0, (double)L);
    }
    /* solver_lbm_init.cu:19-52: tau_L = v0*3 + 0.5*dx_L in ufloat_t */
    for (int L = 0; L < c->max_levels; L++) {
        if (c->fp64) c->tau[L] = p->v0 * 3.0 + 0.5 * c->dxf_d[L];
        else c->tau[L] = (double)(float)(p->v0 * 3.0 + 0.5 * (double)c->dxf[L]);
    }

    int bx = c->Nx / 4, by = c->Ny / 4, bz = (c->dim == 2) ? 1 : c->Nz / 4;
    int64_t n_coarse = (int64_t)bx * by * bz;
    c->nmb = n_maxcblocks;
    if (n_coarse <= 0 || n_coarse > c->nmb) { free(c); return NULL; }
    c->nmc = c->nmb * c->MC;
    const int64_t nmb = c->nmb, nmc = c->nmc;

    c->cells_ID_mask = (int *)xmalloc(sizeof(int) * nmc);
    c->cblock_f_X = (float *)xmalloc(sizeof(float) * c->dim * nmb);
    c->cblock_ID_mask = (int *)xmalloc(sizeof(int) * nmb);
    c->cblock_ID_nbr = (int *)xmalloc(sizeof(int) * c->Qmax * nmb);
    c->cblock_ID_nbr_child = (int *)xmalloc(sizeof(int) * c->Qmax * nmb);
    c->cblock_ID_onb = (int *)xmalloc(sizeof(int) * nmb);
    c->cblock_ID_ref = (int *)xmalloc(sizeof(int) * nmb);
    c->cblock_level = (int *)xmalloc(sizeof(int) * nmb);
    c->id_set = (int *)xmalloc(sizeof(int) * c->max_levels * nmb);
    c->gap_set = (int *)xmalloc(sizeof(int) * nmb);
    size_t es = c->fp64 ? sizeof(double) : sizeof(float);
    c->F = xmalloc(es * (size_t)(c->Q + c->dim + 1) * (size_t)nmc);
    if (!c->cells_ID_mask || !c->cblock_f_X || !c->cblock_ID_mask || !c->cblock_ID_nbr ||
        !c->cblock_ID_nbr_child || !c->cblock_ID_onb || !c->cblock_ID_ref || !c->cblock_level ||
        !c->id_set || !c->gap_set || !c->F) {
        orc_destroy(c);
        return NULL;
    }

    /* Reset values, mesh_init.cu:285-304. */
    for (int64_t i = 0; i < nmc; i++) c->cells_ID_mask[i] = ORC_CELL_INTERIOR;
    for (int64_t i = 0; i < nmb; i++) {
        c->cblock_ID_mask[i] = ORC_BLOCK_REGULAR;
        c->cblock_ID_ref[i] = ORC_REF_INACTIVE;
        c->cblock_level[i] = 0;
        c->cblock_ID_onb[i] = 0;
        c->gap_set[i] = -1;
    }
    for (int64_t i = 0; i < (int64_t)c->Qmax * nmb; i++) {
        c->cblock_ID_nbr[i] = ORC_N_SKIPID;
        c->cblock_ID_nbr_child[i] = ORC_N_SKIPID;
    }
    memset(c->cblock_f_X, 0, sizeof(float) * c->dim * nmb);
    for (int64_t i = 0; i < (int64_t)c->max_levels * nmb; i++) c->id_set[i] = -1;
    if (c->fp64) { double *F = (double *)c->F; for (int64_t i = 0; i < (int64_t)(c->Q + c->dim + 1) * nmc; i++) F[i] = 0.0; }
    else { float *F = (float *)c->F; for (int64_t i = 0; i < (int64_t)(c->Q + c->dim + 1) * nmc; i++) F[i] = 0.0f; }

    /* Root grid: mesh_init.cu:354-516. */
    const int *dcx = (c->dim == 2) ? ORC_C2[0] : ORC_C3[0];
    const int *dcy = (c->dim == 2) ? ORC_C2[1] : ORC_C3[1];
    const int *dcz = (c->dim == 2) ? ORC_C2[2] : ORC_C3[2];
    for (int k = 1; k <= bz; k++)
        for (int j = 1; j <= by; j++)
            for (int i = 1; i <= bx; i++) {
                int b = root_padded_id(c, bx, by, bz, i, j, k);
                c->cblock_f_X[b + 0 * nmb] = (float)(i - 1) * c->dx_cblock;
                c->cblock_f_X[b + 1 * nmb] = (float)(j - 1) * c->dx_cblock;
                if (c->dim == 3) c->cblock_f_X[b + 2 * nmb] = (float)(k - 1) * c->dx_cblock;
                int onb = 0;
                for (int q = 0; q < c->Qmax; q++) {
                    int nb = root_padded_id(c, bx, by, bz, i + dcx[q], j + dcy[q], k + dcz[q]);
                    c->cblock_ID_nbr[b + (int64_t)q * nmb] = nb;
                    if (nb < 0) onb = 1;
                    c->cblock_ID_nbr_child[b + (int64_t)q * nmb] = nb < 0 ? nb : ORC_N_SKIPID;
                }
                c->cblock_ID_onb[b] = onb;
                c->cblock_ID_ref[b] = ORC_REF_UNREFINED;
            }
    for (int L = 0; L <= ORC_MAXL; L++) { c->n_ids[L] = 0; c->id_max[L] = 0; }
    c->n_ids[0] = (int)n_coarse;
    c->id_max[0] = c->id_max[c->max_levels] = (int)n_coarse;
    for (int64_t xi = 0; xi < n_coarse; xi++) c->id_set[xi] = (int)xi;
    for (int64_t xi = 0; xi < nmb - n_coarse; xi++) c->gap_set[xi] = (int)((nmb - 1) - xi);
    c->n_gaps = (int)(nmb - n_coarse);
    return c;
}

void orc_destroy(orc_case *c)
{
    if (!c) return;
    free(c->cells_ID_mask); free(c->cblock_f_X); free(c->cblock_ID_mask);
    free(c->cblock_ID_nbr); free(c->cblock_ID_nbr_child); free(c->cblock_ID_onb);
    free(c->cblock_ID_ref); free(c->cblock_level); free(c->id_set); free(c->gap_set);
    free(c->F);
    free(c);
}

int orc_get_counts(const orc_case *c, int *n_ids, int *id_max, int *n_gaps,
                   int64_t *n_maxcblocks, int *max_levels)
{
    for (int L = 0; L <= c->max_levels; L++) {
        if (n_ids) n_ids[L] = c->n_ids[L];
        if (id_max) id_max[L] = c->id_max[L];
    }
    if (n_gaps) *n_gaps = c->n_gaps;
    if (n_maxcblocks) *n_maxcblocks = c->nmb;
    if (max_levels) *max_levels = c->max_levels;
    return 0;
}

#define DISPATCH(name, ...) (c->fp64 ? name##_f64(__VA_ARGS__) : name##_f32(__VA_ARGS__))

int orc_set_ic(orc_case *c, int L)
{
    if (L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    return DISPATCH(set_ic, c, L);
}
int orc_refresh(orc_case *c, int L)
{
    if (L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    return DISPATCH(refresh, c, L);
}
int orc_collide(orc_case *c, int L)
{
    if (L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    /* S_Collide runs S_RefreshVariables first on a single-level mesh
       (solver_lbm_kernels.cu:469-470); Cu_Collide recomputes the same macros. */
    if (c->max_levels == 1) DISPATCH(refresh, c, L);
    return DISPATCH(collide, c, L);
}
int orc_impose_bc(orc_case *c, int L)
{
    if (L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    return DISPATCH(impose_bc, c, L);
}
int orc_stream(orc_case *c, int L)
{
    if (L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    return DISPATCH(stream, c, L);
}

int orc_advance(orc_case *c, int L)
{
    /* solver_lbm_advance.cu:31-174.  Multi-level sub-cycling is added with the
       interface kernels; the single-level branch is :239-251. */
    if (c->max_levels > 1 && c->max_levels != c->L0 + 1) return AGAL_ERR_UNSUPPORTED;
    int rc;
    if ((rc = orc_collide(c, L))) return rc;
    if ((rc = orc_impose_bc(c, L))) return rc;
    if ((rc = orc_stream(c, L))) return rc;
    return 0;
}

int orc_advance_n(orc_case *c, int n)
{
    for (int i = 0; i < n; i++) {
        int rc = orc_advance(c, c->L0);
        if (rc) return rc;
    }
    return 0;
}

size_t orc_array_bytes(const orc_case *c, int which)
{
    const size_t nmb = (size_t)c->nmb, nmc = (size_t)c->nmc;
    switch (which) {
    case AGAL_ARR_F: return sizeof(double) * (size_t)c->Q * nmc;
    case AGAL_ARR_MACROS: return sizeof(double) * (size_t)(c->dim + 1) * nmc;
    case AGAL_ARR_CELLS_ID_MASK: return sizeof(int) * nmc;
    case AGAL_ARR_CBLOCK_F_X: return sizeof(float) * (size_t)c->dim * nmb;
    case AGAL_ARR_CBLOCK_ID_MASK:
    case AGAL_ARR_CBLOCK_ID_ONB:
    case AGAL_ARR_CBLOCK_ID_REF:
    case AGAL_ARR_CBLOCK_LEVEL:
    case AGAL_ARR_GAP_SET: return sizeof(int) * nmb;
    case AGAL_ARR_CBLOCK_ID_NBR:
    case AGAL_ARR_CBLOCK_ID_NBR_CHILD: return sizeof(int) * (size_t)c->Qmax * nmb;
    case AGAL_ARR_ID_SET: return sizeof(int) * (size_t)c->max_levels * nmb;
    default: return 0;
    }
}

static const void *int_array(const orc_case *c, int which)
{
    switch (which) {
    case AGAL_ARR_CELLS_ID_MASK: return c->cells_ID_mask;
    case AGAL_ARR_CBLOCK_F_X: return c->cblock_f_X;
    case AGAL_ARR_CBLOCK_ID_MASK: return c->cblock_ID_mask;
    case AGAL_ARR_CBLOCK_ID_NBR: return c->cblock_ID_nbr;
    case AGAL_ARR_CBLOCK_ID_NBR_CHILD: return c->cblock_ID_nbr_child;
    case AGAL_ARR_CBLOCK_ID_ONB: return c->cblock_ID_onb;
    case AGAL_ARR_CBLOCK_ID_REF: return c->cblock_ID_ref;
    case AGAL_ARR_CBLOCK_LEVEL: return c->cblock_level;
    case AGAL_ARR_ID_SET: return c->id_set;
    case AGAL_ARR_GAP_SET: return c->gap_set;
    default: return NULL;
    }
}

int orc_dump(const orc_case *c, int which, void *buf, size_t bytes)
{
    size_t need = orc_array_bytes(c, which);
    if (!need || bytes != need || !buf) return AGAL_ERR_PARAM;
    if (which == AGAL_ARR_F || which == AGAL_ARR_MACROS) {
        size_t off = (which == AGAL_ARR_F) ? 0 : (size_t)c->Q * (size_t)c->nmc;
        size_t n = need / sizeof(double);
        double *o = (double *)buf;
        if (c->fp64) memcpy(o, (const double *)c->F + off, need);
        else { const float *F = (const float *)c->F + off; for (size_t i = 0; i < n; i++) o[i] = (double)F[i]; }
        return 0;
    }
    memcpy(buf, int_array(c, which), need);
    return 0;
}

int orc_load(orc_case *c, int which, const void *buf, size_t bytes)
{
    size_t need = orc_array_bytes(c, which);
    if (!need || bytes != need || !buf) return AGAL_ERR_PARAM;
    if (which == AGAL_ARR_F || which == AGAL_ARR_MACROS) {
        size_t off = (which == AGAL_ARR_F) ? 0 : (size_t)c->Q * (size_t)c->nmc;
        size_t n = need / sizeof(double);
        const double *in = (const double *)buf;
        if (c->fp64) memcpy((double *)c->F + off, in, need);
        else { float *F = (float *)c->F + off; for (size_t i = 0; i < n; i++) F[i] = (float)in[i]; }
        return 0;
    }
    memcpy((void *)int_array(c, which), buf, need);
    return 0;
}

int orc_mass_momentum(orc_case *c, double *out)
{
    if (c->fp64) mass_momentum_f64(c, out); else mass_momentum_f32(c, out);
    return 0;
}
