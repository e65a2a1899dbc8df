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
    c->emap = (int *)xmalloc(sizeof(int) * nmb);
    c->first_child = (int *)xmalloc(sizeof(int) * nmb);
    size_t es = c->fp64 ? sizeof(double) : sizeof(float);
    c->F = xmalloc(es * (size_t)(c->Q + c->dim + 1) * (size_t)nmc);
    if (!c->cells_ID_mask || !c->cblock_f_X || !c->cblock_ID_mask || !c->cblock_ID_nbr ||
        !c->cblock_ID_nbr_child || !c->cblock_ID_onb || !c->cblock_ID_ref || !c->cblock_level ||
        !c->id_set || !c->gap_set || !c->F || !c->emap || !c->first_child) {
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
        c->gap_set[i] = 0;
        c->emap[i] = -1;
        c->first_child[i] = -1;
    }
    for (int64_t i = 0; i < (int64_t)c->Qmax * nmb; i++) {
        c->cblock_ID_nbr[i] = ORC_N_SKIPID;
        c->cblock_ID_nbr_child[i] = ORC_N_SKIPID;
    }
    memset(c->cblock_f_X, 0, sizeof(float) * c->dim * nmb);
    /* The reference never initialises id_set beyond level 0 (fresh, zeroed
       device memory); max_element over an empty level reads its first slot
       (mesh_amr.cu:2630), so the initial contents matter for id_max. */
    for (int64_t i = 0; i < (int64_t)c->max_levels * nmb; i++) c->id_set[i] = 0;
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
    /* Voxelizer scratch and solid-boundary state (mesh_init.cu:241-286:
       the upper half of cells_ID_mask starts INTERIOR; c_tmp_1/2 are -1
       after M_ResetIntermediateAMRArraysV1, mesh_amr.cu:2077-2085). */
    if (orc_geometry_alloc(c)) { orc_destroy(c); return NULL; }
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
    free(c->F); free(c->emap); free(c->first_child);
    orc_geometry_free(c);
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

int orc_set_counts(orc_case *c, const int *n_ids, const int *id_max, int n_gaps)
{
    /* Host counts of a restart (mesh_restart.cu:111-121). */
    for (int L = 0; L <= c->max_levels; L++) {
        if (n_ids[L] < 0 || n_ids[L] > c->nmb || id_max[L] > c->nmb) return AGAL_ERR_PARAM;
        c->n_ids[L] = n_ids[L];
        c->id_max[L] = id_max[L];
    }
    if (n_gaps < 0 || n_gaps > c->nmb) return AGAL_ERR_PARAM;
    c->n_gaps = n_gaps;
    return 0;
}

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

int orc_interpolate(orc_case *c, int L, int var)
{
    /* S_Interpolate_*: refresh level L, then interpolate (kernels_comm.cu:141-155, 642-658). */
    if (L < 0 || L >= c->max_levels - 1) return AGAL_ERR_PARAM;
    int rc = orc_refresh(c, L);
    if (rc) return rc;
    if (c->n_ids[L] <= 0) return 0;
    return DISPATCH(interpolate, c, L, var);
}

int orc_average(orc_case *c, int L, int var)
{
    /* S_Average: refresh level L+1, then average (kernels_comm.cu:351-370). */
    if (L < 0 || L >= c->max_levels - 1) return AGAL_ERR_PARAM;
    int rc = orc_refresh(c, L + 1);
    if (rc) return rc;
    if (c->n_ids[L] <= 0) return 0;
    return DISPATCH(average, c, L, var);
}

int orc_ref_criteria(orc_case *c)
{
    if (c->P.S_CRITERION == AGAL_CRITERION_PERCENTILE) return DISPATCH(ref_criteria_pct, c);
    return DISPATCH(ref_criteria, c);
}

static int avg_mode(const orc_case *c)
{
    /* solver_lbm_init.cu:94-97 */
    return (c->P.interp_order != AGAL_INTERP_LINEAR) ? AGAL_AVERAGE_BLOCK : AGAL_AVERAGE_INTERFACE;
}

static int sub_step_f(orc_case *c, int L, int forces)
{
    /* Collide, [MEA before the stream], BC, stream, [MEA after]
       (solver_lbm_advance.cu:115-126, 141-148). */
    int rc;
    if ((rc = orc_collide(c, L))) return rc;
    if (forces && (rc = DISPATCH(forces_mea, c, L, 0))) return rc;
    if ((rc = orc_impose_bc(c, L))) return rc;
    if ((rc = orc_stream(c, L))) return rc;
    if (forces && (rc = DISPATCH(forces_mea, c, L, 1))) return rc;
    return 0;
}

static int sub_step(orc_case *c, int L) { return sub_step_f(c, L, 0); }

int orc_forces(orc_case *c, double *out)
{
    /* Solver_LBM::S_ReportForces sums (solver_lbm_compute.cu:166-215):
       out = {Fpx, Fmx, Fpy, Fmy, Fpz, Fmz}; the partials are then reset. */
    DISPATCH(forces_sum, c, out);
    memset(c->Ff, 0, (size_t)6 * c->nmb * (c->fp64 ? sizeof(double) : sizeof(float)));
    return 0;
}

int orc_advance(orc_case *c, int L)
{
    /* Solver_LBM::S_Advance (solver_lbm_advance.cu:31-174). */
    const int ML = c->max_levels;
    int rc;
    const int mea = c->P.S_FORCE_TYPE == 0;
    if (!(ML > 1 && ML != c->L0 + 1)) return sub_step_f(c, L, mea);   /* :239-251 */
    if (L == c->L0) {                                           /* :39-58 */
        c->liter = 0;
        if ((rc = orc_interpolate(c, L, AGAL_INTERP_INTERFACE))) return rc;
        if ((rc = sub_step(c, L))) return rc;
        if ((rc = orc_advance(c, L + 1))) return rc;
        return orc_average(c, L, avg_mode(c));
    }
    if (L < ML - 1 && (rc = orc_interpolate(c, L, AGAL_INTERP_INTERFACE))) return rc;   /* :96-99 */
    if ((rc = sub_step(c, L))) return rc;
    if (L == ML - 1) c->liter++;
    if (L < ML - 1) {                                                                   /* :106-111 */
        if ((rc = orc_advance(c, L + 1))) return rc;
        if ((rc = orc_average(c, L, avg_mode(c)))) return rc;
        if ((rc = orc_interpolate(c, L, AGAL_INTERP_INTERFACE))) return rc;
    }
    /* :114-126: MEA on the last finest sub-step of the coarse step. */
    if ((rc = sub_step_f(c, L, mea && L == ML - 1 && c->liter == (1 << (ML - 1)) - 1))) return rc;
    if (L == ML - 1) c->liter++;
    if (L < ML - 1) {                                                                   /* :130-134 */
        if ((rc = orc_advance(c, L + 1))) return rc;
        if ((rc = orc_average(c, L, avg_mode(c)))) return rc;
    }
    return 0;
}

/* ---- refinement / coarsening (mesh_amr.cu:2162-2744) ---------------------- */

/* Index of the direction with velocity (ex, ey, ez) in the neighbour table. */
static int dir_index(const orc_case *c, int ex, int ey, int ez)
{
    const int *dx = (c->dim == 2) ? ORC_C2[0] : ORC_C3[0];
    const int *dy = (c->dim == 2) ? ORC_C2[1] : ORC_C3[1];
    const int *dz = (c->dim == 2) ? ORC_C2[2] : ORC_C3[2];
    for (int q = 0; q < c->Qmax; q++)
        if (dx[q] == ex && dy[q] == ey && dz[q] == ez) return q;
    return -1;
}

static int floordiv2(int t) { return (t >= 0) ? t / 2 : -1; }   /* t in {-1..2} */

int orc_refine_coarsen(orc_case *c)
{
    const int64_t nmb = c->nmb;
    const int Qmax = c->Qmax, NCH = c->NCH, ML = c->max_levels, dim = c->dim;
    int *ref = c->cblock_ID_ref, *nbr = c->cblock_ID_nbr, *nch = c->cblock_ID_nbr_child;
    const int idm = c->id_max[ML];
    int nR = 0, nC = 0;
    for (int b = 0; b < idm; b++) {
        nR += (ref[b] == ORC_REF_MARK_REFINE);
        nC += (ref[b] == ORC_REF_MARK_COARSEN);
    }
    /* :2186, :2341; the sum can pass n_maxcblocks on a nearly full pool
       although every ID lies below it: the passes stop at n_maxcblocks. */
    int idm_wnew = (int)(((int64_t)idm + (int64_t)NCH * nR) < nmb ? idm + NCH * nR : nmb);
    int proceed_ref = nR > 0 && NCH * nR <= c->n_gaps;
    int proceed_coarse = nC > 0;
    if (!proceed_ref && nR > 0) {                                   /* :2197-2205 */
        nR = 0;
        idm_wnew = idm;
        for (int b = 0; b < idm_wnew; b++)
            if (ref[b] == ORC_REF_MARK_REFINE) ref[b] = ORC_REF_UNREFINED;
    }
    /* S1 (:2225-2307): efficient map = marked blocks and their neighbours. */
    if (proceed_ref || proceed_coarse) {
        for (int b = 0; b < idm; b++) {
            if (ref[b] != ORC_REF_MARK_REFINE && ref[b] != ORC_REF_MARK_COARSEN) continue;
            int self = nbr[b];
            if (self >= 0) c->emap[self] = self;
            for (int p = 1; p < Qmax; p++) {
                int nb = nbr[b + (int64_t)p * nmb];
                if (nb >= 0) c->emap[nb] = nb;
            }
        }
    }
    /* S2 (:2326-2370): first-child IDs from the end of the gap stack. */
    if (proceed_ref) {
        int *rev = (int *)malloc(sizeof(int) * (size_t)NCH * nR);
        for (int k = 0; k < NCH * nR; k++) rev[k] = c->gap_set[c->n_gaps - 1 - k];
        int mx = rev[0];
        for (int k = 1; k < NCH * nR; k++) mx = rev[k] > mx ? rev[k] : mx;
        if (mx + 1 > idm_wnew) idm_wnew = (mx + 1 < nmb) ? mx + 1 : (int)nmb;
        int i = 0;
        for (int b = 0; b < idm; b++)
            if (ref[b] == ORC_REF_MARK_REFINE) c->first_child[b] = rev[NCH * (i++)];
        free(rev);
        /* Cu_RefineCells_S2_1 (:1602-1669) */
        for (int b = 0; b < idm; b++) {
            if (c->emap[b] < 0) continue;
            for (int d = 0; d < Qmax; d++) {
                int nb = nbr[b + (int64_t)d * nmb];
                if (nb > -1 && ref[nb] == ORC_REF_MARK_REFINE) nch[b + (int64_t)d * nmb] = c->first_child[nb];
            }
        }
    }
    /* S3 (:2384-2425): 2:1 quality control of coarsening. */
    if (proceed_coarse) {
        for (int b = 0; b < idm; b++) {                              /* Q1_1 (:1401) */
            if (ref[b] != ORC_REF_UNREFINED) continue;
            for (int p = 1; p < Qmax; p++)
                if (nch[b + (int64_t)p * nmb] >= 0) { ref[b] = ORC_REF_UNREFINED_VIO; break; }
        }
        for (int b = 0; b < idm; b++) {                              /* Q1_2 (:1429) */
            if (ref[b] != ORC_REF_MARK_COARSEN) continue;
            int ic = nch[b];
            int vio = 0;
            for (int x = 0; x < NCH; x++) {
                int r = ref[ic + x];
                if (r == ORC_REF_UNREFINED_VIO || r == ORC_REF_MARK_REFINE) vio = 1;
            }
            if (vio) ref[b] = ORC_REF_REFINED;
        }
        nC = 0;
        for (int b = 0; b < idm; b++) nC += (ref[b] == ORC_REF_MARK_COARSEN);
        proceed_coarse = nC > 0;
        if (proceed_coarse) {                                         /* S2_2 (:1671) */
            for (int b = 0; b < idm; b++) {
                if (c->emap[b] < 0) continue;
                for (int d = 1; d < Qmax; d++) {
                    int nb = nbr[b + (int64_t)d * nmb];
                    if (nb > -1 && ref[nb] == ORC_REF_MARK_COARSEN) nch[b + (int64_t)d * nmb] = ORC_N_SKIPID;
                }
            }
        }
    }
    /* S4 (:2441-2457): Cu_AddRemoveBlocks (:1495). */
    if (proceed_ref || proceed_coarse) {
        /* Parents are visited before their children are written; new child
           IDs are free gaps and children of coarsened blocks are leaves, so
           the order of the block loop does not matter. */
        int *snap = (int *)malloc(sizeof(int) * (size_t)(idm > 0 ? idm : 1));
        memcpy(snap, ref, sizeof(int) * (size_t)idm);
        for (int b = 0; b < idm; b++) {
            if (snap[b] == ORC_REF_MARK_REFINE) {
                int f = c->first_child[b];
                nch[b] = f;
                int lev = c->cblock_level[b] + 1;
                float h = c->dx_cblock / (float)(1 << lev);
                for (int x = 0; x < NCH; x++) {
                    int ch = f + x;
                    c->cblock_level[ch] = lev;
                    ref[ch] = ORC_REF_NEW;
                    c->cblock_f_X[ch] = c->cblock_f_X[b] + (float)(unsigned)(x % 2) * h;
                    c->cblock_f_X[ch + nmb] = c->cblock_f_X[b + nmb] + (float)(unsigned)((x / 2) % 2) * h;
                    if (dim == 3) c->cblock_f_X[ch + 2 * nmb] = c->cblock_f_X[b + 2 * nmb] + (float)(unsigned)((x / 4) % 2) * h;
                    nch[ch] = ORC_N_SKIPID;
                }
            }
            if (snap[b] == ORC_REF_MARK_COARSEN) {
                int f = nch[b];
                nch[b] = ORC_N_SKIPID;
                for (int x = 0; x < NCH; x++) ref[f + x] = ORC_REF_REMOVE;
            }
        }
        free(snap);
    }
    /* S5 (:2471-2538): remove children of coarsened blocks from the ID sets,
       push their IDs back on the gap stack. */
    if (proceed_coarse) {
        int nrem = 0;
        int *rem = (int *)malloc(sizeof(int) * (size_t)(idm_wnew > 0 ? idm_wnew : 1));
        for (int L = 1; L < ML; L++)          /* stable sort by level of an ascending list */
            for (int b = 0; b < idm_wnew; b++)
                if (ref[b] == ORC_REF_REMOVE && c->cblock_level[b] == L) rem[nrem++] = b;
        int prev = 0;
        for (int L = 1; L < ML; L++) {
            int cnt = 0;
            while (prev + cnt < nrem && c->cblock_level[rem[prev + cnt]] == L) cnt++;
            if (cnt == 0) continue;
            int *ids = &c->id_set[(int64_t)L * nmb];
            int n = c->n_ids[L], w = 0;
            for (int k = 0; k < n; k++) {     /* Cu_CoarsenCells_S1 + remove_if (tail keeps old values) */
                int v = ids[k];
                int removed = 0;
                for (int r = 0; r < cnt; r++)
                    if (v == rem[prev + r]) removed = 1;
                if (removed) ids[k] = ORC_N_SKIPID;
            }
            for (int k = 0; k < n; k++)
                if (ids[k] != ORC_N_SKIPID) ids[w++] = ids[k];
            c->n_ids[L] -= cnt;
            prev += cnt;
        }
        for (int k = 0; k < prev; k++)        /* Cu_ConcatReverse (:40) */
            c->gap_set[c->n_gaps - NCH * nR + k] = rem[prev - 1 - k];
        c->n_gaps += prev;
        for (int b = 0; b < idm; b++) {       /* Cu_CoarsenCells_S2 (:1861) */
            if (ref[b] != ORC_REF_REMOVE) continue;
            for (int p = 0; p < Qmax; p++) {
                if (p > 0) nbr[b + (int64_t)p * nmb] = ORC_N_SKIPID;
                nch[b + (int64_t)p * nmb] = ORC_N_SKIPID;
            }
        }
        free(rem);
    }
    /* S6 (:2552-2611): insert the new children into the ID sets. */
    if (proceed_ref) {
        for (int L = 1; L < ML; L++) {
            int *ids = &c->id_set[(int64_t)L * nmb];
            int cnt = 0;
            for (int b = 0; b < idm_wnew; b++)
                if (ref[b] == ORC_REF_NEW && c->cblock_level[b] == L) ids[c->n_ids[L] + cnt++] = b;
            if (cnt == 0) continue;
            c->n_ids[L] += cnt;
            /* thrust::sort of the level's set (unique IDs): insertion sort */
            for (int i = 1; i < c->n_ids[L]; i++) {
                int v = ids[i], j = i - 1;
                while (j >= 0 && ids[j] > v) { ids[j + 1] = ids[j]; j--; }
                ids[j + 1] = v;
            }
        }
        c->n_gaps -= NCH * nR;
    }
    /* S7 (:2627-2651). */
    if (proceed_ref || proceed_coarse) {
        for (int L = 1; L < ML; L++) {       /* max_element; an empty level reads slot 0 */
            const int *ids = &c->id_set[(int64_t)L * nmb];
            int mx = ids[0];
            for (int k = 1; k < c->n_ids[L]; k++) mx = ids[k] > mx ? ids[k] : mx;
            c->id_max[L] = mx + 1;
        }
        int mx = c->id_max[0];
        for (int L = 1; L < ML; L++) mx = c->id_max[L] > mx ? c->id_max[L] : mx;
        c->id_max[ML] = mx;
        const int idmN = c->id_max[ML];
        for (int b = 0; b < idmN; b++) {     /* Cu_UpdateMasks_1 (:948) */
            if (ref[b] == ORC_REF_INACTIVE) continue;
            int m = ORC_BLOCK_REGULAR;
            if (nch[b] > -1)
                for (int p = 1; p < Qmax; p++)
                    if (nch[b + (int64_t)p * nmb] == ORC_N_SKIPID) m = ORC_BLOCK_INTERFACE;
            if (c->cblock_ID_mask[b] > -1) c->cblock_ID_mask[b] = m;
        }
        for (int L = 0; L < ML - 1; L++) {   /* M_Interpolate(V_INTERP_ADDED) */
            int rc = orc_interpolate(c, L, AGAL_INTERP_ADDED);
            if (rc) return rc;
        }
        for (int b = 0; b < idm_wnew; b++) { /* Cu_RefineCells_S3 (:1731) */
            int r = ref[b];
            if (r == ORC_REF_MARK_REFINE) ref[b] = ORC_REF_REFINED;
            if (r == ORC_REF_NEW || r == ORC_REF_MARK_COARSEN) ref[b] = ORC_REF_UNREFINED;
            if (r == ORC_REF_REMOVE) ref[b] = ORC_REF_INACTIVE;
            if (r == ORC_REF_UNREFINED_VIO) ref[b] = ORC_REF_UNREFINED;
        }
        int *snap = (int *)malloc(sizeof(int) * (size_t)(idm_wnew > 0 ? idm_wnew : 1));
        memcpy(snap, ref, sizeof(int) * (size_t)idm_wnew);
        for (int b = 0; b < idm_wnew; b++) { /* Cu_RefineCells_S4 (:1774) */
            if (snap[b] != ORC_REF_REFINED && snap[b] != ORC_REF_REFINED_WCHILD) continue;
            int ic = nch[b], nr = ORC_REF_REFINED;
            for (int x = 0; x < NCH; x++) {
                int r = (ic + x < idm_wnew) ? snap[ic + x] : ref[ic + x];
                if (r == ORC_REF_REFINED || r == ORC_REF_REFINED_WCHILD) nr = ORC_REF_REFINED_WCHILD;
            }
            ref[b] = nr;
        }
        free(snap);
    }
    /* S8 (:2668-2700). */
    if (proceed_ref || proceed_coarse) {
        const int idmN = c->id_max[ML];
        int qv[8][27], qi[8][27];             /* child x direction -> (parent direction, child offset) */
        const int *dx = (dim == 2) ? ORC_C2[0] : ORC_C3[0];
        const int *dy = (dim == 2) ? ORC_C2[1] : ORC_C3[1];
        const int *dz = (dim == 2) ? ORC_C2[2] : ORC_C3[2];
        for (int x = 0; x < NCH; x++)
            for (int d = 0; d < Qmax; d++) {
                int tx = (x & 1) + dx[d], ty = ((x >> 1) & 1) + dy[d], tz = ((x >> 2) & 1) + dz[d];
                qv[x][d] = dir_index(c, floordiv2(tx), floordiv2(ty), dim == 3 ? floordiv2(tz) : 0);
                qi[x][d] = (tx & 1) + 2 * (ty & 1) + (dim == 3 ? 4 * (tz & 1) : 0);
            }
        for (int b = 0; b < idmN; b++) {     /* Cu_UpdateConnectivity (:156) */
            if (!(c->emap[b] > -1 && nch[b] > -1)) continue;
            int f = nch[b];
            for (int x = 0; x < NCH; x++)
                for (int d = 0; d < Qmax; d++) {
                    int v = nch[b + (int64_t)qv[x][d] * nmb];
                    nbr[(f + x) + (int64_t)d * nmb] = (v < 0) ? v : v + qi[x][d];
                }
        }
        for (int b = 0; b < idmN; b++) {     /* Cu_UpdateBoundaries (:106) */
            int on = 0;
            for (int p = 1; p < Qmax; p++) {
                int v = nbr[b + (int64_t)p * nmb];
                if (v < 0) {
                    nch[b + (int64_t)p * nmb] = v;
                    if (v != ORC_N_SKIPID) on = 1;
                }
            }
            if (c->cblock_ID_mask[b] == ORC_BLOCK_SOLIDA) on = 1;
            c->cblock_ID_onb[b] = on;
        }
        for (int b = 0; b < idmN; b++) {     /* Cu_UpdateMasks_2 (:983) */
            if (ref[b] == ORC_REF_INACTIVE) continue;
            int skip[27], any = 0;
            for (int p = 1; p < Qmax; p++) { skip[p] = (nbr[b + (int64_t)p * nmb] == ORC_N_SKIPID); any |= skip[p]; }
            for (int t = 0; t < c->MC; t++) {
                int64_t o = (int64_t)b * c->MC + t;
                if (c->cells_ID_mask[o] < 0) continue;
                int I = t % 4, J = (t / 4) % 4, K = (dim == 3) ? (t / 4) / 4 : 0;
                int m = any ? 1 : 0;
                for (int p = 1; p < Qmax; p++) {
                    if (!skip[p]) continue;
                    int in = 1;
                    if (dx[p] > 0 && !(I >= 2)) in = 0;
                    if (dx[p] < 0 && !(I < 2)) in = 0;
                    if (dy[p] > 0 && !(J >= 2)) in = 0;
                    if (dy[p] < 0 && !(J < 2)) in = 0;
                    if (dim == 3 && dz[p] > 0 && !(K >= 2)) in = 0;
                    if (dim == 3 && dz[p] < 0 && !(K < 2)) in = 0;
                    if (in) m = 2;
                }
                c->cells_ID_mask[o] = m;
            }
        }
        for (int b = 0; b < idmN; b++) c->emap[b] = -1;
    }
    for (int b = 0; b < idm_wnew && b < nmb; b++) c->first_child[b] = -1;
    c->n_ref_last = nR;
    c->n_coarse_last = proceed_coarse ? nC : 0;
    return 0;
}

int orc_refine_with_solution(orc_case *c)
{
    /* Mesh::M_Advance_RefineWithSolution (mesh_advance.cu:185-243). */
    const int ML = c->max_levels;
    int rc;
    if (!(c->P.MAX_LEVELS_INTERIOR > 1 && c->P.N_PROBE_AVE == 0)) return 0;
    for (int L = ML - 2; L >= c->L0; L--)
        if ((rc = orc_average(c, L, AGAL_AVERAGE_GRID))) return rc;
    for (int L = c->L0; L < ML - 1; L++)
        if ((rc = orc_interpolate(c, L, AGAL_INTERP_INTERFACE))) return rc;
    if ((rc = orc_ref_criteria(c))) return rc;
    return orc_refine_coarsen(c);
}

/* Cu_RefineRegion presets on the block bounds of mesh_criterion.cu:28-33. */
static int in_region(const orc_case *c, int b, float dxb)
{
    const int64_t nmb = c->nmb;
    const float *fX = c->cblock_f_X;
    switch (c->P.region_preset) {
    case AGAL_REGION_BOUNDARY: return c->cblock_ID_onb[b] == 1;
    case AGAL_REGION_BOX: {
        for (int d = 0; d < c->dim; d++) {
            const float lo = fX[b + d * nmb] + 1e-5f;
            const float hi = fX[b + d * nmb] + dxb - 1e-5f;
            if (!(lo >= 0.25f && hi <= 0.75f)) return 0;
        }
        return 1;
    }
    default: return 0;
    }
}

static void mark_level(orc_case *c, int L, int uniform)
{
    /* Cu_ComputeRefCriteria_Uniform / _NearWall_Cases (mesh_criterion.cu:10-85). */
    const int *ids = &c->id_set[(int64_t)L * c->nmb];
    const float dxb = c->dxf[L] * 4.0f;
    for (int k = 0; k < c->n_ids[L]; k++) {
        const int b = ids[k];
        if (c->cblock_ID_ref[b] != ORC_REF_UNREFINED) continue;
        if (uniform || in_region(c, b, dxb)) c->cblock_ID_ref[b] = ORC_REF_MARK_REFINE;
    }
}

int orc_refine_near_wall(orc_case *c)
{
    /* Mesh::M_Advance_RefineNearWall (mesh_advance.cu:54-122), with the
       voxelizer passes when a geometry is attached. */
    const int ML = c->max_levels, MLW = c->P.MAX_LEVELS_WALL;
    const int geo = c->geometry_init;
    int rc;
    for (int L = 0; L < c->L0; L++) {
        mark_level(c, L, 1);
        if ((rc = orc_refine_coarsen(c))) return rc;
    }
    for (int L = c->L0; L < MLW; L++) {
        if (L < MLW - 1) mark_level(c, L, 0);
        if (geo && (rc = orc_voxelize_s1(c, L))) return rc;
        if (ML > 1 && L < MLW - 1 && (rc = orc_refine_coarsen(c))) return rc;
        if (geo && (rc = orc_update_solid_children(c, L))) return rc;
        if ((rc = orc_set_ic(c, L))) return rc;
    }
    if (geo) {
        for (int L = c->L0; L < MLW; L++)
            if ((rc = orc_voxelize_s2(c, L))) return rc;
        if ((rc = orc_voxelize_s3(c))) return rc;
        if (c->P.G_BIN_MAKE_LINKS)
            for (int L = c->L0; L < MLW; L++)
                if ((rc = orc_link_lengths(c, L))) return rc;
    }
    if (ML > 1) {
        /* M_FreezeRefinedCells(0): Cu_FreezeRefined over id_max[MAX_LEVELS] (mesh_amr.cu:1888-1904). */
        for (int b = 0; b < c->id_max[ML]; b++) {
            if (c->cblock_ID_ref[b] == ORC_REF_REFINED) c->cblock_ID_ref[b] = ORC_REF_REFINED_PERM;
            if (c->cblock_ID_ref[b] == ORC_REF_REFINED_WCHILD) c->cblock_ID_ref[b] = ORC_REF_REFINED_WCHILD_PERM;
        }
    }
    return 0;
}

int orc_advance_n(orc_case *c, int n)
{
    /* Loop body of Mesh::M_AdvanceLoop (mesh_advance.cu:421-463). */
    const int ML = c->max_levels;
    const int iter_mult = 1 << c->L0;
    for (int s = 0; s < n; s++) {
        const long i = c->iter;
        for (int j = 0; j < iter_mult; j++) {
            int rc = orc_advance(c, c->L0);
            if (rc) return rc;
        }
        if (ML > 1 && ML != c->L0 + 1 && (i + 1) % c->P.P_REFINE == 0 && i > 0) {
            int rc = orc_refine_with_solution(c);
            if (rc) return rc;
        }
        c->iter++;
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
    case AGAL_ARR_CBLOCK_ID_ONB_SOLID: return sizeof(int) * nmb;
    case AGAL_ARR_CELLS_F_X_B: return c->X_b ? sizeof(float) * (size_t)c->Qmax * (size_t)c->n_maxcells_b : 0;
    case AGAL_ARR_CBLOCK_F_FF: return sizeof(double) * 6 * nmb;
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
    case AGAL_ARR_CBLOCK_ID_ONB_SOLID: return c->onb_solid;
    case AGAL_ARR_CELLS_F_X_B: return c->X_b;
    default: return NULL;
    }
}

int orc_dump(const orc_case *c, int which, void *buf, size_t bytes)
{
    size_t need = orc_array_bytes(c, which);
    if (!need || bytes != need || !buf) return AGAL_ERR_PARAM;
    if (which == AGAL_ARR_CBLOCK_F_FF) {
        double *o = (double *)buf;
        for (size_t i = 0; i < 6 * (size_t)c->nmb; i++)
            o[i] = c->fp64 ? ((const double *)c->Ff)[i] : (double)((const float *)c->Ff)[i];
        return 0;
    }
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
    if (which == AGAL_ARR_CBLOCK_F_FF) {
        const double *in = (const double *)buf;
        for (size_t i = 0; i < 6 * (size_t)c->nmb; i++) {
            if (c->fp64) ((double *)c->Ff)[i] = in[i];
            else ((float *)c->Ff)[i] = (float)in[i];
        }
        return 0;
    }
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
