/*
 * ORACLE (test infrastructure only): CPU restatement of AGAL's geometry
 * chain - triangle binning (geometry_bins_gpu.cu), voxelization and
 * near-wall block marking (mesh_voxelizer*.cu) and link lengths
 * (mesh_voxelizer_links.cu) - for 3D cases.
 *
 * The reference evaluates this geometry in FP32 on the device, where the
 * compiler fuses a multiply into the add or subtract that consumes it.  The
 * vector helpers below spell that fusion out with fmaf() in the pattern
 * a*b + c*d -> fma(a, b, c*d), a*b - c*d -> fma(a, b, -(c*d)) (the first
 * product fused), so that the restatement rounds like the reference build;
 * ORC_GEO_FMA=0 selects plain rounding of every operation instead.  Parity
 * is pinned by the fixtures tests/golden/geom_*.npz written by the
 * reference's own build.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "orc_internal.h"

#ifndef ORC_GEO_FMA
#define ORC_GEO_FMA 1
#endif

typedef struct { float x, y, z; } v3;

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsubs(v3 a, float s) { return V(a.x - s, a.y - s, a.z - s); }
static inline v3 vadds(v3 a, float s) { return V(a.x + s, a.y + s, a.z + s); }
static inline v3 vmuls(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }

/* a*b + c*d */
static inline float pr2(float a, float b, float c, float d)
{
#if ORC_GEO_FMA
    return fmaf(a, b, c * d);
#else
    return a * b + c * d;
#endif
}
/* a*b - c*d */
static inline float pd2(float a, float b, float c, float d)
{
#if ORC_GEO_FMA
    return fmaf(a, b, -(c * d));
#else
    return a * b - c * d;
#endif
}
/* s + a*b */
static inline float acc(float s, float a, float b)
{
#if ORC_GEO_FMA
    return fmaf(a, b, s);
#else
    return s + a * b;
#endif
}

/* DotV, CrossV, NormV, UnitV (inc/util.h:367-406). */
static inline float dotv(v3 a, v3 b) { return acc(pr2(a.x, b.x, a.y, b.y), a.z, b.z); }
static inline v3 crossv(v3 a, v3 b)
{
    return V(pd2(a.y, b.z, a.z, b.y), pd2(a.z, b.x, a.x, b.z), pd2(a.x, b.y, a.y, b.x));
}
static inline v3 unitv(v3 a)
{
    const float onorm = 1.0f / sqrtf(dotv(a, a));
    return vmuls(a, onorm);
}
/* FaceNormal / FaceNormalUnit in 3D (util.h:419-432). */
static inline v3 face_normal(v3 v1, v3 v2, v3 v3_) { return crossv(vsub(v2, v1), vsub(v3_, v1)); }
static inline v3 face_normal_unit(v3 v1, v3 v2, v3 v3_) { return unitv(face_normal(v1, v2, v3_)); }

static inline void load_face(const orc_case *c, int f, v3 *v1, v3 *v2, v3 *v3_)
{
    const float *X = c->faces;
    const int64_t n = c->n_faces;
    *v1 = V(X[f + 0 * n], X[f + 1 * n], X[f + 2 * n]);
    *v2 = V(X[f + 3 * n], X[f + 4 * n], X[f + 5 * n]);
    *v3_ = V(X[f + 6 * n], X[f + 7 * n], X[f + 8 * n]);
}

/* TriangleBinOverlap2D_AxisGap (util_tribin.h:92-125): true when the
   projections on axis `axis` of the triangle and of the box are disjoint. */
static int axis_gap(int axis, float v1x, float v1y, float v2x, float v2y, float v3x, float v3y,
                    float rmx, float rmy, float rMx, float rMy)
{
    float ex = 0.0f, ey = 0.0f;
    if (axis == 0) { ex = 1.0f; ey = 0.0f; }
    if (axis == 1) { ex = 0.0f; ey = 1.0f; }
    if (axis == 2) { ex = v2y - v1y; ey = v1x - v2x; }
    if (axis == 3) { ex = v3y - v2y; ey = v2x - v3x; }
    if (axis == 4) { ex = v1y - v3y; ey = v3x - v1x; }
    float t = fmaxf(fmaxf(pr2(v1x, ex, v1y, ey), pr2(v2x, ex, v2y, ey)), pr2(v3x, ex, v3y, ey));
    float r = fminf(fminf(fminf(pr2(rmx, ex, rmy, ey), pr2(rMx, ex, rmy, ey)), pr2(rmx, ex, rMy, ey)),
                    pr2(rMx, ex, rMy, ey));
    int b = t < r;
    t = fminf(fminf(pr2(v1x, ex, v1y, ey), pr2(v2x, ex, v2y, ey)), pr2(v3x, ex, v3y, ey));
    r = fmaxf(fmaxf(fmaxf(pr2(rmx, ex, rmy, ey), pr2(rMx, ex, rmy, ey)), pr2(rmx, ex, rMy, ey)),
              pr2(rMx, ex, rMy, ey));
    return b || (r < t);
}

/* TrianglePlaneCutsBox (util_tribin.h:60-74). */
static int plane_cuts_box(v3 vm, v3 vM, v3 v1, v3 v2, v3 v3_)
{
    const v3 n = face_normal(v1, v2, v3_);
    const v3 cc = V(n.x > 0 ? (vM.x - vm.x) : 0.0f, n.y > 0 ? (vM.y - vm.y) : 0.0f, n.z > 0 ? (vM.z - vm.z) : 0.0f);
    const float d = dotv(n, vm);
    const float d1 = dotv(n, vsub(cc, v1));
    const float d2 = dotv(n, vsub(vsub(vsub(vM, vm), cc), v1));
    return (d + d1) * (d + d2) <= 0;
}

/* TriangleBinOverlap3D (util_tribin.h:127-150). */
static int tri_box_overlap(v3 vm, v3 vM, v3 v1, v3 v2, v3 v3_)
{
    if (!plane_cuts_box(vm, vM, v1, v2, v3_)) return 0;
    for (int a = 0; a < 5; a++)
        if (axis_gap(a, v1.x, v1.y, v2.x, v2.y, v3_.x, v3_.y, vm.x, vm.y, vM.x, vM.y)) return 0;
    for (int a = 0; a < 5; a++)
        if (axis_gap(a, v1.y, v1.z, v2.y, v2.z, v3_.y, v3_.z, vm.y, vm.z, vM.y, vM.z)) return 0;
    for (int a = 0; a < 5; a++)
        if (axis_gap(a, v1.z, v1.x, v2.z, v2.x, v3_.z, v3_.x, vm.z, vm.x, vM.z, vM.x)) return 0;
    return 1;
}

/* CheckPointInTriangleAABB with eps = 2 FLT_EPSILON (util_tribin.h:190-209). */
static int point_in_face_aabb(v3 vp, v3 v1, v3 v2, v3 v3_)
{
    const float eps = FLT_EPSILON * 2.0f;
    return tri_box_overlap(vsubs(vp, eps), vadds(vp, eps), v1, v2, v3_);
}

/* CheckPointInTriangleExtended with eps = FLT_EPSILON (util.h:521-543). */
static int point_in_tri_ext(v3 vp, v3 v1, v3 v2, v3 v3_, v3 n)
{
    const float eps = FLT_EPSILON;
    v3 ven = unitv(crossv(vsub(v2, v1), n));
    if (dotv(vsub(v1, vp), ven) <= -eps) return 0;
    ven = unitv(crossv(vsub(v3_, v2), n));
    if (dotv(vsub(v2, vp), ven) <= -eps) return 0;
    ven = unitv(crossv(vsub(v1, v3_), n));
    if (dotv(vsub(v3_, vp), ven) <= -eps) return 0;
    return 1;
}

/* The x-ray distance of Cu_Voxelize_V1 and the 1D ray filter
   (mesh_voxelizer_voxelize.cu:283, geometry_bins_gpu.cu:247):
   d = (v1.x - vp.x) + (v1.y - vp.y)(n.y/n.x) + (v1.z - vp.z)(n.z/n.x). */
static inline float xray_dist(v3 v1, v3 vp, v3 n)
{
    return acc(acc(v1.x - vp.x, v1.y - vp.y, n.y / n.x), v1.z - vp.z, n.z / n.x);
}

/* ---- state ------------------------------------------------------------- */

int orc_geometry_alloc(orc_case *c)
{
    const int64_t nmb = c->nmb, nmc = c->nmc;
    c->tmp_1 = (int *)malloc(sizeof(int) * nmb);
    c->tmp_2 = (int *)malloc(sizeof(int) * nmb);
    c->onb_solid = (int *)malloc(sizeof(int) * nmb);
    c->cells_mask_hi = (int *)malloc(sizeof(int) * nmc);
    const size_t es = c->fp64 ? sizeof(double) : sizeof(float);
    c->Ff = calloc((size_t)6 * nmb, es);
    if (!c->tmp_1 || !c->tmp_2 || !c->onb_solid || !c->cells_mask_hi || !c->Ff) return AGAL_ERR_OOM;
    for (int64_t i = 0; i < nmb; i++) { c->tmp_1[i] = -1; c->tmp_2[i] = -1; c->onb_solid[i] = -1; }
    for (int64_t i = 0; i < nmc; i++) c->cells_mask_hi[i] = ORC_CELL_INTERIOR;
    return 0;
}

static void free_bins(orc_bins *b)
{
    free(b->n); free(b->N); free(b->ids);
    memset(b, 0, sizeof(*b));
}

void orc_geometry_free(orc_case *c)
{
    free(c->faces); c->faces = NULL;
    for (int L = 0; L < ORC_MAXL; L++) free_bins(&c->bins[L]);
    free_bins(&c->bins_md);
    free(c->onb_solid); free(c->X_b); free(c->tmp_1); free(c->tmp_2); free(c->cells_mask_hi); free(c->Ff);
    c->onb_solid = NULL; c->X_b = NULL; c->tmp_1 = c->tmp_2 = c->cells_mask_hi = NULL; c->Ff = NULL;
}

/* Bin grid constants of the Bins constructor (geometry_bins.h:106-170). */
typedef struct {
    float Lx, Ly, Lz;
    int nbl, dens[ORC_MAXL], Nxi[3][ORC_MAXL];
    float dxf[3][ORC_MAXL], Lx0g[3][ORC_MAXL];
} bin_grid;

static void bin_grid_init(const orc_case *c, bin_grid *g)
{
    const agal_params *P = &c->P;
    g->Lx = (float)P->L_c;
    g->Ly = (float)(P->L_fy * g->Lx);
    g->Lz = (float)(P->L_fz * g->Lx);
    const int Nx = P->Nx;
    const int Ny = (int)(Nx * (g->Ly / g->Lx)), Nz = (int)(Nx * (g->Lz / g->Lx));
    int nbl = P->G_BIN_LEVELS;
    if (nbl > P->MAX_LEVELS_WALL) nbl = P->MAX_LEVELS_WALL;
    if (nbl < 1) nbl = 1;
    if (nbl > ORC_MAXL) nbl = ORC_MAXL;
    g->nbl = nbl;
    g->dens[0] = P->G_BIN_DENSITY;
    g->dxf[0][0] = g->Lx / (float)Nx;
    g->dxf[1][0] = g->Ly / (float)Ny;
    g->dxf[2][0] = g->Lz / (float)Ny;          /* dz divides by the y count (geometry_bins.h:131) */
    g->Lx0g[0][0] = g->Lx / (float)g->dens[0];
    g->Lx0g[1][0] = g->Ly / (float)g->dens[0];
    g->Lx0g[2][0] = g->Lz / (float)g->dens[0];
    g->Nxi[0][0] = Nx; g->Nxi[1][0] = Ny; g->Nxi[2][0] = Nz;
    for (int L = 1; L < nbl; L++) {
        g->dens[L] = g->dens[L - 1] * 2;
        for (int d = 0; d < 3; d++) {
            g->dxf[d][L] = g->dxf[d][L - 1] * 0.5f;
            g->Lx0g[d][L] = g->Lx0g[d][L - 1] * 0.5f;
            g->Nxi[d][L] = g->Nxi[d][L - 1] * 2;
        }
    }
}

/* Cu_ComputeVoxelRayIndicators_1D, 3D branch (geometry_bins_gpu.cu:174-280):
   one +x ray per cell centre of the face's y-z bounding box. */
static int ray_filter_1d(const orc_case *c, int f, float dxL, float dxLo2, float Ny, float Nz)
{
    v3 v1, v2, v3_;
    load_face(c, f, &v1, &v2, &v3_);
    const v3 n = face_normal_unit(v1, v2, v3_);
    int iymin = (int)(fminf(fminf(v1.y, v2.y), v3_.y) * Ny);
    int izmin = (int)(fminf(fminf(v1.z, v2.z), v3_.z) * Nz);
    int iymax = (int)(fmaxf(fmaxf(v1.y, v2.y), v3_.y) * Ny);
    int izmax = (int)(fmaxf(fmaxf(v1.z, v2.z), v3_.z) * Nz);
    for (int iz = izmin; iz <= izmax; iz++)
        for (int iy = iymin; iy <= iymax; iy++) {
            const v3 vp = V(0.0f, acc(dxLo2, dxL, (float)iy), acc(dxLo2, dxL, (float)iz));
            v3 vi = vp;
            vi.x += xray_dist(v1, vp, n);
            if (point_in_face_aabb(vi, v1, v2, v3_)) return 1;
        }
    return 0;
}

/* Cu_ComputeVoxelRayIndicators_MD, 3D branch (geometry_bins_gpu.cu:24-160):
   rays along the half set of the 27 directions from every cell centre of the
   face's bounding box.  A direction parallel to the face gives an infinite
   or undefined distance; the extended point test then passes, as in the
   reference, which does not guard that division. */
static int ray_filter_md(const orc_case *c, int f, float dxL, float dxLo2, float Nx, float Ny, float Nz)
{
    v3 v1, v2, v3_;
    load_face(c, f, &v1, &v2, &v3_);
    const v3 n = face_normal_unit(v1, v2, v3_);
    const int ixmin = (int)(fminf(fminf(v1.x, v2.x), v3_.x) * Nx);
    const int iymin = (int)(fminf(fminf(v1.y, v2.y), v3_.y) * Ny);
    const int izmin = (int)(fminf(fminf(v1.z, v2.z), v3_.z) * Nz);
    const int ixmax = (int)(fmaxf(fmaxf(v1.x, v2.x), v3_.x) * Nx);
    const int iymax = (int)(fmaxf(fmaxf(v1.y, v2.y), v3_.y) * Ny);
    const int izmax = (int)(fmaxf(fmaxf(v1.z, v2.z), v3_.z) * Nz);
    for (int p = 1; p < 27; p++) {
        if (!orc_half(3, p)) continue;
        const v3 ray = V((float)ORC_C3[0][p], (float)ORC_C3[1][p], (float)ORC_C3[2][p]);
        for (int iz = izmin; iz <= izmax; iz++)
            for (int iy = iymin; iy <= iymax; iy++)
                for (int ix = ixmin; ix <= ixmax; ix++) {
                    const v3 vp = V(acc(dxLo2, dxL, (float)ix), acc(dxLo2, dxL, (float)iy), acc(dxLo2, dxL, (float)iz));
                    const float d = dotv(vsub(v1, vp), n) / dotv(ray, n);
                    const v3 vi = V(acc(vp.x, ray.x, d), acc(vp.y, ray.y, d), acc(vp.z, ray.z, d));
                    if (point_in_tri_ext(vi, v1, v2, v3_, n)) return 1;
                }
    }
    return 0;
}

/* ---- binning (Bins::G_MakeBinsGPU / _MD, geometry_bins_gpu.cu:587-1300) ---- */

/* One bin set at bin level L.  md = 0: the voxelizer's bins; md = 1: the
   link-length bins.  Every face that passes the ray filter is tested against
   the bins (2 + G_BIN_SPEC)^3 around its bounding box, grown by one cell
   width dx_L + FLT_EPSILON on every side (Cu_ComputeBoundingBoxLimits3D,
   :423-560); each hit is recorded as the pair (bin, face) in slot
   [counter][filtered face index], so that after the stable compaction and
   the stable sort by bin (thrust::remove_if / sort_by_key) the faces of a
   bin are ordered by (counter, face). */
static int make_bins(orc_case *c, const bin_grid *g, int L, int md, orc_bins *out)
{
    const int nf = c->n_faces;
    const int dens = g->dens[L];
    const int n_bins = dens * dens * dens;
    const int spec = c->P.G_BIN_SPEC;
    const int64_t n_limits = (int64_t)(2 + spec) * (2 + spec) * (2 + spec);
    int use_ray;
    if (!md) use_ray = !(L == g->nbl - 1 && g->nbl != c->P.MAX_LEVELS_WALL);
    else use_ray = (c->P.MAX_LEVELS_WALL == L + 1);
    const float dxL = g->dxf[0][L], dxLo2 = 0.5f * g->dxf[0][L];

    int *ray = (int *)malloc(sizeof(int) * (nf > 0 ? nf : 1));
    if (!ray) return AGAL_ERR_OOM;
    int n_filtered = nf;
    if (use_ray) {
#pragma omp parallel for schedule(dynamic, 64)
        for (int f = 0; f < nf; f++) {
            /* cells per unit length on every axis: the reference's
               coordinate x N per axis, which agrees with it on the unit
               cube and stays consistent on a channel */
            const float cpl = (float)g->Nxi[0][L] / g->Lx;
            const int hit = md ? ray_filter_md(c, f, dxL, dxLo2, cpl, cpl, cpl) : ray_filter_1d(c, f, dxL, dxLo2, cpl, cpl);
            ray[f] = hit ? f : -1;
        }
        /* copy_if + scatter: ray[f] becomes the rank of f among the kept faces. */
        n_filtered = 0;
        for (int f = 0; f < nf; f++) ray[f] = (ray[f] >= 0) ? n_filtered++ : -1;
    } else {
        for (int f = 0; f < nf; f++) ray[f] = f;
    }
    const int64_t n_lim = n_limits * (int64_t)n_filtered;
    int *key = (int *)malloc(sizeof(int) * (size_t)(n_lim > 0 ? n_lim : 1));
    int *val = (int *)malloc(sizeof(int) * (size_t)(n_lim > 0 ? n_lim : 1));
    if (!key || !val) { free(ray); free(key); free(val); return AGAL_ERR_OOM; }
    for (int64_t i = 0; i < n_lim; i++) { key[i] = n_bins; val[i] = -1; }
    const float dx = g->dxf[0][L] + FLT_EPSILON;
    const float Lx = g->Lx, Ly = g->Ly, Lz = g->Lz;
    const float L0x = g->Lx0g[0][L], L0y = g->Lx0g[1][L], L0z = g->Lx0g[2][L];
    /* bins per unit length per axis (the reference's coordinate x density on
       the unit cube) */
    const float sx = (float)dens / Lx, sy = (float)dens / Ly, sz = (float)dens / Lz;
    int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
    for (int f = 0; f < nf; f++) {
        const int map_val = ray[f];
        if (map_val < 0) continue;
        v3 v1, v2, v3_;
        load_face(c, f, &v1, &v2, &v3_);
        const v3 bm = V(fminf(fminf(v1.x, v2.x), v3_.x), fminf(fminf(v1.y, v2.y), v3_.y), fminf(fminf(v1.z, v2.z), v3_.z));
        const v3 bM = V(fmaxf(fmaxf(v1.x, v2.x), v3_.x), fmaxf(fmaxf(v1.y, v2.y), v3_.y), fmaxf(fmaxf(v1.z, v2.z), v3_.z));
        if ((bm.x < -dx && bM.x < -dx) || (bm.x > Lx + dx && bM.x > Lx + dx)) continue;
        if ((bm.y < -dx && bM.y < -dx) || (bm.y > Ly + dx && bM.y > Ly + dx)) continue;
        if ((bm.z < -dx && bM.z < -dx) || (bm.z > Lz + dx && bM.z > Lz + dx)) continue;
        const int xl = (int)(bm.x * sx) - 1, yl = (int)(bm.y * sy) - 1, zl = (int)(bm.z * sz) - 1;
        const int xL = (int)(bM.x * sx) + 1, yL = (int)(bM.y * sy) + 1, zL = (int)(bM.z * sz) + 1;
        int counter = 0;
        for (int K = zl; K < zL + 1; K++)
            for (int J = yl; J < yL + 1; J++)
                for (int I = xl; I < xL + 1; I++) {
                    const v3 vm = V((float)I * L0x - dx, (float)J * L0y - dx, (float)K * L0z - dx);
                    const v3 vM = V((float)(I + 1) * L0x + dx, (float)(J + 1) * L0y + dx, (float)(K + 1) * L0z + dx);
                    if (tri_box_overlap(vm, vM, v1, v2, v3_) && counter < n_limits) {
                        const int gid = I + dens * J + dens * dens * K;
                        /* The reference writes bins outside the grid unchecked. */
                        if (I < 0 || J < 0 || K < 0 || I >= dens || J >= dens || K >= dens) bad = 1;
                        key[map_val + (int64_t)counter * n_filtered] = gid;
                        val[map_val + (int64_t)counter * n_filtered] = f;
                        counter++;
                    }
                }
    }
    free(ray);
    if (bad) { free(key); free(val); return AGAL_ERR_PARAM; }
    /* Stable compaction, then a stable counting sort by bin. */
    int *cnt = (int *)calloc((size_t)n_bins, sizeof(int));
    int *start = (int *)calloc((size_t)n_bins, sizeof(int));
    if (!cnt || !start) { free(key); free(val); free(cnt); free(start); return AGAL_ERR_OOM; }
    int64_t ne = 0;
    for (int64_t i = 0; i < n_lim; i++)
        if (key[i] != n_bins) { cnt[key[i]]++; ne++; }
    int *ids = (int *)malloc(sizeof(int) * (size_t)(ne > 0 ? ne : 1));
    int *pos = (int *)malloc(sizeof(int) * (size_t)n_bins);
    if (!ids || !pos) { free(key); free(val); free(cnt); free(start); free(ids); free(pos); return AGAL_ERR_OOM; }
    int64_t s = 0;
    for (int b = 0; b < n_bins; b++) { start[b] = cnt[b] ? (int)s : 0; pos[b] = (int)s; s += cnt[b]; }
    for (int64_t i = 0; i < n_lim; i++)
        if (key[i] != n_bins) ids[pos[key[i]]++] = val[i];
    free(pos); free(key); free(val);
    free_bins(out);
    out->density = dens;
    out->sx = sx; out->sy = sy; out->sz = sz;
    out->n_bins = n_bins;
    out->n_entries = ne;
    out->n = cnt;
    out->N = start;
    out->ids = ids;
    return 0;
}

int orc_set_geometry(orc_case *c, const float *faces, int n_faces)
{
    /* Geometry::G_Init_Arrays_CoordsList_CPU (geometry_init.cu:71-190) with
       the faces as given (any face splitting already applied), then
       Geometry::G_InitBins (geometry_bins.h:106-203). */
    if (c->dim != 3 || n_faces < 0 || (n_faces > 0 && !faces)) return AGAL_ERR_PARAM;
    free(c->faces);
    c->faces = (float *)malloc(sizeof(float) * 9 * (size_t)(n_faces > 0 ? n_faces : 1));
    if (!c->faces) return AGAL_ERR_OOM;
    c->n_faces = n_faces;
    for (int f = 0; f < n_faces; f++)
        for (int r = 0; r < 9; r++) c->faces[f + (int64_t)r * n_faces] = faces[(int64_t)f * 9 + r];
    bin_grid g;
    bin_grid_init(c, &g);
    for (int L = 0; L < ORC_MAXL; L++) free_bins(&c->bins[L]);
    free_bins(&c->bins_md);
    c->n_bin_levels = g.nbl;
    for (int L = 0; L < g.nbl; L++) {
        int rc = make_bins(c, &g, L, 0, &c->bins[L]);
        if (rc) return rc;
    }
    c->bin_level_md = -1;
    if (c->P.G_BIN_MAKE_LINKS) {
        int lmd = (c->P.MAX_LEVELS_WALL < g.nbl ? c->P.MAX_LEVELS_WALL : g.nbl) - 1;
        c->bin_level_md = lmd;
        int rc = make_bins(c, &g, lmd, 1, &c->bins_md);
        if (rc) return rc;
    }
    c->geometry_init = 1;
    return 0;
}

int orc_bins_info(const orc_case *c, int level, int *density, int *n_bins, int64_t *n_entries)
{
    const orc_bins *b = (level < 0) ? &c->bins_md : ((level < c->n_bin_levels) ? &c->bins[level] : NULL);
    if (!b || !b->n) return AGAL_ERR_PARAM;
    if (density) *density = b->density;
    if (n_bins) *n_bins = b->n_bins;
    if (n_entries) *n_entries = b->n_entries;
    return 0;
}

int orc_bins_copy(const orc_case *c, int level, int *n, int *N, int *ids)
{
    const orc_bins *b = (level < 0) ? &c->bins_md : ((level < c->n_bin_levels) ? &c->bins[level] : NULL);
    if (!b || !b->n) return AGAL_ERR_PARAM;
    if (n) memcpy(n, b->n, sizeof(int) * (size_t)b->n_bins);
    if (N) memcpy(N, b->N, sizeof(int) * (size_t)b->n_bins);
    if (ids) memcpy(ids, b->ids, sizeof(int) * (size_t)b->n_entries);
    return 0;
}

/* ---- voxelization (Mesh::M_Geometry_Voxelize_S1/S2/S3, mesh_voxelizer.cu) ---- */

/* Cell centre as Cu_Voxelize_V1 forms it: X + I dx_L in float, then
   + 0.5 dx_L in double, stored as float (mesh_voxelizer_voxelize.cu:241-246). */
static inline float cell_centre(float X, int I, float dxL)
{
    const float a = X + (float)I * dxL;
    return (float)((double)a + 0.5 * (double)dxL);
}

/* Cu_Voxelize_V1 (mesh_voxelizer_voxelize.cu:203-351) on one block: the
   signed x-distance to the closest face of the cell's bin whose small box
   around the ray hit overlaps it; the side of that face (sign of the
   distance and of n.x) makes the cell a guard or a solid; three sweeps
   carry guards and solids along x inside the block. */
static void voxelize_block(orc_case *c, int b, float dxL, const orc_bins *bins)
{
    const int64_t nmb = c->nmb;
    const int MC = c->MC;
    const int dens = bins->density;
    int cm[64], any = 0;
    for (int t = 0; t < MC; t++) {
        const int I = t % 4, J = (t / 4) % 4, K = t / 16;
        const v3 vp = V(cell_centre(c->cblock_f_X[b + 0 * nmb], I, dxL), cell_centre(c->cblock_f_X[b + 1 * nmb], J, dxL),
                        cell_centre(c->cblock_f_X[b + 2 * nmb], K, dxL));
        const int gb = (int)(vp.x * bins->sx) + dens * (int)(vp.y * bins->sy) +
                       dens * dens * (int)(vp.z * bins->sz);
        int pmin = -1, mask = ORC_CELL_INTERIOR;
        float dmin = 1.0f;
        const int n_f = (gb >= 0 && gb < bins->n_bins) ? bins->n[gb] : 0;
        const int *fl = (n_f > 0) ? &bins->ids[bins->N[gb]] : NULL;
        for (int p = 0; p < n_f; p++) {
            v3 v1, v2, v3_;
            load_face(c, fl[p], &v1, &v2, &v3_);
            const v3 n = face_normal_unit(v1, v2, v3_);
            const float d = xray_dist(v1, vp, n);
            v3 vi = vp;
            vi.x += d;
            if ((fabsf(d) < dmin || pmin == -1) && point_in_face_aabb(vi, v1, v2, v3_)) {
                dmin = fabsf(d);
                pmin = p;
                if (d > 0 && n.x < 0) mask = ORC_CELL_LL;
                if (d < 0 && n.x < 0) mask = ORC_CELL_LR;
                if (d > 0 && n.x > 0) mask = ORC_CELL_RL;
                if (d < 0 && n.x > 0) mask = ORC_CELL_RR;
            }
        }
        if (pmin != -1) any = 1;
        cm[t] = mask;
    }
    if (!any) return;
    for (int t = 0; t < MC; t++) {
        if (cm[t] == ORC_CELL_LL || cm[t] == ORC_CELL_RR) cm[t] = ORC_CELL_GUARD;
        if (cm[t] == ORC_CELL_LR || cm[t] == ORC_CELL_RL) cm[t] = ORC_CELL_SOLID;
    }
    /* Three synchronous sweeps: every cell reads its x-neighbours' states of
       the previous sweep (the warp's loads precede its stores). */
    for (int l = 0; l < 3; l++) {
        int nx[64];
        for (int t = 0; t < MC; t++) {
            const int I = t % 4;
            int m = cm[t];
            if (I > 0) {
                const int nm = cm[t - 1];
                if (nm == ORC_CELL_GUARD && m == ORC_CELL_INTERIOR) m = ORC_CELL_GUARD;
                if (nm == ORC_CELL_SOLID && m != ORC_CELL_GUARD) m = ORC_CELL_SOLID;
            }
            if (I < 3) {
                const int nm = cm[t + 1];
                if (nm == ORC_CELL_GUARD && m == ORC_CELL_INTERIOR) m = ORC_CELL_GUARD;
                if (nm == ORC_CELL_SOLID && m != ORC_CELL_GUARD) m = ORC_CELL_SOLID;
            }
            nx[t] = m;
        }
        memcpy(cm, nx, sizeof(int) * MC);
    }
    for (int t = 0; t < MC; t++) {
        const int64_t o = (int64_t)b * MC + t;
        const int orig = c->cells_ID_mask[o];
        if (cm[t] == ORC_CELL_SOLID || (orig != ORC_CELL_GHOST && orig != ORC_CELL_INTERFACE)) c->cells_ID_mask[o] = cm[t];
    }
}

/* Cu_Voxelize_Propagate_Right / _Left (mesh_voxelizer_propagate.cu:97-215):
   from every block without a same-level neighbour on one side, walk the row
   of blocks in the other direction; a row of cells whose previous block
   ended in a solid cell becomes solid up to the next guard.  dir = +1
   walks right (neighbour slot 1), -1 walks left (slot 2). */
static void propagate(orc_case *c, int L, int dir, int dense)
{
    const int64_t nmb = c->nmb;
    const int MC = c->MC;
    const int N_LEFT = 2, N_RIGHT = 1;
    const int from = dir > 0 ? N_LEFT : N_RIGHT, to = dir > 0 ? N_RIGHT : N_LEFT;
    const int edge = dir > 0 ? 3 : 0;
    const int *ids = &c->id_set[(int64_t)L * nmb];
    const int n = c->n_ids[L];
#pragma omp parallel for schedule(dynamic, 8)
    for (int kap = 0; kap < n; kap++) {
        const int b = ids[kap];
        const int start = c->cblock_ID_nbr[b + (int64_t)from * nmb];
        if (start >= 0) continue;
        int status[16];
        for (int r = 0; r < 16; r++) {
            status[r] = c->cells_ID_mask[(int64_t)b * MC + edge + 4 * r];
            if (start == ORC_N_SPECID && status[r] != ORC_CELL_GUARD) status[r] = ORC_CELL_SOLID;
        }
        int nb = c->cblock_ID_nbr[b + (int64_t)to * nmb];
        for (int k = 0; nb > -1 && k < 1000; k++) {
            int m[64];
            for (int t = 0; t < MC; t++) {
                m[t] = c->cells_ID_mask[(int64_t)nb * MC + t];
                if (status[t / 4] == ORC_CELL_SOLID && m[t] != ORC_CELL_GUARD) m[t] = ORC_CELL_SOLID;
            }
            for (int r = 0; r < 16; r++) status[r] = m[edge + 4 * r];
            for (int t = 0; t < MC; t++) {
                if ((dir < 0 || dense) && m[t] == ORC_CELL_GUARD) m[t] = ORC_CELL_INTERIOR;
                c->cells_ID_mask[(int64_t)nb * MC + t] = m[t];
            }
            nb = c->cblock_ID_nbr[nb + (int64_t)to * nmb];
        }
    }
}

/* Cu_Voxelize_UpdateMasks (mesh_voxelizer_masks.cu:227-256). */
static void update_block_masks(orc_case *c, int L)
{
    const int *ids = &c->id_set[(int64_t)L * c->nmb];
    for (int kap = 0; kap < c->n_ids[L]; kap++) {
        const int b = ids[kap];
        for (int t = 0; t < c->MC; t++)
            if (c->cells_ID_mask[(int64_t)b * c->MC + t] == ORC_CELL_SOLID) { c->cblock_ID_mask[b] = ORC_BLOCK_SOLID; break; }
    }
}

static int eligible(const orc_case *c, int b)
{
    for (int q = 0; q < c->Qmax; q++)
        if (c->cblock_ID_nbr[b + (int64_t)q * c->nmb] == ORC_N_SKIPID) return 0;
    return 1;
}

/* Cu_MarkBlocks_MarkBoundary / _MarkExterior / _Propagate / _Finalize
   (mesh_voxelizer_refine.cu:20-414).  Their shared-memory staging writes
   thread-major and reads direction-major, but the per-entry test is
   elementwise, so each block simply tests all of its neighbours. */
static void mark_blocks(orc_case *c, int L, int hit_max, int n_prop)
{
    const int64_t nmb = c->nmb;
    const int Qm = c->Qmax;
    const int n = c->id_max[L];
    char *flag = (char *)calloc((size_t)(n > 0 ? n : 1), 1);
    if (!flag) return;
    /* MarkBoundary: solid blocks next to a regular block are on the solid boundary. */
    for (int b = 0; b < n; b++) {
        if (c->cblock_level[b] != L || c->cblock_ID_mask[b] != ORC_BLOCK_SOLID) continue;
        for (int q = 0; q < Qm; q++) {
            const int nb = c->cblock_ID_nbr[b + (int64_t)q * nmb];
            if (nb > -1 && c->cblock_ID_mask[nb] == ORC_BLOCK_REGULAR) { flag[b] = 1; break; }
        }
    }
    for (int b = 0; b < n; b++) {
        if (!flag[b] || c->cblock_ID_ref[b] != ORC_REF_UNREFINED) continue;
        c->cblock_ID_mask[b] = ORC_BLOCK_SOLIDB;
        if (!hit_max && eligible(c, b)) c->cblock_ID_ref[b] = ORC_REF_MARK_REFINE;
    }
    /* MarkExterior: blocks next to a solid-boundary block. */
    memset(flag, 0, (size_t)(n > 0 ? n : 1));
    for (int b = 0; b < n; b++) {
        if (c->cblock_level[b] != L) continue;
        for (int q = 0; q < Qm; q++) {
            const int nb = c->cblock_ID_nbr[b + (int64_t)q * nmb];
            if (nb > -1 && c->cblock_ID_mask[nb] == ORC_BLOCK_SOLIDB) { flag[b] = 1; break; }
        }
    }
    for (int b = 0; b < n; b++) {
        if (!flag[b] || c->cblock_ID_ref[b] != ORC_REF_UNREFINED) continue;
        if (!hit_max && eligible(c, b)) c->cblock_ID_ref[b] = ORC_REF_INDET_E;
        if (c->cblock_ID_mask[b] == ORC_BLOCK_REGULAR) c->cblock_ID_mask[b] = ORC_BLOCK_SOLIDA;
    }
    /* Propagate: alternate between the even (ref = 11) and odd (tmp_1 = 12) fronts. */
    for (int j = 0; j < n_prop; j++) {
        const int even = (j % 2) == 0;
        memset(flag, 0, (size_t)(n > 0 ? n : 1));
        for (int b = 0; b < n; b++) {
            if (c->cblock_level[b] != L) continue;
            if (!(c->cblock_ID_mask[b] > -1 || (j == 0 && c->cblock_ID_mask[b] == ORC_BLOCK_SOLID))) continue;
            for (int q = 0; q < Qm; q++) {
                const int nb = c->cblock_ID_nbr[b + (int64_t)q * nmb];
                if (nb < 0) continue;
                if (even ? c->cblock_ID_ref[nb] == ORC_REF_INDET_E : c->tmp_1[nb] == ORC_REF_INDET_O) { flag[b] = 1; break; }
            }
        }
        for (int b = 0; b < n; b++) {
            if (!flag[b]) continue;
            const int C = even ? c->cblock_ID_ref[b] == ORC_REF_UNREFINED : c->tmp_1[b] == -1;
            if (!C || !eligible(c, b)) continue;
            if (even) c->tmp_1[b] = ORC_REF_INDET_O;
            else c->cblock_ID_ref[b] = ORC_REF_INDET_E;
        }
    }
    /* Finalize. */
    for (int b = 0; b < n; b++) {
        if (c->cblock_ID_ref[b] == ORC_REF_INDET_E || c->tmp_1[b] == ORC_REF_INDET_O) {
            c->cblock_ID_ref[b] = ORC_REF_MARK_REFINE;
            c->tmp_1[b] = -1;
        }
    }
    free(flag);
}

int orc_voxelize_s1(orc_case *c, int L)
{
    /* Mesh::M_Geometry_Voxelize_S1 (mesh_voxelizer.cu:34-156). */
    if (!c->geometry_init || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    const float R = (float)((double)(float)c->P.G_NEAR_WALL_DISTANCE / pow(2.0, (double)(float)L));
    const int n_prop = (int)(R / (float)(4.0 * sqrt(2.0) * (double)c->dxf[L])) + 1;
    const int hit_max = (L == c->max_levels - 1);
    const int Lbin = L < c->n_bin_levels - 1 ? L : c->n_bin_levels - 1;
    const float dxL = c->dxf[L];
    const int *ids = &c->id_set[(int64_t)L * c->nmb];
#pragma omp parallel for schedule(dynamic, 4)
    for (int kap = 0; kap < c->n_ids[L]; kap++) voxelize_block(c, ids[kap], dxL, &c->bins[Lbin]);
    propagate(c, L, +1, L == c->L0);
    if (L > c->L0) propagate(c, L, -1, 0);
    update_block_masks(c, L);
    mark_blocks(c, L, hit_max, n_prop);
    return 0;
}

int orc_update_solid_children(orc_case *c, int L)
{
    /* Mesh::M_UpdateSolidChildren -> Cu_MarkBlocks_UpdateSolidChildren
       (mesh_voxelizer_refine.cu:203-245): children of a solid block mark an
       absent left/right neighbour as N_SPECID, the start of a solid row for
       the propagation on the finer level.  The child index is formed from
       cblock_ID_nbr_child even for a block without children, as there. */
    if (L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    const int64_t nmb = c->nmb;
    const int N_LEFT = 2, N_RIGHT = 1;
    for (int b = 0; b < c->id_max[L]; b++) {
        if (c->cblock_level[b] != L || c->cblock_ID_mask[b] != ORC_BLOCK_SOLID) continue;
        for (int p = 0; p < c->NCH; p++) {
            const int ch = c->cblock_ID_nbr_child[b] + p;
            if (ch < 0) continue;
            if (c->cblock_ID_nbr[ch + N_LEFT * nmb] == ORC_N_SKIPID) c->cblock_ID_nbr[ch + N_LEFT * nmb] = ORC_N_SPECID;
            if (c->cblock_ID_nbr[ch + N_RIGHT * nmb] == ORC_N_SKIPID) c->cblock_ID_nbr[ch + N_RIGHT * nmb] = ORC_N_SPECID;
        }
    }
    return 0;
}

/* Cu_GetNbrIndices (util_index.h:144-190): block and cell of the neighbour
   of cell (I, J, K) along direction p of the 27-direction table. */
static inline void nbr_of(const orc_case *c, const int *s_nbr, int I, int J, int K, int p, int *nb, int *nc)
{
    const int Ip = I + ORC_C3[0][p], Jp = J + ORC_C3[1][p], Kp = K + ORC_C3[2][p];
    *nb = s_nbr[orc_nbrslot(3, Ip, Jp, Kp)];
    *nc = orc_nbrcell(3, Ip, Jp, Kp);
    (void)c;
}

int orc_voxelize_s2(orc_case *c, int L)
{
    /* Mesh::M_Geometry_Voxelize_S2 (mesh_voxelizer.cu:158-189):
       Cu_MarkBlocks_CheckMasks_S1<AP,1> then _S2 (mesh_voxelizer_masks.cu:19-179). */
    if (!c->geometry_init || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0) return 0;
    const int64_t nmb = c->nmb;
    const int MC = c->MC, ML = c->max_levels;
    if (L == 0)
        for (int b = 0; b < c->id_max[ML]; b++) { c->tmp_1[b] = 0; c->tmp_2[b] = 0; }
    const int *ids = &c->id_set[(int64_t)L * nmb];
#pragma omp parallel for schedule(dynamic, 8)
    for (int kap = 0; kap < c->n_ids[L]; kap++) {
        const int b = ids[kap];
        if (!(c->cblock_ID_nbr_child[b] < 0 && c->cblock_ID_mask[b] < 0 && c->cblock_ID_mask[b] != ORC_BLOCK_SOLID)) continue;
        int s_nbr[27];
        for (int S = 0; S < 27; S++) s_nbr[S] = c->cblock_ID_nbr[b + (int64_t)c->map[S] * nmb];
        int count = 0;
        for (int t = 0; t < MC; t++) {
            const int I = t % 4, J = (t / 4) % 4, K = t / 16;
            const int curr = c->cells_ID_mask[(int64_t)b * MC + t];
            int near = 0;
            for (int p = 0; p < 27 && !near; p++) {
                int nb, nc;
                nbr_of(c, s_nbr, I, J, K, p, &nb, &nc);
                if (nb >= 0 && c->cells_ID_mask[(int64_t)nb * MC + nc] == ORC_CELL_SOLID) near = 1;
            }
            if (near && curr != ORC_CELL_SOLID) {
                c->cells_mask_hi[(int64_t)b * MC + t] = ORC_CELL_BOUNDARY;
                count++;
            }
        }
        if (count > 0) { c->tmp_1[b] = count; c->cblock_ID_onb[b] = 1; }
    }
    for (int kap = 0; kap < c->n_ids[L]; kap++) {
        const int b = ids[kap];
        if (c->cblock_ID_onb[b] != 1) continue;
        for (int t = 0; t < MC; t++)
            if (c->cells_mask_hi[(int64_t)b * MC + t] == ORC_CELL_BOUNDARY) c->cells_ID_mask[(int64_t)b * MC + t] = ORC_CELL_BOUNDARY;
    }
    return 0;
}

int orc_voxelize_s3(orc_case *c)
{
    /* Mesh::M_Geometry_Voxelize_S3 (mesh_voxelizer.cu:191-245): count the
       blocks with boundary cells, give each a slot in ascending block order
       and size the link-length array for them (rounded up to 128 blocks). */
    if (!c->geometry_init) return AGAL_ERR_PARAM;
    const int ML = c->max_levels;
    const int n = c->id_max[ML];
    int64_t sa = 0;
    int sb = 0;
    for (int b = 0; b < n; b++) { sa += c->tmp_1[b]; if (c->tmp_1[b] > 0) sb++; }
    c->n_solida = sa;
    const int sb_old = sb;
    c->n_solidb = ((sb + 128) / 128) * 128;
    c->n_maxcells_b = (int64_t)c->n_solidb * c->MC;
    if (sb_old > 0 || c->n_solidb > 0) {
        for (int64_t b = 0; b < c->nmb; b++) c->onb_solid[b] = -1;
        int slot = 0;
        for (int b = 0; b < n; b++)
            if (c->tmp_1[b] > 0) c->onb_solid[b] = slot++;
        free(c->X_b);
        c->X_b = NULL;
        if (c->P.G_BIN_MAKE_LINKS) {
            const int64_t nx = c->n_maxcells_b * c->Qmax;
            c->X_b = (float *)malloc(sizeof(float) * (size_t)(nx > 0 ? nx : 1));
            if (!c->X_b) return AGAL_ERR_OOM;
            for (int64_t i = 0; i < nx; i++) c->X_b[i] = -1.0f;
        }
        for (int b = 0; b < n; b++) { c->tmp_1[b] = -1; c->tmp_2[b] = -1; }
    }
    return 0;
}

/* ---- link lengths (mesh_voxelizer_links.cu) ------------------------------ */

int orc_link_lengths(orc_case *c, int L)
{
    /* Mesh::M_LinkLengthComputation (mesh_voxelizer.cu:261-294):
       Cu_LinkLengthComputation (links.cu:26-196) then
       Cu_LinkLengthValidation (links.cu:203-358). */
    if (!c->geometry_init || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    if (!(c->n_solidb > 0 && c->n_ids[L] > 0 && c->P.G_BIN_MAKE_LINKS && c->X_b)) return 0;
    const int64_t nmb = c->nmb, ncb = c->n_maxcells_b;
    const int MC = c->MC;
    const float dxL = c->dxf[L];
    const orc_bins *bins = &c->bins_md;
    const int dens = bins->density;
    const int *ids = &c->id_set[(int64_t)L * nmb];
    /* Computation: for every cell of a wall block, the distance along each of
       the 26 directions to the faces of its bin that the ray meets within one
       cell; kept for boundary cells only.  The running minimum compares the
       new distance with the stored normalised one, as the reference does. */
#pragma omp parallel for schedule(dynamic, 4)
    for (int kap = 0; kap < c->n_ids[L]; kap++) {
        const int b = ids[kap];
        const int slot = c->onb_solid[b];
        if (slot < 0) continue;
        for (int t = 0; t < MC; t++) {
            const int I = t % 4, J = (t / 4) % 4, K = t / 16;
            const v3 vp = V(cell_centre(c->cblock_f_X[b + 0 * nmb], I, dxL), cell_centre(c->cblock_f_X[b + 1 * nmb], J, dxL),
                            cell_centre(c->cblock_f_X[b + 2 * nmb], K, dxL));
            const int gb = (int)(vp.x * bins->sx) + dens * (int)(vp.y * bins->sy) +
                           dens * dens * (int)(vp.z * bins->sz);
            const int n_f = (gb >= 0 && gb < bins->n_bins) ? bins->n[gb] : 0;
            if (n_f <= 0) continue;
            float dQ[27];
            for (int q = 0; q < 27; q++) dQ[q] = -1.0f;
            const int *fl = &bins->ids[bins->N[gb]];
            for (int p = 0; p < n_f; p++) {
                v3 v1, v2, v3_;
                load_face(c, fl[p], &v1, &v2, &v3_);
                const v3 n = face_normal_unit(v1, v2, v3_);
                for (int q = 1; q < 27; q++) {
                    const v3 ray = V((float)ORC_C3[0][q], (float)ORC_C3[1][q], (float)ORC_C3[2][q]);
                    float d = dotv(ray, n);
                    if (d == 0.0f) continue;
                    d = dotv(vsub(v1, vp), n) / d;
                    if (d > 0.0f && d < dxL + FLT_EPSILON) {
                        const v3 vi = V(acc(vp.x, ray.x, d), acc(vp.y, ray.y, d), acc(vp.z, ray.z, d));
                        if (point_in_tri_ext(vi, v1, v2, v3_, n)) {
                            const float dist_q = dQ[q];
                            if (d < dist_q || dist_q < 0) dQ[q] = d / dxL;
                        }
                    }
                }
            }
            if (c->cells_ID_mask[(int64_t)b * MC + t] == ORC_CELL_BOUNDARY)
                for (int q = 1; q < 27; q++) c->X_b[(int64_t)slot * MC + t + (int64_t)q * ncb] = dQ[q];
        }
    }
    /* Validation: a boundary cell with no link towards a solid neighbour
       gets the link length 1/2.  The neighbour's mask is read at the
       neighbour's slot number used as a block ID, as the reference does
       (links.cu:263-266); only the 1/2 corrections are ever stored. */
    for (int kap = 0; kap < c->n_ids[L]; kap++) {
        const int b = ids[kap];
        const int slot = c->onb_solid[b];
        if (slot < 0) continue;
        int s_nbr[27];
        for (int S = 0; S < 27; S++) s_nbr[S] = c->cblock_ID_nbr[b + (int64_t)c->map[S] * nmb];
        for (int t = 0; t < MC; t++) {
            const int I = t % 4, J = (t / 4) % 4, K = t / 16;
            for (int p = 1; p < 27; p++) {
                if (!orc_half(3, p)) continue;
                int nb, nc;
                nbr_of(c, s_nbr, I, J, K, p, &nb, &nc);
                if (nb > -1) nb = c->onb_solid[nb];
                if (nb <= -1) continue;
                const int pb = ORC_PB3[p];
                float *xp = &c->X_b[(int64_t)slot * MC + t + (int64_t)p * ncb];
                float *xq = &c->X_b[(int64_t)nb * MC + nc + (int64_t)pb * ncb];
                const int mask_p = c->cells_ID_mask[(int64_t)b * MC + t];
                const int mask_pb = c->cells_ID_mask[(int64_t)nb * MC + nc];
                if (mask_p == ORC_CELL_BOUNDARY && *xp < 0 && mask_pb == ORC_CELL_SOLID) *xp = 0.5f;
                if (mask_pb == ORC_CELL_BOUNDARY && *xq < 0 && mask_p == ORC_CELL_SOLID) *xq = 0.5f;
            }
        }
    }
    return 0;
}

int orc_geometry_counts(const orc_case *c, int64_t *out)
{
    /* n_faces, n_solida, n_solidb, n_maxcells_b. */
    out[0] = c->n_faces;
    out[1] = c->n_solida;
    out[2] = c->n_solidb;
    out[3] = c->n_maxcells_b;
    return 0;
}
