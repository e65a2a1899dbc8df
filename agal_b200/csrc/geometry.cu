// Geometry set-up on the device: triangle binning, voxelization with
// near-wall block marking, solid-boundary slots and link lengths
// (Geometry::G_InitBins / Bins::G_MakeBinsGPU(_MD), geometry_bins_gpu.cu;
// Mesh::M_Geometry_Voxelize_S1/S2/S3, M_UpdateSolidChildren,
// M_LinkLengthComputation, mesh_voxelizer*.cu).  3D.
//
// Floating point: the reference evaluates this geometry in FP32 with the
// compiler fusing each multiply into the add or subtract that consumes it.
// These kernels spell every operation out with round-to-nearest intrinsics
// in that pattern (a*b + c*d = fma(a, b, c*d), a*b - c*d = fma(a, b, -(c*d)),
// s + a*b = fma(a, b, s)), so the integer results (bins, masks, block
// states) and the FP32 link lengths come out bit for bit as the reference's.
//
// Data on the device (agal_ctx):
//   faces       [9][n_faces] float, v1x v1y v1z v2x .. v3z
//   bins[L]     CSR over density^3 bins of the unit cube: n (count),
//               N (start), ids (face IDs ordered by (bin, slot, face))
//   bins_md     the link-length bins
//   onb_solid   [n_maxcblocks] slot of each wall block, -1 otherwise
//   X_b         [27][n_maxcells_b] link length per direction, -1 = none
//   vox_tmp     [n_maxcblocks] marking scratch (c_tmp_1), -1 at rest
//   bnd_bits    [n_maxcblocks] boundary-cell flags of S2 (64 bits a block)
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "compact.cuh"
#include "ctx.h"
#include "lattice.cuh"

namespace agal {
namespace geo {

// ---- FP32 vector algebra, rounded as the reference's fused code ----------
struct v3 {
    float x, y, z;
};
__device__ __forceinline__ v3 V(float x, float y, float z) { return v3{x, y, z}; }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ v3 vsub(v3 a, v3 b) { return V(fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)); }
__device__ __forceinline__ v3 vsubs(v3 a, float s) { return V(fsub(a.x, s), fsub(a.y, s), fsub(a.z, s)); }
__device__ __forceinline__ v3 vadds(v3 a, float s) { return V(fadd(a.x, s), fadd(a.y, s), fadd(a.z, s)); }
__device__ __forceinline__ v3 vmuls(v3 a, float s) { return V(fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)); }
// a*b + c*d, a*b - c*d, s + a*b
__device__ __forceinline__ float pr2(float a, float b, float c, float d) { return __fmaf_rn(a, b, fmul(c, d)); }
__device__ __forceinline__ float pd2(float a, float b, float c, float d) { return __fmaf_rn(a, b, -fmul(c, d)); }
__device__ __forceinline__ float acc(float s, float a, float b) { return __fmaf_rn(a, b, s); }
// DotV, CrossV, UnitV, FaceNormal(Unit) of inc/util.h:367-432
__device__ __forceinline__ float dotv(v3 a, v3 b) { return acc(pr2(a.x, b.x, a.y, b.y), a.z, b.z); }
__device__ __forceinline__ v3 crossv(v3 a, v3 b)
{
    return V(pd2(a.y, b.z, a.z, b.y), pd2(a.z, b.x, a.x, b.z), pd2(a.x, b.y, a.y, b.x));
}
__device__ __forceinline__ v3 unitv(v3 a) { return vmuls(a, __fdiv_rn(1.0f, __fsqrt_rn(dotv(a, a)))); }
__device__ __forceinline__ v3 face_normal(v3 a, v3 b, v3 c) { return crossv(vsub(b, a), vsub(c, a)); }
__device__ __forceinline__ v3 face_normal_unit(v3 a, v3 b, v3 c) { return unitv(face_normal(a, b, c)); }

__device__ __forceinline__ void load_face(const float *X, int nf, int f, v3 &a, v3 &b, v3 &c)
{
    a = V(X[f], X[f + nf], X[f + 2LL * nf]);
    b = V(X[f + 3LL * nf], X[f + 4LL * nf], X[f + 5LL * nf]);
    c = V(X[f + 6LL * nf], X[f + 7LL * nf], X[f + 8LL * nf]);
}

// TriangleBinOverlap2D_AxisGap (util_tribin.h:92-125).
__device__ bool axis_gap(int axis, float v1x, float v1y, float v2x, float v2y, float v3x, float v3y, float rmx,
                         float rmy, float rMx, float rMy)
{
    float ex = 0.f, ey = 0.f;
    if (axis == 0) { ex = 1.f; ey = 0.f; }
    if (axis == 1) { ex = 0.f; ey = 1.f; }
    if (axis == 2) { ex = fsub(v2y, v1y); ey = fsub(v1x, v2x); }
    if (axis == 3) { ex = fsub(v3y, v2y); ey = fsub(v2x, v3x); }
    if (axis == 4) { ex = fsub(v1y, v3y); ey = fsub(v3x, v1x); }
    const float a1 = pr2(v1x, ex, v1y, ey), a2 = pr2(v2x, ex, v2y, ey), a3 = pr2(v3x, ex, v3y, ey);
    const float r1 = pr2(rmx, ex, rmy, ey), r2 = pr2(rMx, ex, rmy, ey), r3 = pr2(rmx, ex, rMy, ey),
                r4 = pr2(rMx, ex, rMy, ey);
    float t = fmaxf(fmaxf(a1, a2), a3);
    float r = fminf(fminf(fminf(r1, r2), r3), r4);
    const bool b = t < r;
    t = fminf(fminf(a1, a2), a3);
    r = fmaxf(fmaxf(fmaxf(r1, r2), r3), r4);
    return b || (r < t);
}

// TrianglePlaneCutsBox and TriangleBinOverlap3D (util_tribin.h:60-150).
__device__ bool tri_box_overlap(v3 vm, v3 vM, v3 a, v3 b, v3 c)
{
    const v3 n = face_normal(a, b, c);
    const v3 cc = V(n.x > 0 ? fsub(vM.x, vm.x) : 0.f, n.y > 0 ? fsub(vM.y, vm.y) : 0.f, n.z > 0 ? fsub(vM.z, vm.z) : 0.f);
    const float d = dotv(n, vm), d1 = dotv(n, vsub(cc, a)), d2 = dotv(n, vsub(vsub(vsub(vM, vm), cc), a));
    if (!(fmul(fadd(d, d1), fadd(d, d2)) <= 0)) return false;
    for (int k = 0; k < 5; k++)
        if (axis_gap(k, a.x, a.y, b.x, b.y, c.x, c.y, vm.x, vm.y, vM.x, vM.y)) return false;
    for (int k = 0; k < 5; k++)
        if (axis_gap(k, a.y, a.z, b.y, b.z, c.y, c.z, vm.y, vm.z, vM.y, vM.z)) return false;
    for (int k = 0; k < 5; k++)
        if (axis_gap(k, a.z, a.x, b.z, b.x, c.z, c.x, vm.z, vm.x, vM.z, vM.x)) return false;
    return true;
}

// CheckPointInTriangleAABB, eps = 2 FLT_EPSILON (util_tribin.h:190-209).
__device__ __forceinline__ bool point_in_face_aabb(v3 p, v3 a, v3 b, v3 c)
{
    const float eps = FLT_EPSILON * 2.0f;
    return tri_box_overlap(vsubs(p, eps), vadds(p, eps), a, b, c);
}

// CheckPointInTriangleExtended, eps = FLT_EPSILON (util.h:521-543).  With an
// undefined point (a ray parallel to the face) every test is false and the
// point passes, as there.
__device__ bool point_in_tri_ext(v3 p, v3 a, v3 b, v3 c, v3 n)
{
    const float eps = FLT_EPSILON;
    v3 e = unitv(crossv(vsub(b, a), n));
    if (dotv(vsub(a, p), e) <= -eps) return false;
    e = unitv(crossv(vsub(c, b), n));
    if (dotv(vsub(b, p), e) <= -eps) return false;
    e = unitv(crossv(vsub(a, c), n));
    if (dotv(vsub(c, p), e) <= -eps) return false;
    return true;
}

// x-distance from the point to the face plane along +x
// (mesh_voxelizer_voxelize.cu:283, geometry_bins_gpu.cu:247).
__device__ __forceinline__ float xray_dist(v3 a, v3 p, v3 n)
{
    return acc(acc(fsub(a.x, p.x), fsub(a.y, p.y), __fdiv_rn(n.y, n.x)), fsub(a.z, p.z), __fdiv_rn(n.z, n.x));
}

// Cell centre of Cu_Voxelize_V1: X + I dx in FP32, + 0.5 dx in FP64, to FP32.
__device__ __forceinline__ float cell_centre(float X, int I, float dx)
{
    return (float)__dadd_rn((double)__fmaf_rn((float)I, dx, X), 0.5 * (double)dx);
}

__device__ __forceinline__ float fminf3(float a, float b, float c) { return fminf(fminf(a, b), c); }
__device__ __forceinline__ float fmaxf3(float a, float b, float c) { return fmaxf(fmaxf(a, b), c); }

// ---- binning --------------------------------------------------------------
// The reference indexes bins as coordinate x density and cells as
// coordinate x N (geometry_bins_gpu.cu:174-560, mesh_voxelizer_voxelize.cu:
// 253-258), which is right on the unit cube it is built for but disagrees
// with its own bin sizes L / density on any other box.  Here bins are
// indexed per axis with sx = density / Lx (sy, sz alike) and cells with
// cpl = Nx / Lx (cells per unit length): the same floats on the unit cube,
// consistent bins on a channel.
struct BinGrid {
    float dxL, Lx, Ly, Lz, L0x, L0y, L0z;
    float sx, sy, sz, cpl;
    int dens, Nx, Ny, Nz;
};

// Cu_ComputeVoxelRayIndicators_1D / _MD, 3D branches (geometry_bins_gpu.cu:24-280).
__global__ void k_ray_filter(const float *X, int nf, BinGrid g, int md, int *found)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    v3 a, b, c;
    load_face(X, nf, f, a, b, c);
    const v3 n = face_normal_unit(a, b, c);
    const float dxL = g.dxL, dxo2 = fmul(0.5f, g.dxL);
    int hit = 0;
    const int iymin = (int)fmul(fminf3(a.y, b.y, c.y), g.cpl), iymax = (int)fmul(fmaxf3(a.y, b.y, c.y), g.cpl);
    const int izmin = (int)fmul(fminf3(a.z, b.z, c.z), g.cpl), izmax = (int)fmul(fmaxf3(a.z, b.z, c.z), g.cpl);
    if (!md) {
        for (int iz = izmin; iz <= izmax && !hit; iz++)
            for (int iy = iymin; iy <= iymax && !hit; iy++) {
                const v3 p = V(0.f, acc(dxo2, dxL, (float)iy), acc(dxo2, dxL, (float)iz));
                v3 q = p;
                q.x = fadd(q.x, xray_dist(a, p, n));
                if (point_in_face_aabb(q, a, b, c)) hit = 1;
            }
    } else {
        const int ixmin = (int)fmul(fminf3(a.x, b.x, c.x), g.cpl), ixmax = (int)fmul(fmaxf3(a.x, b.x, c.x), g.cpl);
        for (int p = 1; p < 27 && !hit; p++) {
            if (!lat_half(3, p)) continue;
            const v3 ray = V((float)lat_c(3, 0, p), (float)lat_c(3, 1, p), (float)lat_c(3, 2, p));
            const float den = dotv(ray, n);
            for (int iz = izmin; iz <= izmax && !hit; iz++)
                for (int iy = iymin; iy <= iymax && !hit; iy++)
                    for (int ix = ixmin; ix <= ixmax && !hit; ix++) {
                        const v3 pc = V(acc(dxo2, dxL, (float)ix), acc(dxo2, dxL, (float)iy), acc(dxo2, dxL, (float)iz));
                        const float d = __fdiv_rn(dotv(vsub(a, pc), n), den);
                        const v3 q = V(acc(pc.x, ray.x, d), acc(pc.y, ray.y, d), acc(pc.z, ray.z, d));
                        if (point_in_tri_ext(q, a, b, c, n)) hit = 1;
                    }
        }
    }
    found[f] = hit;
}

struct RankFaces {   // copy_if + scatter of the ray indicators: rank of each kept face
    const int *found;
    int *rank;
    __device__ bool pred(int f) const { return found[f] != 0; }
    __device__ void emit(int f, int r) const { rank[f] = r; }
};

// Cu_ComputeBoundingBoxLimits3D (geometry_bins_gpu.cu:423-560): the bins of
// the face's grown bounding box it overlaps, in slot [counter][rank].
__global__ void k_bin_limits(const float *X, int nf, BinGrid g, const int *rank, int n_filtered, int n_limits,
                             int n_bins, int *key, int *val, int *bad)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int r = rank[f];
    if (r < 0) return;
    v3 a, b, c;
    load_face(X, nf, f, a, b, c);
    const float dx = fadd(g.dxL, FLT_EPSILON);
    const v3 bm = V(fminf3(a.x, b.x, c.x), fminf3(a.y, b.y, c.y), fminf3(a.z, b.z, c.z));
    const v3 bM = V(fmaxf3(a.x, b.x, c.x), fmaxf3(a.y, b.y, c.y), fmaxf3(a.z, b.z, c.z));
    const float Lxd = fadd(g.Lx, dx), Lyd = fadd(g.Ly, dx), Lzd = fadd(g.Lz, dx);
    if ((bm.x < -dx && bM.x < -dx) || (bm.x > Lxd && bM.x > Lxd)) return;
    if ((bm.y < -dx && bM.y < -dx) || (bm.y > Lyd && bM.y > Lyd)) return;
    if ((bm.z < -dx && bM.z < -dx) || (bm.z > Lzd && bM.z > Lzd)) return;
    const int xl = (int)fmul(bm.x, g.sx) - 1, yl = (int)fmul(bm.y, g.sy) - 1, zl = (int)fmul(bm.z, g.sz) - 1;
    const int xL = (int)fmul(bM.x, g.sx) + 1, yL = (int)fmul(bM.y, g.sy) + 1, zL = (int)fmul(bM.z, g.sz) + 1;
    int counter = 0;
    for (int K = zl; K < zL + 1; K++)
        for (int J = yl; J < yL + 1; J++)
            for (int I = xl; I < xL + 1; I++) {
                const v3 vm = V(fsub(fmul((float)I, g.L0x), dx), fsub(fmul((float)J, g.L0y), dx), fsub(fmul((float)K, g.L0z), dx));
                const v3 vM = V(fadd(fmul((float)(I + 1), g.L0x), dx), fadd(fmul((float)(J + 1), g.L0y), dx),
                                fadd(fmul((float)(K + 1), g.L0z), dx));
                if (tri_box_overlap(vm, vM, a, b, c) && counter < n_limits) {
                    // The reference writes bins outside the grid unchecked; refuse them.
                    if (I < 0 || J < 0 || K < 0 || I >= g.dens || J >= g.dens || K >= g.dens) {
                        atomicExch(bad, 1);
                    } else {
                        const long long s = r + (long long)counter * n_filtered;
                        key[s] = I + g.dens * J + g.dens * g.dens * K;
                        val[s] = f;
                    }
                    counter++;
                }
            }
    (void)n_bins;
}

__global__ void k_bin_count(const int *key, long long n, int n_bins, int *cnt)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && key[i] < n_bins) atomicAdd(&cnt[key[i]], 1);
}

// Exclusive scan of n ints in one CTA of 1024 threads (set-up sizes).
__global__ void __launch_bounds__(1024) k_scan_small(const int *in, int n, int *out, int *total)
{
    __shared__ int s[1024];
    const int per = (n + 1023) / 1024;
    const int lo = threadIdx.x * per, hi = min(n, lo + per);
    int sum = 0;
    for (int i = lo; i < hi; i++) sum += in[i];
    s[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int v = (threadIdx.x >= o) ? s[threadIdx.x - o] : 0;
        __syncthreads();
        s[threadIdx.x] += v;
        __syncthreads();
    }
    int run = s[threadIdx.x] - sum;
    for (int i = lo; i < hi; i++) {
        const int v = in[i];
        out[i] = run;
        run += v;
    }
    if (threadIdx.x == 1023) *total = s[1023];
}

// Entries land in their bin in arbitrary order, each carrying its slot index;
// k_bin_order then sorts every bin by slot, which is the reference's stable
// order (counter, rank).
__global__ void k_bin_place(const int *key, long long n, int n_bins, const int *start, int *fillc, int *slot)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || key[i] >= n_bins) return;
    const int k = key[i];
    slot[start[k] + atomicAdd(&fillc[k], 1)] = (int)i;
}

__global__ void k_bin_order(int n_bins, const int *cnt, int *start, int *slot, const int *val, int *ids)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_bins) return;
    const int m = cnt[k], s0 = start[k];
    for (int i = 1; i < m; i++) {
        const int v = slot[s0 + i];
        int j = i - 1;
        while (j >= 0 && slot[s0 + j] > v) {
            slot[s0 + j + 1] = slot[s0 + j];
            j--;
        }
        slot[s0 + j + 1] = v;
    }
    for (int i = 0; i < m; i++) ids[s0 + i] = val[slot[s0 + i]];
    if (m == 0) start[k] = 0;   // empty bins keep the reset value
}

// ---- voxelization ---------------------------------------------------------
constexpr int MC3 = 64;
constexpr int N_LEFT = 2, N_RIGHT = 1;   // neighbour rows of -x / +x in 3D

struct BinsView {
    const int *n, *N, *ids;
    int density, n_bins;
    float sx, sy, sz;
};

// Bin of a point (per-axis bins per unit length, see BinGrid).
__device__ __forceinline__ int bin_of(const BinsView &b, v3 p)
{
    const int D = b.density;
    return (int)fmul(p.x, b.sx) + D * (int)fmul(p.y, b.sy) + D * D * (int)fmul(p.z, b.sz);
}

// Cu_Voxelize_V1 (mesh_voxelizer_voxelize.cu:203-351), one CTA of 64 threads
// per block: each cell takes the closest face of its bin crossed by its +x
// ray (first in bin order on ties); the side of that face makes it a guard
// or a solid; three synchronous sweeps carry both along x in the block.
__global__ void __launch_bounds__(MC3) k_voxelize(const int *ids, long long nmb, float dxL, const float *X, int nf,
                                                  BinsView bins, const float *fX, int *cmask)
{
    __shared__ int s_m[MC3];
    __shared__ int s_any;
    const int b = ids[blockIdx.x];
    const int t = threadIdx.x, I = t & 3, J = (t >> 2) & 3, K = t >> 4;
    if (t == 0) s_any = 0;
    const v3 p = V(cell_centre(fX[b], I, dxL), cell_centre(fX[b + nmb], J, dxL), cell_centre(fX[b + 2 * nmb], K, dxL));
    const int gb = bin_of(bins, p);
    const int n_f = (gb >= 0 && gb < bins.n_bins) ? bins.n[gb] : 0;
    int pmin = -1, mask = CELL_INTERIOR;
    float dmin = 1.0f;
    for (int k = 0; k < n_f; k++) {
        v3 a, bb, c;
        load_face(X, nf, bins.ids[bins.N[gb] + k], a, bb, c);
        const v3 n = face_normal_unit(a, bb, c);
        const float d = xray_dist(a, p, n);
        v3 q = p;
        q.x = fadd(q.x, d);
        if ((fabsf(d) < dmin || pmin == -1) && point_in_face_aabb(q, a, bb, c)) {
            dmin = fabsf(d);
            pmin = k;
            if (d > 0 && n.x < 0) mask = -10;   // LL
            if (d < 0 && n.x < 0) mask = -11;   // LR
            if (d > 0 && n.x > 0) mask = -12;   // RL
            if (d < 0 && n.x > 0) mask = -13;   // RR
        }
    }
    __syncthreads();
    if (pmin != -1) atomicOr(&s_any, 1);
    __syncthreads();
    if (!s_any) return;
    if (mask == -10 || mask == -13) mask = CELL_GUARD;
    if (mask == -11 || mask == -12) mask = CELL_SOLID;
    s_m[t] = mask;
    __syncthreads();
    for (int l = 0; l < 3; l++) {
        if (I > 0) {
            const int nm = s_m[t - 1];
            if (nm == CELL_GUARD && mask == CELL_INTERIOR) mask = CELL_GUARD;
            if (nm == CELL_SOLID && mask != CELL_GUARD) mask = CELL_SOLID;
        }
        if (I < 3) {
            const int nm = s_m[t + 1];
            if (nm == CELL_GUARD && mask == CELL_INTERIOR) mask = CELL_GUARD;
            if (nm == CELL_SOLID && mask != CELL_GUARD) mask = CELL_SOLID;
        }
        __syncthreads();
        s_m[t] = mask;
        __syncthreads();
    }
    const long long o = (long long)b * MC3 + t;
    const int orig = cmask[o];
    if (mask == CELL_SOLID || (orig != CELL_GHOST && orig != CELL_INTERFACE)) cmask[o] = mask;
}

// Cu_Voxelize_Propagate_Right / _Left (mesh_voxelizer_propagate.cu:97-215):
// one warp per block, lane r < 16 walks cell row r along the chain of
// same-level neighbours starting at a block without one on the other side.
__global__ void k_propagate(const int *ids, int n, long long nmb, const int *nbr, int *cmask, int dir, int dense)
{
    const int kap = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int r = threadIdx.x & 31;
    if (kap >= n || r >= 16) return;
    const int b = ids[kap];
    const int from = dir > 0 ? N_LEFT : N_RIGHT, to = dir > 0 ? N_RIGHT : N_LEFT;
    const int edge = dir > 0 ? 3 : 0;
    const int start = nbr[b + from * nmb];
    if (start >= 0) return;
    int status = cmask[(long long)b * MC3 + 4 * r + edge];
    if (start == N_SPECID && status != CELL_GUARD) status = CELL_SOLID;
    int nb = nbr[b + to * nmb];
    for (int k = 0; nb > -1 && k < 1000; k++) {
        int m[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            m[i] = cmask[(long long)nb * MC3 + 4 * r + i];
            if (status == CELL_SOLID && m[i] != CELL_GUARD) m[i] = CELL_SOLID;
        }
        status = m[edge];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            if ((dir < 0 || dense) && m[i] == CELL_GUARD) m[i] = CELL_INTERIOR;
            cmask[(long long)nb * MC3 + 4 * r + i] = m[i];
        }
        nb = nbr[nb + to * nmb];
    }
}

// Cu_Voxelize_UpdateMasks (mesh_voxelizer_masks.cu:227-256).
__global__ void k_solid_blocks(const int *ids, int n, const int *cmask, int *bmask)
{
    const int kap = blockIdx.x * blockDim.x + threadIdx.x;
    if (kap >= n) return;
    const int b = ids[kap];
    for (int t = 0; t < MC3; t++)
        if (cmask[(long long)b * MC3 + t] == CELL_SOLID) {
            bmask[b] = BLOCK_SOLID;
            return;
        }
}

__device__ __forceinline__ bool eligible(const int *nbr, long long nmb, int b)
{
    for (int q = 0; q < 27; q++)
        if (nbr[b + q * nmb] == N_SKIPID) return false;
    return true;
}

// Cu_MarkBlocks_MarkBoundary (mesh_voxelizer_refine.cu:20-88): solid blocks
// next to a regular block become solid-boundary blocks, marked for refinement.
// Only regular masks are read and only solid ones rewritten.
__global__ void k_mark_boundary(int n, long long nmb, int L, int hit_max, int *ref, int *bmask, const int *nbr,
                                const int *level)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || level[b] != L || bmask[b] != BLOCK_SOLID) return;
    bool mark = false;
    for (int q = 0; q < 27 && !mark; q++) {
        const int nb = nbr[b + q * nmb];
        if (nb > -1 && bmask[nb] == BLOCK_REGULAR) mark = true;
    }
    if (!mark || ref[b] != REF_UNREFINED) return;
    bmask[b] = BLOCK_SOLIDB;
    if (!hit_max && eligible(nbr, nmb, b)) ref[b] = REF_MARK_REFINE;
}

// Cu_MarkBlocks_MarkExterior (mesh_voxelizer_refine.cu:95-160).
__global__ void k_mark_exterior(int n, long long nmb, int L, int hit_max, int *ref, int *bmask, const int *nbr,
                                const int *level)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || level[b] != L) return;
    bool mark = false;
    for (int q = 0; q < 27 && !mark; q++) {
        const int nb = nbr[b + q * nmb];
        if (nb > -1 && bmask[nb] == BLOCK_SOLIDB) mark = true;
    }
    if (!mark || ref[b] != REF_UNREFINED) return;
    if (!hit_max && eligible(nbr, nmb, b)) ref[b] = REF_INDET_E;
    if (bmask[b] == BLOCK_REGULAR) bmask[b] = BLOCK_SOLIDA;
}

// Cu_MarkBlocks_Propagate (mesh_voxelizer_refine.cu:252-345): the marking
// front alternates between ref = 11 (even passes read it) and tmp = 12.
__global__ void k_mark_propagate(int n, long long nmb, int L, int j, int *ref, const int *bmask, const int *nbr,
                                 const int *level, int *tmp)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || level[b] != L) return;
    const bool even = (j % 2) == 0;
    if (!(bmask[b] > -1 || (j == 0 && bmask[b] == BLOCK_SOLID))) return;
    bool mark = false;
    for (int q = 0; q < 27 && !mark; q++) {
        const int nb = nbr[b + q * nmb];
        if (nb < 0) continue;
        if (even ? ref[nb] == REF_INDET_E : tmp[nb] == REF_INDET_O) mark = true;
    }
    const bool C = even ? ref[b] == REF_UNREFINED : tmp[b] == -1;
    if (!mark || !C || !eligible(nbr, nmb, b)) return;
    if (even) tmp[b] = REF_INDET_O;
    else ref[b] = REF_INDET_E;
}

// Cu_MarkBlocks_Finalize (mesh_voxelizer_refine.cu:352-370).
__global__ void k_mark_finalize(int n, int *ref, int *tmp)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    if (ref[b] == REF_INDET_E || tmp[b] == REF_INDET_O) {
        ref[b] = REF_MARK_REFINE;
        tmp[b] = -1;
    }
}

// Cu_MarkBlocks_UpdateSolidChildren (mesh_voxelizer_refine.cu:203-245).  The
// child index is formed from cblock_ID_nbr_child even when the block has no
// children, as there.
__global__ void k_solid_children(int n, long long nmb, int L, const int *bmask, int *nbr, const int *nbr_child,
                                 const int *level)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || level[b] != L || bmask[b] != BLOCK_SOLID) return;
    for (int p = 0; p < 8; p++) {
        const int ch = nbr_child[b] + p;
        if (ch < 0) continue;
        if (nbr[ch + N_LEFT * nmb] == N_SKIPID) nbr[ch + N_LEFT * nmb] = N_SPECID;
        if (nbr[ch + N_RIGHT * nmb] == N_SKIPID) nbr[ch + N_RIGHT * nmb] = N_SPECID;
    }
}

// Neighbour block and cell of cell (I, J, K) along direction p of the
// 27-direction table (util_index.h:144-190); s_nbr in lexicographic slots.
__device__ __forceinline__ void nbr_of(const int *s_nbr, int I, int J, int K, int p, int &nb, int &nc)
{
    const int Ip = I + lat_c(3, 0, p), Jp = J + lat_c(3, 1, p), Kp = K + lat_c(3, 2, p);
    const int S = (Ip < 0 ? 0 : (Ip < 4 ? 1 : 2)) + 3 * (Jp < 0 ? 0 : (Jp < 4 ? 1 : 2)) + 9 * (Kp < 0 ? 0 : (Kp < 4 ? 1 : 2));
    nb = s_nbr[S];
    nc = (Ip & 3) + 4 * (Jp & 3) + 16 * (Kp & 3);
}

// Cu_MarkBlocks_CheckMasks_S1<AP,1> (mesh_voxelizer_masks.cu:19-151): cells of
// leaf solid-adjacent blocks next to a solid cell are boundary cells; the
// flags go to bnd_bits (the reference's upper half of cells_ID_mask), the
// count to tmp and the block is flagged on a boundary.
__global__ void __launch_bounds__(MC3) k_check_masks(const int *ids, long long nmb, const int *cmask, const int *bmask,
                                                     const int *nbr, const int *nbr_child, int *onb, int *tmp,
                                                     unsigned long long *bits)
{
    __shared__ int s_nbr[27];
    __shared__ int s_cnt;
    const int b = ids[blockIdx.x];
    if (!(nbr_child[b] < 0 && bmask[b] < 0 && bmask[b] != BLOCK_SOLID)) return;
    const int t = threadIdx.x, I = t & 3, J = (t >> 2) & 3, K = t >> 4;
    if (t < 27) s_nbr[t] = nbr[b + (long long)lat_map(3, t) * nmb];
    if (t == 0) s_cnt = 0;
    __syncthreads();
    const int curr = cmask[(long long)b * MC3 + t];
    bool near = false;
    for (int p = 0; p < 27 && !near; p++) {
        int nb, nc;
        nbr_of(s_nbr, I, J, K, p, nb, nc);
        if (nb >= 0 && cmask[(long long)nb * MC3 + nc] == CELL_SOLID) near = true;
    }
    const bool set = near && curr != CELL_SOLID;
    const unsigned m = __ballot_sync(0xffffffffu, set);
    if ((t & 31) == 0 && m) {
        atomicOr(&bits[b], (unsigned long long)m << (t & 32));
        atomicAdd(&s_cnt, __popc(m));
    }
    __syncthreads();
    if (t == 0 && s_cnt > 0) {
        tmp[b] = s_cnt;
        onb[b] = 1;
    }
}

// Cu_MarkBlocks_CheckMasks_S2 (mesh_voxelizer_masks.cu:158-179).
__global__ void k_apply_masks(const int *ids, int n, const int *onb, const unsigned long long *bits, int *cmask)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)n * MC3) return;
    const int b = ids[g / MC3], t = (int)(g % MC3);
    if (onb[b] == 1 && ((bits[b] >> t) & 1ull)) cmask[(long long)b * MC3 + t] = CELL_BOUNDARY;
}

__global__ void k_fill_range(int *p, int n, int v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// M_Geometry_Voxelize_S3 counts (mesh_voxelizer.cu:193-196): sum and number
// of positive entries of tmp over [0, n).
__global__ void k_solid_counts(const int *tmp, int n, unsigned long long *sum, int *cnt)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = (b < n) ? tmp[b] : 0;
    const unsigned long long s = __reduce_add_sync(0xffffffffu, (unsigned)(v > 0 ? v : 0));
    const unsigned c = __reduce_add_sync(0xffffffffu, (unsigned)(v > 0));
    if ((threadIdx.x & 31) == 0) {
        if (s) atomicAdd(sum, s);
        if (c) atomicAdd(cnt, (int)c);
    }
}

struct WallSlots {   // copy_if + scatter: slot of every block with boundary cells
    const int *tmp;
    int *onb_solid;
    __device__ bool pred(int b) const { return tmp[b] > 0; }
    __device__ void emit(int b, int r) const { onb_solid[b] = r; }
};

__global__ void k_fill_float(float *p, long long n, float v)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// ---- link lengths ---------------------------------------------------------
// Cu_LinkLengthComputation (mesh_voxelizer_links.cu:26-196): per cell of a
// wall block, the distance along each of the 26 directions to the faces of
// its link bin met within one cell, in cell units; boundary cells keep them.
// The running minimum compares the new distance with the stored normalised
// one, as the reference does.
__global__ void __launch_bounds__(MC3) k_links(const int *ids, long long nmb, float dxL, const float *X, int nf,
                                               BinsView bins, const float *fX, const int *cmask, const int *onb_solid,
                                               long long ncb, float *Xb)
{
    const int b = ids[blockIdx.x];
    const int slot = onb_solid[b];
    if (slot < 0) return;
    const int t = threadIdx.x, I = t & 3, J = (t >> 2) & 3, K = t >> 4;
    const v3 p = V(cell_centre(fX[b], I, dxL), cell_centre(fX[b + nmb], J, dxL), cell_centre(fX[b + 2 * nmb], K, dxL));
    const int gb = bin_of(bins, p);
    const int n_f = (gb >= 0 && gb < bins.n_bins) ? bins.n[gb] : 0;
    if (n_f <= 0) return;
    float dQ[27];
#pragma unroll
    for (int q = 0; q < 27; q++) dQ[q] = -1.0f;
    const float lim = fadd(dxL, FLT_EPSILON);
    for (int k = 0; k < n_f; k++) {
        v3 a, bb, c;
        load_face(X, nf, bins.ids[bins.N[gb] + k], a, bb, c);
        const v3 n = face_normal_unit(a, bb, c);
        const float num = dotv(vsub(a, p), n);
#pragma unroll
        for (int q = 1; q < 27; q++) {
            const v3 ray = V((float)lat_c(3, 0, q), (float)lat_c(3, 1, q), (float)lat_c(3, 2, q));
            const float den = dotv(ray, n);
            if (den == 0.0f) continue;
            const float d = __fdiv_rn(num, den);
            if (d > 0.0f && d < lim) {
                const v3 qp = V(acc(p.x, ray.x, d), acc(p.y, ray.y, d), acc(p.z, ray.z, d));
                if (point_in_tri_ext(qp, a, bb, c, n)) {
                    if (d < dQ[q] || dQ[q] < 0) dQ[q] = __fdiv_rn(d, dxL);
                }
            }
        }
    }
    if (cmask[(long long)b * MC3 + t] != CELL_BOUNDARY) return;
#pragma unroll
    for (int q = 1; q < 27; q++) Xb[(long long)slot * MC3 + t + q * ncb] = dQ[q];
}

// Cu_LinkLengthValidation (mesh_voxelizer_links.cu:203-358): a boundary cell
// without a link towards a solid neighbour gets the length 1/2.  The
// neighbour's mask is read at the neighbour's slot number used as a block ID,
// as the reference does; only the 1/2 corrections are ever stored, and each
// goes to an entry that was negative, so concurrent threads agree.
__global__ void __launch_bounds__(MC3) k_links_validate(const int *ids, long long nmb, const int *nbr,
                                                        const int *cmask, const int *onb_solid, long long ncb,
                                                        float *Xb)
{
    __shared__ int s_nbr[27];
    const int b = ids[blockIdx.x];
    const int slot = onb_solid[b];
    if (slot < 0) return;
    const int t = threadIdx.x, I = t & 3, J = (t >> 2) & 3, K = t >> 4;
    if (t < 27) s_nbr[t] = nbr[b + (long long)lat_map(3, t) * nmb];
    __syncthreads();
    const int mask_p = cmask[(long long)b * MC3 + t];
    for (int p = 1; p < 27; p++) {
        if (!lat_half(3, p)) continue;
        int nb, nc;
        nbr_of(s_nbr, I, J, K, p, nb, nc);
        if (nb > -1) nb = onb_solid[nb];
        if (nb <= -1) continue;
        const int pb = lat_pb(3, p);
        float *xp = &Xb[(long long)slot * MC3 + t + p * ncb];
        float *xq = &Xb[(long long)nb * MC3 + nc + pb * ncb];
        const float dp = *xp, dq = *xq;
        const int mask_pb = cmask[(long long)nb * MC3 + nc];
        if (mask_p == CELL_BOUNDARY && dp < 0 && mask_pb == CELL_SOLID) *xp = 0.5f;
        if (mask_pb == CELL_BOUNDARY && dq < 0 && mask_p == CELL_SOLID) *xq = 0.5f;
    }
}

unsigned grid_for(long long n, int per = 256) { return (unsigned)((n + per - 1) / per); }

}  // namespace geo
}  // namespace agal

using namespace agal;
using namespace agal::geo;

namespace {

void free_bins(agal_bins_d &b)
{
    if (b.n) cudaFree(b.n);
    if (b.N) cudaFree(b.N);
    if (b.ids) cudaFree(b.ids);
    b = agal_bins_d{};
}

// Constants of the Bins constructor (geometry_bins.h:106-170) at bin level L.
BinGrid bin_grid(const agal_ctx *c, int L, int *nbl_out)
{
    const agal_params &P = c->P;
    const float Lx = (float)P.L_c, Ly = (float)(P.L_fy * Lx), Lz = (float)(P.L_fz * Lx);
    const int Nx = P.Nx, Ny = (int)(Nx * (Ly / Lx)), Nz = (int)(Nx * (Lz / Lx));
    int nbl = std::min(P.G_BIN_LEVELS, P.MAX_LEVELS_WALL);
    nbl = std::max(1, std::min(nbl, 16));
    if (nbl_out) *nbl_out = nbl;
    BinGrid g;
    g.Lx = Lx; g.Ly = Ly; g.Lz = Lz;
    float dxf = Lx / (float)Nx, L0x = Lx / (float)P.G_BIN_DENSITY, L0y = Ly / (float)P.G_BIN_DENSITY,
          L0z = Lz / (float)P.G_BIN_DENSITY;
    int dens = P.G_BIN_DENSITY, nx = Nx, ny = Ny, nz = Nz;
    for (int l = 1; l <= L; l++) {
        dens *= 2;
        dxf *= 0.5f; L0x *= 0.5f; L0y *= 0.5f; L0z *= 0.5f;
        nx *= 2; ny *= 2; nz *= 2;
    }
    g.dxL = dxf; g.L0x = L0x; g.L0y = L0y; g.L0z = L0z;
    g.dens = dens; g.Nx = nx; g.Ny = ny; g.Nz = nz;
    g.sx = (float)dens / Lx; g.sy = (float)dens / Ly; g.sz = (float)dens / Lz;
    g.cpl = (float)nx / Lx;
    return g;
}

// Bins::G_MakeBinsGPU (md = 0) / G_MakeBinsGPU_MD (md = 1) at bin level L.
int make_bins(agal_ctx *c, int L, int md, agal_bins_d &out)
{
    int nbl = 1;
    const BinGrid g = bin_grid(c, L, &nbl);
    const int nf = c->n_faces;
    const long long n_bins = (long long)g.dens * g.dens * g.dens;
    if (n_bins > (1LL << 30)) return agal_set_err(c, AGAL_ERR_PARAM, "bin grid too large");
    const int spec = c->P.G_BIN_SPEC;
    const int n_limits = (2 + spec) * (2 + spec) * (2 + spec);
    const bool use_ray = md ? (c->P.MAX_LEVELS_WALL == L + 1) : !(L == nbl - 1 && nbl != c->P.MAX_LEVELS_WALL);
    int *found = nullptr, *rank = nullptr, *parts = nullptr, *small = nullptr;
    AGAL_CUDA(c, cudaMalloc(&found, sizeof(int) * std::max(nf, 1)));
    AGAL_CUDA(c, cudaMalloc(&rank, sizeof(int) * std::max(nf, 1)));
    AGAL_CUDA(c, cudaMalloc(&parts, sizeof(int) * std::max(cmp::parts_for(nf), 1)));
    AGAL_CUDA(c, cudaMalloc(&small, sizeof(int) * 4));
    int n_filtered = nf;
    if (nf > 0) k_fill_range<<<grid_for(nf), 256, 0, c->stream>>>(rank, nf, -1);
    if (use_ray) {
        if (nf > 0) k_ray_filter<<<grid_for(nf, 64), 64, 0, c->stream>>>(c->faces, nf, g, md, found);
        AGAL_CUDA(c, cmp::compact_async(c->stream, parts, small, RankFaces{found, rank}, nf));
        AGAL_CUDA(c, cudaMemcpyAsync(&n_filtered, small, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    } else {
        if (nf > 0) k_fill_range<<<grid_for(nf), 256, 0, c->stream>>>(found, nf, 1);
        AGAL_CUDA(c, cmp::compact_async(c->stream, parts, small, RankFaces{found, rank}, nf));
    }
    const long long n_lim = (long long)n_limits * n_filtered;
    int *key = nullptr, *val = nullptr, *cnt = nullptr, *start = nullptr, *fillc = nullptr, *slot = nullptr;
    AGAL_CUDA(c, cudaMalloc(&key, sizeof(int) * std::max(n_lim, 1LL)));
    AGAL_CUDA(c, cudaMalloc(&val, sizeof(int) * std::max(n_lim, 1LL)));
    AGAL_CUDA(c, cudaMalloc(&cnt, sizeof(int) * n_bins));
    AGAL_CUDA(c, cudaMalloc(&start, sizeof(int) * n_bins));
    AGAL_CUDA(c, cudaMalloc(&fillc, sizeof(int) * n_bins));
    if (n_lim > 0) k_fill_range<<<grid_for(n_lim), 256, 0, c->stream>>>(key, (int)n_lim, (int)n_bins);
    AGAL_CUDA(c, cudaMemsetAsync(cnt, 0, sizeof(int) * n_bins, c->stream));
    AGAL_CUDA(c, cudaMemsetAsync(fillc, 0, sizeof(int) * n_bins, c->stream));
    AGAL_CUDA(c, cudaMemsetAsync(small, 0, sizeof(int) * 4, c->stream));
    if (nf > 0)
        k_bin_limits<<<grid_for(nf, 64), 64, 0, c->stream>>>(c->faces, nf, g, rank, n_filtered, n_limits, (int)n_bins,
                                                              key, val, small + 1);
    if (n_lim > 0) k_bin_count<<<grid_for(n_lim), 256, 0, c->stream>>>(key, n_lim, (int)n_bins, cnt);
    k_scan_small<<<1, 1024, 0, c->stream>>>(cnt, (int)n_bins, start, small + 2);
    int host[4] = {0, 0, 0, 0};
    AGAL_CUDA(c, cudaMemcpyAsync(host, small, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream));
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    int rc = AGAL_OK;
    if (host[1]) {
        rc = agal_set_err(c, AGAL_ERR_PARAM, "geometry reaches bins outside the unit cube");
    } else {
        const long long ne = host[2];
        AGAL_CUDA(c, cudaMalloc(&slot, sizeof(int) * std::max(ne, 1LL)));
        free_bins(out);
        AGAL_CUDA(c, cudaMalloc(&out.ids, sizeof(int) * std::max(ne, 1LL)));
        if (n_lim > 0) k_bin_place<<<grid_for(n_lim), 256, 0, c->stream>>>(key, n_lim, (int)n_bins, start, fillc, slot);
        k_bin_order<<<grid_for(n_bins), 256, 0, c->stream>>>((int)n_bins, cnt, start, slot, val, out.ids);
        AGAL_CUDA(c, cudaGetLastError());
        out.n = cnt;
        out.N = start;
        cnt = start = nullptr;
        out.density = g.dens;
        out.sx = g.sx; out.sy = g.sy; out.sz = g.sz;
        out.n_bins = (int)n_bins;
        out.n_entries = ne;
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    for (void *p : {(void *)found, (void *)rank, (void *)parts, (void *)small, (void *)key, (void *)val, (void *)cnt,
                    (void *)start, (void *)fillc, (void *)slot})
        if (p) cudaFree(p);
    return rc;
}

int ensure_geometry_state(agal_ctx *c)
{
    if (!c->onb_solid) {
        AGAL_CUDA(c, cudaMalloc(&c->onb_solid, sizeof(int) * c->nmb));
        k_fill_range<<<grid_for(c->nmb), 256, 0, c->stream>>>(c->onb_solid, (int)c->nmb, -1);
    }
    if (!c->vox_tmp) {
        AGAL_CUDA(c, cudaMalloc(&c->vox_tmp, sizeof(int) * c->nmb));
        k_fill_range<<<grid_for(c->nmb), 256, 0, c->stream>>>(c->vox_tmp, (int)c->nmb, -1);
    }
    if (!c->bnd_bits) {
        AGAL_CUDA(c, cudaMalloc(&c->bnd_bits, sizeof(unsigned long long) * c->nmb));
        AGAL_CUDA(c, cudaMemsetAsync(c->bnd_bits, 0, sizeof(unsigned long long) * c->nmb, c->stream));
    }
    if (!c->Ff) {
        const size_t cs = (c->storage == AGAL_STORE_FP64) ? 8 : 4;
        AGAL_CUDA(c, cudaMalloc(&c->Ff, cs * 6 * c->nmb));
        AGAL_CUDA(c, cudaMemsetAsync(c->Ff, 0, cs * 6 * c->nmb, c->stream));
    }
    if (!c->geo_small) AGAL_CUDA(c, cudaMalloc(&c->geo_small, 64));
    if (!c->geo_parts) AGAL_CUDA(c, cudaMalloc(&c->geo_parts, sizeof(int) * std::max(cmp::parts_for(c->nmb), 1)));
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

BinsView view(const agal_bins_d &b) { return BinsView{b.n, b.N, b.ids, b.density, b.n_bins, b.sx, b.sy, b.sz}; }

}  // namespace

void agal_geometry_release(agal_ctx *c)
{
    for (auto &b : c->bins) free_bins(b);
    free_bins(c->bins_md);
    void *ptrs[] = {c->faces, c->onb_solid, c->X_b, c->vox_tmp, c->bnd_bits, c->Ff, c->geo_small, c->geo_parts,
                    c->wall_ids};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    c->faces = nullptr; c->onb_solid = nullptr; c->X_b = nullptr; c->vox_tmp = nullptr; c->bnd_bits = nullptr;
    c->Ff = nullptr; c->geo_small = nullptr; c->geo_parts = nullptr; c->wall_ids = nullptr;
}

namespace agal {
namespace geo {
__global__ void k_faces_soa(const float *aos, int nf, float *soa)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    for (int r = 0; r < 9; r++) soa[f + (long long)r * nf] = aos[(long long)f * 9 + r];
}

struct WallList {   // wall blocks of one level in ID-set order
    const int *ids, *onb, *onb_solid;
    int *out;
    __device__ bool pred(int k) const { const int b = ids[k]; return onb[b] == 1 && onb_solid[b] >= 0; }
    __device__ void emit(int k, int r) const { out[r] = ids[k]; }
};
}  // namespace geo
}  // namespace agal

namespace {
bool geo_ready(const agal_ctx *c) { return c && c->geometry_init && c->faces && c->dim == 3; }
// FP32 cell width of level L (ufloat_g_t), whatever the solver precision.
float geo_dx(const agal_ctx *c, int L) { return (float)((double)c->dx / std::pow(2.0, (double)L)); }
}  // namespace

int agal_wall_active(const agal_ctx *c)
{
    return c->onb_solid && c->X_b && c->P.S_BC_TYPE > 0 && c->n_solidb > 0;
}

int agal_build_wall_lists(agal_ctx *c)
{
    c->wall_off.assign(c->max_levels, 0);
    c->wall_n.assign(c->max_levels, 0);
    if (!c->onb_solid) return AGAL_OK;
    if (!c->wall_ids) AGAL_CUDA(c, cudaMalloc(&c->wall_ids, sizeof(int) * c->nmb));
    int off = 0;
    for (int L = 0; L < c->max_levels; L++) {
        c->wall_off[L] = off;
        const int n = c->n_ids[L];
        if (n <= 0) continue;
        WallList f{c->id_set + (long long)L * c->nmb, c->cblock_ID_onb, c->onb_solid, c->wall_ids + off};
        AGAL_CUDA(c, cmp::compact_async(c->stream, c->geo_parts, c->geo_small + 8, f, n));
        int cnt = 0;
        AGAL_CUDA(c, cudaMemcpyAsync(&cnt, c->geo_small + 8, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
        c->wall_n[L] = cnt;
        off += cnt;
    }
    return AGAL_OK;
}

extern "C" int agal_set_geometry(agal_ctx *c, const float *faces, long long n_faces)
{
    if (!c) return AGAL_ERR_PARAM;
    if (c->dim != 3) return agal_set_err(c, AGAL_ERR_UNSUPPORTED, "geometry: 3D velocity sets only");
    if (n_faces < 0 || n_faces > (1LL << 28) || (n_faces > 0 && !faces))
        return agal_set_err(c, AGAL_ERR_PARAM, "faces");
    int rc;
    if ((rc = ensure_geometry_state(c))) return rc;
    for (auto &b : c->bins) free_bins(b);
    free_bins(c->bins_md);
    if (c->faces) cudaFree(c->faces);
    c->faces = nullptr;
    const int nf = (int)n_faces;
    c->n_faces = nf;
    float *aos = nullptr;
    AGAL_CUDA(c, cudaMalloc(&c->faces, sizeof(float) * 9 * std::max(nf, 1)));
    AGAL_CUDA(c, cudaMalloc(&aos, sizeof(float) * 9 * std::max(nf, 1)));
    if (nf > 0) {
        AGAL_CUDA(c, cudaMemcpyAsync(aos, faces, sizeof(float) * 9 * nf, cudaMemcpyHostToDevice, c->stream));
        k_faces_soa<<<grid_for(nf), 256, 0, c->stream>>>(aos, nf, c->faces);
    }
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(aos);
    // Geometry::G_InitBins (geometry_bins.h:106-203).
    int nbl = 1;
    bin_grid(c, 0, &nbl);
    c->n_bin_levels = nbl;
    for (int L = 0; L < nbl; L++)
        if ((rc = make_bins(c, L, 0, c->bins[L]))) return rc;
    c->bin_level_md = -1;
    if (c->P.G_BIN_MAKE_LINKS) {
        c->bin_level_md = std::min(c->P.MAX_LEVELS_WALL, nbl) - 1;
        if ((rc = make_bins(c, c->bin_level_md, 1, c->bins_md))) return rc;
    }
    c->geometry_init = 1;   // Mesh::M_AddGeometry (mesh_init.cu:570-577)
    agal_drop_graphs(c);
    return AGAL_OK;
}

extern "C" int agal_bins_get(agal_ctx *c, int level, int *density, int *n_bins, long long *n_entries, int *n,
                             int *N, int *ids)
{
    if (!c) return AGAL_ERR_PARAM;
    const agal_bins_d *b = (level < 0) ? &c->bins_md : (level < c->n_bin_levels ? &c->bins[level] : nullptr);
    if (!b || !b->n) return agal_set_err(c, AGAL_ERR_PARAM, "no such bin level");
    if (density) *density = b->density;
    if (n_bins) *n_bins = b->n_bins;
    if (n_entries) *n_entries = b->n_entries;
    if (n) AGAL_CUDA(c, cudaMemcpy(n, b->n, sizeof(int) * b->n_bins, cudaMemcpyDeviceToHost));
    if (N) AGAL_CUDA(c, cudaMemcpy(N, b->N, sizeof(int) * b->n_bins, cudaMemcpyDeviceToHost));
    if (ids && b->n_entries) AGAL_CUDA(c, cudaMemcpy(ids, b->ids, sizeof(int) * b->n_entries, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

extern "C" int agal_voxelize_s1(agal_ctx *c, int L)
{
    // Mesh::M_Geometry_Voxelize_S1 (mesh_voxelizer.cu:34-156).
    if (!geo_ready(c) || L < 0 || L >= c->max_levels) return c ? agal_set_err(c, AGAL_ERR_PARAM, "voxelize_s1") : AGAL_ERR_PARAM;
    const int n = c->n_ids[L];
    if (n <= 0) return AGAL_OK;
    const float dxL = geo_dx(c, L);
    const float R = (float)((double)(float)c->P.G_NEAR_WALL_DISTANCE / std::pow(2.0, (double)(float)L));
    const int n_prop = (int)(R / (float)(4.0 * std::sqrt(2.0) * (double)dxL)) + 1;
    const int hit_max = (L == c->max_levels - 1);
    const int Lbin = std::min(L, c->n_bin_levels - 1);
    const long long nmb = c->nmb;
    const int *ids = c->id_set + (long long)L * nmb;
    const int idm = c->id_max[L];
    k_voxelize<<<n, MC3, 0, c->stream>>>(ids, nmb, dxL, c->faces, c->n_faces, view(c->bins[Lbin]), c->cblock_f_X,
                                         c->cells_ID_mask);
    k_propagate<<<(n + 7) / 8, 256, 0, c->stream>>>(ids, n, nmb, c->cblock_ID_nbr, c->cells_ID_mask, +1, L == c->L0);
    if (L > c->L0)
        k_propagate<<<(n + 7) / 8, 256, 0, c->stream>>>(ids, n, nmb, c->cblock_ID_nbr, c->cells_ID_mask, -1, 0);
    k_solid_blocks<<<grid_for(n), 256, 0, c->stream>>>(ids, n, c->cells_ID_mask, c->cblock_ID_mask);
    if (idm > 0) {
        k_mark_boundary<<<grid_for(idm), 256, 0, c->stream>>>(idm, nmb, L, hit_max, c->cblock_ID_ref,
                                                              c->cblock_ID_mask, c->cblock_ID_nbr, c->cblock_level);
        k_mark_exterior<<<grid_for(idm), 256, 0, c->stream>>>(idm, nmb, L, hit_max, c->cblock_ID_ref,
                                                              c->cblock_ID_mask, c->cblock_ID_nbr, c->cblock_level);
        for (int j = 0; j < n_prop; j++)
            k_mark_propagate<<<grid_for(idm), 256, 0, c->stream>>>(idm, nmb, L, j, c->cblock_ID_ref, c->cblock_ID_mask,
                                                                   c->cblock_ID_nbr, c->cblock_level, c->vox_tmp);
        k_mark_finalize<<<grid_for(idm), 256, 0, c->stream>>>(idm, c->cblock_ID_ref, c->vox_tmp);
    }
    AGAL_CUDA(c, cudaGetLastError());
    agal_drop_graphs(c);
    return agal_build_meta(c);
}

extern "C" int agal_update_solid_children(agal_ctx *c, int L)
{
    // Mesh::M_UpdateSolidChildren (mesh_voxelizer.cu:247-259).
    if (!geo_ready(c) || L < 0 || L >= c->max_levels) return c ? agal_set_err(c, AGAL_ERR_PARAM, "update_solid_children") : AGAL_ERR_PARAM;
    if (c->n_ids[L] <= 0 || c->id_max[L] <= 0) return AGAL_OK;
    k_solid_children<<<grid_for(c->id_max[L]), 256, 0, c->stream>>>(c->id_max[L], c->nmb, L, c->cblock_ID_mask,
                                                                    c->cblock_ID_nbr, c->cblock_ID_nbr_child,
                                                                    c->cblock_level);
    AGAL_CUDA(c, cudaGetLastError());
    agal_drop_graphs(c);
    return agal_build_meta(c);
}

extern "C" int agal_voxelize_s2(agal_ctx *c, int L)
{
    // Mesh::M_Geometry_Voxelize_S2 (mesh_voxelizer.cu:158-189).
    if (!geo_ready(c) || L < 0 || L >= c->max_levels) return c ? agal_set_err(c, AGAL_ERR_PARAM, "voxelize_s2") : AGAL_ERR_PARAM;
    const int n = c->n_ids[L];
    if (n <= 0) return AGAL_OK;
    const int idm = c->id_max[c->max_levels];
    if (L == 0 && idm > 0) k_fill_range<<<grid_for(idm), 256, 0, c->stream>>>(c->vox_tmp, idm, 0);
    const int *ids = c->id_set + (long long)L * c->nmb;
    k_check_masks<<<n, MC3, 0, c->stream>>>(ids, c->nmb, c->cells_ID_mask, c->cblock_ID_mask, c->cblock_ID_nbr,
                                            c->cblock_ID_nbr_child, c->cblock_ID_onb, c->vox_tmp, c->bnd_bits);
    k_apply_masks<<<grid_for((long long)n * MC3), 256, 0, c->stream>>>(ids, n, c->cblock_ID_onb, c->bnd_bits,
                                                                       c->cells_ID_mask);
    AGAL_CUDA(c, cudaGetLastError());
    agal_drop_graphs(c);
    return agal_build_meta(c);
}

extern "C" int agal_voxelize_s3(agal_ctx *c)
{
    // Mesh::M_Geometry_Voxelize_S3 (mesh_voxelizer.cu:191-245): one slot per
    // block with boundary cells, in block-ID order; the link-length array
    // sized for the slot count rounded up to 128 blocks.
    if (!geo_ready(c)) return c ? agal_set_err(c, AGAL_ERR_PARAM, "voxelize_s3") : AGAL_ERR_PARAM;
    const int idm = c->id_max[c->max_levels];
    AGAL_CUDA(c, cudaMemsetAsync(c->geo_small, 0, 16, c->stream));
    if (idm > 0)
        k_solid_counts<<<grid_for(idm), 256, 0, c->stream>>>(c->vox_tmp, idm, (unsigned long long *)c->geo_small,
                                                             c->geo_small + 2);
    long long host[2] = {0, 0};
    AGAL_CUDA(c, cudaMemcpyAsync(host, c->geo_small, 16, cudaMemcpyDeviceToHost, c->stream));
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    c->n_solida = host[0];
    const int sb = (int)(host[1] & 0xffffffff);
    c->n_solidb = ((sb + 128) / 128) * 128;
    c->n_maxcells_b = (long long)c->n_solidb * MC3;
    k_fill_range<<<grid_for(c->nmb), 256, 0, c->stream>>>(c->onb_solid, (int)c->nmb, -1);
    if (idm > 0) AGAL_CUDA(c, cmp::compact_async(c->stream, c->geo_parts, c->geo_small + 4, WallSlots{c->vox_tmp, c->onb_solid}, idm));
    if (c->X_b) cudaFree(c->X_b);
    c->X_b = nullptr;
    if (c->P.G_BIN_MAKE_LINKS) {
        const long long nx = c->n_maxcells_b * 27;
        AGAL_CUDA(c, cudaMalloc(&c->X_b, sizeof(float) * nx));
        k_fill_float<<<grid_for(nx), 256, 0, c->stream>>>(c->X_b, nx, -1.0f);
    }
    if (idm > 0) k_fill_range<<<grid_for(idm), 256, 0, c->stream>>>(c->vox_tmp, idm, -1);
    AGAL_CUDA(c, cudaGetLastError());
    agal_drop_graphs(c);
    return agal_build_meta(c);
}

extern "C" int agal_link_lengths(agal_ctx *c, int L)
{
    // Mesh::M_LinkLengthComputation (mesh_voxelizer.cu:261-294).
    if (!geo_ready(c) || L < 0 || L >= c->max_levels) return c ? agal_set_err(c, AGAL_ERR_PARAM, "link_lengths") : AGAL_ERR_PARAM;
    const int n = c->n_ids[L];
    if (!(c->n_solidb > 0 && n > 0 && c->P.G_BIN_MAKE_LINKS && c->X_b && c->bins_md.n)) return AGAL_OK;
    const int *ids = c->id_set + (long long)L * c->nmb;
    k_links<<<n, MC3, 0, c->stream>>>(ids, c->nmb, geo_dx(c, L), c->faces, c->n_faces, view(c->bins_md), c->cblock_f_X,
                                      c->cells_ID_mask, c->onb_solid, c->n_maxcells_b, c->X_b);
    k_links_validate<<<n, MC3, 0, c->stream>>>(ids, c->nmb, c->cblock_ID_nbr, c->cells_ID_mask, c->onb_solid,
                                               c->n_maxcells_b, c->X_b);
    AGAL_CUDA(c, cudaGetLastError());
    // the step's wall flags depend on the link lengths
    return agal_build_meta(c);
}

extern "C" int agal_geometry_counts(const agal_ctx *c, long long *out)
{
    if (!c || !out) return AGAL_ERR_PARAM;
    out[0] = c->n_faces;
    out[1] = c->n_solida;
    out[2] = c->n_solidb;
    out[3] = c->n_maxcells_b;
    return AGAL_OK;
}
