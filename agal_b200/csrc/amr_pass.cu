// The refine/coarsen pass (Mesh::M_RefineAndCoarsenBlocks, mesh_amr.cu:2162-2744)
// and the near-wall marking of M_Advance_RefineNearWall, on the device.
//
// Every stage of the reference pass is one or a few kernels over the block-ID
// range [0, id_max) in the same order, so the block arrays come out
// identical (block IDs, neighbour lists, masks, ID sets, gap stack):
//   marks        count MARK_REFINE / MARK_COARSEN; refinement that would
//                exhaust the gap stack is cancelled (:2197-2205)
//   S1           efficient map: marked blocks and their neighbours (:2225-2307)
//   S2           first-child IDs popped from the end of the gap stack, in
//                block-ID order of the marked blocks (ordered compaction);
//                neighbours learn their new children (Cu_RefineCells_S2_1)
//   S3           2:1 quality control of coarsening (Cu_RefineCells_Q1_1/_2,
//                Cu_RefineCells_S2_2)
//   S4           new children written / children of coarsened blocks marked
//                for removal (Cu_AddRemoveBlocks)
//   S5           removed children leave their level's ID set (stable
//                compaction; the tail keeps its old values like remove_if) and
//                return to the gap stack in (level, ID) order, reversed
//   S6           new children join their level's ID set, which stays sorted
//   S7           id_max per level (an empty level reads its first slot)
//   S8           interface masks, interpolation into new children, reference
//                state transitions, WCHILD update from a snapshot,
//                connectivity of new children from their parents' child table,
//                boundary flags and cell masks.
// The host reads back only counts (marks, gaps, per-level sizes and id_max),
// as the reference does to size its launches.
//
// Compaction: each CTA takes a contiguous chunk of SCAN_T x SCAN_I indices,
// counts its flagged ones, the per-CTA counts are scanned in one CTA, and a
// second pass emits every flagged index with its rank, warp-shuffle scans
// keeping index order.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <cstdio>
#include <string>
#include <vector>

#include "ctx.h"
#include "compact.cuh"
#include "lattice.cuh"

namespace agal {
namespace {

using cmp::SCAN_CHUNK;
constexpr int NT = 256;   // threads per CTA of the per-block kernels

// Small device counters (amr_small, AGAL_AMR_SMALL ints).
// S_KEEP / S_MERGE: the sizes of the S5 / S6 compactions per level, checked
// on the host with the S7 readback (one wait instead of one per level).
// S_NEW / S_REM: new and removed blocks per level, read back together after
// S4.
enum {
    S_NR = 0, S_NC = 1, S_GMAX = 2, S_TOTAL = 3, S_NEW = 8, S_IDMAX = 32, S_NIDS = 64, S_KEEP = 96, S_MERGE = 128,
    S_REM = 160
};
static_assert(S_REM + 17 <= AGAL_AMR_SMALL, "small counter layout");

unsigned grid_for(long long n, int per = NT) { return (unsigned)((n + per - 1) / per); }

// Ordered compaction over [0, n): f.emit(i, rank) for every i with f.pred(i).
// The predicate must not read what emit writes.  *count receives the count.
template <class F>
int compact(agal_ctx *c, const F &f, int n, int *count)
{
    *count = 0;
    if (n <= 0) return AGAL_OK;
    AGAL_CUDA(c, cmp::compact_async(c->stream, c->amr_parts, c->amr_small + S_TOTAL, f, n));
    int *h = c->h_small ? c->h_small : count;   // pinned: a direct copy
    AGAL_CUDA(c, cudaMemcpyAsync(h, c->amr_small + S_TOTAL, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    *count = *h;
    return AGAL_OK;
}

// The same without reading the count back (a compaction whose count the host
// does not need).
template <class F>
int compact_nowait(agal_ctx *c, const F &f, int n)
{
    if (n <= 0) return AGAL_OK;
    AGAL_CUDA(c, cmp::compact_async(c->stream, c->amr_parts, c->amr_small + S_TOTAL, f, n));
    return AGAL_OK;
}

// ---- compaction functors --------------------------------------------------
struct FirstChild {   // S2: the i-th marked block takes gap_set[n_gaps - 1 - NCH i]
    const int *ref, *gaps;
    int *first;
    int top, nch;
    __device__ bool pred(int b) const { return ref[b] == REF_MARK_REFINE; }
    __device__ void emit(int b, int r) const { first[b] = gaps[top - 1 - nch * r]; }
};
struct RemovedAtLevel {   // S5: blocks leaving level L, in ID order
    const int *ref, *level;
    int L;
    int *out;
    __device__ bool pred(int b) const { return ref[b] == REF_REMOVE && level[b] == L; }
    __device__ void emit(int b, int r) const { out[r] = b; }
};
struct KeepIds {   // S5: ID-set entries not marked N_SKIPID
    const int *ids;
    int *out;
    __device__ bool pred(int k) const { return ids[k] != N_SKIPID; }
    __device__ void emit(int k, int r) const { out[r] = ids[k]; }
};
struct MergeLevel {   // S6: old members and new children of level L, sorted
    const int *member, *ref, *level;
    int L;
    int *ids;
    __device__ bool pred(int b) const { return member[b] || (ref[b] == REF_NEW && level[b] == L); }
    __device__ void emit(int b, int r) const { ids[r] = b; }
};

// ---- per-block kernels ----------------------------------------------------
// Kernels that use warp reductions take no early return before them.
__device__ __forceinline__ void warp_add(int *dst, int v)
{
    const int s = __reduce_add_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(dst, s);
}

__global__ void k_count_marks(const int *ref, int n, int *out)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = (b < n) ? ref[b] : -1;
    warp_add(out + S_NR, r == REF_MARK_REFINE);
    warp_add(out + S_NC, r == REF_MARK_COARSEN);
}

__global__ void k_unmark_refine(int *ref, int n)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < n && ref[b] == REF_MARK_REFINE) ref[b] = REF_UNREFINED;
}

__global__ void k_emap(const int *ref, const int *nbr, long long nmb, int qmax, int n, int *emap)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int r = ref[b];
    if (r != REF_MARK_REFINE && r != REF_MARK_COARSEN) return;
    for (int p = 0; p < qmax; p++) {
        const int nb = nbr[b + p * nmb];
        if (nb >= 0) emap[nb] = nb;
    }
}

__global__ void k_max_range(const int *a, int lo, int hi, int *out)
{
    const int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    const int v = (i < hi) ? a[i] : INT_MIN;
    const int m = __reduce_max_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_s2_1(const int *emap, const int *nbr, const int *ref, const int *first, long long nmb, int qmax,
                       int n, int *nch)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || emap[b] < 0) return;
    for (int d = 0; d < qmax; d++) {
        const int nb = nbr[b + d * nmb];
        if (nb > -1 && ref[nb] == REF_MARK_REFINE) nch[b + d * nmb] = first[nb];
    }
}

__global__ void k_q1_1(const int *nch, long long nmb, int qmax, int n, int *ref)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || ref[b] != REF_UNREFINED) return;
    for (int p = 1; p < qmax; p++)
        if (nch[b + p * nmb] >= 0) {
            ref[b] = REF_UNREFINED_VIO;
            return;
        }
}

// A block marked for coarsening has only leaf children, which are never
// marked for coarsening themselves: no thread reads a state another writes.
__global__ void k_q1_2(const int *nch, int nchild, int n, int *ref)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || ref[b] != REF_MARK_COARSEN) return;
    const int ic = nch[b];
    if (ic < 0) return;
    bool vio = false;
    for (int x = 0; x < nchild; x++) {
        const int r = ref[ic + x];
        if (r == REF_UNREFINED_VIO || r == REF_MARK_REFINE) vio = true;
    }
    if (vio) ref[b] = REF_REFINED;
}

__global__ void k_s2_2(const int *emap, const int *nbr, const int *ref, long long nmb, int qmax, int n, int *nch)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || emap[b] < 0) return;
    for (int d = 1; d < qmax; d++) {
        const int nb = nbr[b + d * nmb];
        if (nb > -1 && ref[nb] == REF_MARK_COARSEN) nch[b + d * nmb] = N_SKIPID;
    }
}

// Cu_AddRemoveBlocks (mesh_amr.cu:1495).  A thread reads only its own mark;
// new children are former gaps and children of coarsened blocks are leaves,
// so no thread acts on a state another thread writes.
__global__ void k_add_remove(const int *first, long long nmb, int dim, int nchild, float dx_cblock, int n, int *ref,
                             int *nch, int *level, float *fX)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int r = ref[b];
    if (r == REF_MARK_REFINE) {
        const int f = first[b];
        if (f < 0) return;
        nch[b] = f;
        const int lev = level[b] + 1;
        const float h = __fdiv_rn(dx_cblock, (float)(1 << lev));
        for (int x = 0; x < nchild; x++) {
            const int ch = f + x;
            level[ch] = lev;
            ref[ch] = REF_NEW;
            fX[ch] = __fadd_rn(fX[b], __fmul_rn((float)(x & 1), h));
            fX[ch + nmb] = __fadd_rn(fX[b + nmb], __fmul_rn((float)((x >> 1) & 1), h));
            if (dim == 3) fX[ch + 2 * nmb] = __fadd_rn(fX[b + 2 * nmb], __fmul_rn((float)((x >> 2) & 1), h));
            nch[ch] = N_SKIPID;
        }
    } else if (r == REF_MARK_COARSEN) {
        const int f = nch[b];
        if (f < 0) return;
        nch[b] = N_SKIPID;
        for (int x = 0; x < nchild; x++) ref[f + x] = REF_REMOVE;
    }
}

__global__ void k_mark_removed_ids(int *ids, int n, const int *ref)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && ref[ids[k]] == REF_REMOVE) ids[k] = N_SKIPID;
}


__global__ void k_fill_int(int *dst, int n, int v)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = v;
}

// small[slot] = small[S_TOTAL]: keeps a compaction's size past the next one.
__global__ void k_keep_total(int *small, int slot) { small[slot] = small[S_TOTAL]; }

// dst[k] = src[k] for k < *count (count on the device, n an upper bound).
__global__ void k_copy_counted(const int *src, int *dst, const int *count, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && k < *count) dst[k] = src[k];
}

struct Ints17 {
    int v[17];
};
__global__ void k_set_ints(int *dst, Ints17 a)
{
    if (threadIdx.x < 17) dst[threadIdx.x] = a.v[threadIdx.x];
}

// Cu_ConcatReverse (mesh_amr.cu:40): removed IDs onto the gap stack, reversed.
__global__ void k_concat_reverse(int *gaps, int base, const int *rem, int cnt)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < cnt) gaps[base + k] = rem[cnt - 1 - k];
}

__global__ void k_coarsen_s2(const int *ref, long long nmb, int qmax, int n, int *nbr, int *nch)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || ref[b] != REF_REMOVE) return;
    for (int p = 0; p < qmax; p++) {
        if (p > 0) nbr[b + p * nmb] = N_SKIPID;
        nch[b + p * nmb] = N_SKIPID;
    }
}

// Blocks in refinement state `state` per level (new children, removed ones).
__global__ void k_count_state(const int *ref, const int *level, int n, int state, int *cnt)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < n && ref[b] == state) atomicAdd(&cnt[level[b]], 1);
}

__global__ void k_scatter_member(const int *ids, int n, int *member)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) member[ids[k]] = 1;
}

// S7: max ID per level 1..ML-1 (grid.y = level - 1); an empty level reads its
// first slot as thrust::max_element's end iterator does (mesh_amr.cu:2630).
__global__ void k_level_max(const int *id_set, long long nmb, const int *n_ids, int *out)
{
    const int L = blockIdx.y + 1;
    const int n = n_ids[L];
    const int *ids = id_set + (long long)L * nmb;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    int v = INT_MIN;
    if (n == 0) {
        if (k == 0) v = ids[0];
    } else if (k < n) {
        v = ids[k];
    }
    const int m = __reduce_max_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && m != INT_MIN) atomicMax(&out[L], m);
}

// Cu_UpdateMasks_1 (mesh_amr.cu:948): refined blocks with a coarse-side
// neighbour are interface blocks.
__global__ void k_masks_1(const int *ref, const int *nch, long long nmb, int qmax, int n, int *bmask)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n || ref[b] == REF_INACTIVE) return;
    int m = BLOCK_REGULAR;
    if (nch[b] > -1)
        for (int p = 1; p < qmax; p++)
            if (nch[b + p * nmb] == N_SKIPID) m = BLOCK_INTERFACE;
    if (bmask[b] > -1) bmask[b] = m;
}

// Cu_RefineCells_S3 (mesh_amr.cu:1731).
__global__ void k_s3(int *ref, int n)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int r = ref[b];
    if (r == REF_MARK_REFINE) ref[b] = REF_REFINED;
    if (r == REF_NEW || r == REF_MARK_COARSEN) ref[b] = REF_UNREFINED;
    if (r == REF_REMOVE) ref[b] = REF_INACTIVE;
    if (r == REF_UNREFINED_VIO) ref[b] = REF_UNREFINED;
}

// Cu_RefineCells_S4 (mesh_amr.cu:1774): a refined block with a refined
// child is REFINED_WCHILD; children's states read from the snapshot.
__global__ void k_s4(const int *snap, const int *nch, int nchild, int n, int *ref)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int s = snap[b];
    if (s != REF_REFINED && s != REF_REFINED_WCHILD) return;
    const int ic = nch[b];
    if (ic < 0) return;
    int nr = REF_REFINED;
    for (int x = 0; x < nchild; x++) {
        const int r = (ic + x < n) ? snap[ic + x] : ref[ic + x];
        if (r == REF_REFINED || r == REF_REFINED_WCHILD) nr = REF_REFINED_WCHILD;
    }
    ref[b] = nr;
}

// Index of the direction with velocity (ex, ey, ez) in the neighbour table.
__device__ __forceinline__ int dir_of(int dim, int qmax, int ex, int ey, int ez)
{
    for (int q = 0; q < qmax; q++)
        if (lat_c(dim, 0, q) == ex && lat_c(dim, 1, q) == ey && lat_c(dim, 2, q) == ez) return q;
    return 0;
}

// Cu_UpdateConnectivity (mesh_amr.cu:156): the neighbour of child x of block
// b in direction d is a child (offset qi) of b's child-table entry in the
// parent direction that x + c_d falls into.  One thread per (block, child).
__global__ void k_connectivity(const int *emap, const int *nch, long long nmb, int dim, int qmax, int nchild, int n,
                               int *nbr)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)n * nchild) return;
    const int b = (int)(g / nchild), x = (int)(g % nchild);
    if (!(emap[b] > -1 && nch[b] > -1)) return;
    const int f = nch[b];
    for (int d = 0; d < qmax; d++) {
        const int tx = (x & 1) + lat_c(dim, 0, d), ty = ((x >> 1) & 1) + lat_c(dim, 1, d);
        const int tz = (dim == 3) ? ((x >> 2) & 1) + lat_c(dim, 2, d) : 0;
        const int px = tx >= 0 ? tx / 2 : -1, py = ty >= 0 ? ty / 2 : -1, pz = tz >= 0 ? tz / 2 : -1;
        const int qv = dir_of(dim, qmax, px, py, dim == 3 ? pz : 0);
        const int qi = (tx & 1) + 2 * (ty & 1) + (dim == 3 ? 4 * (tz & 1) : 0);
        const int v = nch[b + qv * nmb];
        nbr[(f + x) + d * nmb] = (v < 0) ? v : v + qi;
    }
}

// Cu_UpdateBoundaries (mesh_amr.cu:106).
__global__ void k_boundaries(const int *nbr, const int *bmask, long long nmb, int qmax, int n, int *nch, int *onb)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    int on = 0;
    for (int p = 1; p < qmax; p++) {
        const int v = nbr[b + p * nmb];
        if (v < 0) {
            nch[b + p * nmb] = v;
            if (v != N_SKIPID) on = 1;
        }
    }
    if (bmask[b] == BLOCK_SOLIDA) on = 1;
    onb[b] = on;
}

// Cu_UpdateMasks_2 (mesh_amr.cu:983): cells facing a coarser neighbour are
// ghost cells (2), the rest of such a block interface cells (1).
__global__ void k_masks_2(const int *ref, const int *nbr, long long nmb, int dim, int qmax, int mc, int n, int *cmask)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)n * mc) return;
    const int b = (int)(g / mc), t = (int)(g % mc);
    if (ref[b] == REF_INACTIVE) return;
    const long long o = (long long)b * mc + t;
    if (cmask[o] < 0) return;
    const int I = t & 3, J = (t >> 2) & 3, K = (dim == 3) ? (t >> 4) : 0;
    bool any = false, ghost = false;
    for (int p = 1; p < qmax; p++) {
        if (nbr[b + p * nmb] != N_SKIPID) continue;
        any = true;
        const int cx = lat_c(dim, 0, p), cy = lat_c(dim, 1, p), cz = lat_c(dim, 2, p);
        bool in = true;
        if (cx > 0 && !(I >= 2)) in = false;
        if (cx < 0 && !(I < 2)) in = false;
        if (cy > 0 && !(J >= 2)) in = false;
        if (cy < 0 && !(J < 2)) in = false;
        if (dim == 3 && cz > 0 && !(K >= 2)) in = false;
        if (dim == 3 && cz < 0 && !(K < 2)) in = false;
        if (in) ghost = true;
    }
    cmask[o] = ghost ? CELL_GHOST : (any ? CELL_INTERFACE : CELL_INTERIOR);
}

// Cu_ComputeRefCriteria_Uniform / _NearWall_Cases (mesh_criterion.cu:10-85)
// with the Cu_RefineRegion presets on the block bounds (x + 1e-5,
// x + 4 dx_L - 1e-5).
__global__ void k_mark_level(const int *ids, int n, long long nmb, int dim, int uniform, int region, float dxb,
                             const int *onb, const float *fX, int *ref)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int b = ids[k];
    if (ref[b] != REF_UNREFINED) return;
    bool mark = uniform != 0;
    if (!mark && region == AGAL_REGION_BOUNDARY) mark = onb[b] == 1;
    if (!mark && region == AGAL_REGION_BOX) {
        mark = true;
        for (int d = 0; d < dim; d++) {
            const float lo = __fadd_rn(fX[b + d * nmb], 1e-5f);
            const float hi = __fadd_rn(__fadd_rn(fX[b + d * nmb], dxb), -1e-5f);
            if (!(lo >= 0.25f && hi <= 0.75f)) mark = false;
        }
    }
    if (mark) ref[b] = REF_MARK_REFINE;
}

// Cu_FreezeRefined / Cu_UnfreezeRefined (mesh_amr.cu:1888-1923): refined
// blocks become permanent (thaw = 0) or eligible for coarsening again (1).
__global__ void k_freeze(int *ref, int n, int thaw)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const int r = ref[b];
    if (!thaw) {
        if (r == REF_REFINED) ref[b] = REF_REFINED_PERM;
        if (r == REF_REFINED_WCHILD) ref[b] = REF_REFINED_WCHILD_PERM;
    } else {
        if (r == REF_REFINED_PERM) ref[b] = REF_REFINED;
        if (r == REF_REFINED_WCHILD_PERM) ref[b] = REF_REFINED_WCHILD;
    }
}

int read_small(agal_ctx *c, int *h, int off, int n)
{
    int *dst = c->h_small ? c->h_small : h;   // pinned: a direct copy
    AGAL_CUDA(c, cudaMemcpyAsync(dst, c->amr_small + off, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (dst != h) std::memcpy(h, dst, sizeof(int) * n);
    return AGAL_OK;
}

}  // namespace
}  // namespace agal

using namespace agal;

size_t agal_amr_scratch_ints(int64_t nmb)
{
    return (size_t)5 * nmb + (size_t)(nmb / SCAN_CHUNK + 2) + AGAL_AMR_SMALL;
}

int agal_mark_level(agal_ctx *c, int L, int uniform)
{
    const int n = c->n_ids[L];
    if (n <= 0) return AGAL_OK;
    const float dxb = (float)c->dxf[L] * 4.0f;
    k_mark_level<<<grid_for(n), NT, 0, c->stream>>>(c->id_set + (long long)L * c->nmb, n, c->nmb, c->dim, uniform,
                                                    c->P.region_preset, dxb, c->cblock_ID_onb, c->cblock_f_X,
                                                    c->cblock_ID_ref);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

namespace agal {
namespace {
struct IfaceList {   // interface parents of one level, in ID-set order
    const int *ids, *bmask, *nch;
    int *out;
    __device__ bool pred(int k) const { const int b = ids[k]; return bmask[b] == BLOCK_INTERFACE && nch[b] > -1; }
    __device__ void emit(int k, int r) const { out[r] = ids[k]; }
};
}  // namespace
}  // namespace agal

int agal_build_iface_lists(agal_ctx *c)
{
    c->iface_off.assign(c->max_levels, 0);
    c->iface_n.assign(c->max_levels, 0);
    if (!c->amr) return AGAL_OK;
    if (!c->iface_ids) AGAL_CUDA(c, cudaMalloc(&c->iface_ids, sizeof(int) * c->nmb));
    int off = 0;
    for (int L = 0; L + 1 < c->max_levels; L++) {
        c->iface_off[L] = off;
        const int n = c->n_ids[L];
        if (n <= 0) continue;
        IfaceList f{c->id_set + (long long)L * c->nmb, c->cblock_ID_mask, c->cblock_ID_nbr_child, c->iface_ids + off};
        int cnt = 0;
        int rc = compact(c, f, n, &cnt);
        if (rc) return rc;
        c->iface_n[L] = cnt;
        off += cnt;
    }
    return AGAL_OK;
}

int agal_freeze_refined(agal_ctx *c, int thaw)
{
    const int n = c->id_max[c->max_levels];
    if (n <= 0) return AGAL_OK;
    k_freeze<<<grid_for(n), NT, 0, c->stream>>>(c->cblock_ID_ref, n, thaw);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

int agal_refine_pass(agal_ctx *c)
{
    if (!c->amr) return agal_set_err(c, AGAL_ERR_STATE, "refinement needs MAX_LEVELS > 1");
    const int ML = c->max_levels, NCH = c->NCH, Qmax = c->Qmax;
    const long long nmb = c->nmb;
    int *ref = c->cblock_ID_ref, *nbr = c->cblock_ID_nbr, *nch = c->cblock_ID_nbr_child;
    const int idm = c->id_max[ML];
    int rc, h[AGAL_AMR_SMALL];

    AGAL_CUDA(c, cudaMemsetAsync(c->amr_small, 0, sizeof(int) * AGAL_AMR_SMALL, c->stream));
    if (idm > 0) k_count_marks<<<grid_for(idm), NT, 0, c->stream>>>(ref, idm, c->amr_small);
    AGAL_CUDA(c, cudaGetLastError());
    if ((rc = read_small(c, h, 0, 2))) return rc;
    int nR = h[S_NR], nC = h[S_NC];
    // Bound of the IDs a pass can touch (mesh_amr.cu:2186 and :2341).  The
    // reference's sum can pass n_maxcblocks when the pool is nearly full,
    // although every ID lies below it; the passes stop at n_maxcblocks.
    int idm_wnew = (int)std::min<long long>((long long)idm + (long long)NCH * nR, nmb);
    const bool proceed_ref = nR > 0 && (long long)NCH * nR <= c->n_gaps;
    bool proceed_coarse = nC > 0;
    if (!proceed_ref && nR > 0) {   // mesh_amr.cu:2197-2205
        nR = 0;
        idm_wnew = idm;
        k_unmark_refine<<<grid_for(idm), NT, 0, c->stream>>>(ref, idm);
    }
    // S1: efficient map.
    if (proceed_ref || proceed_coarse)
        k_emap<<<grid_for(idm), NT, 0, c->stream>>>(ref, nbr, nmb, Qmax, idm, c->amr_emap);
    // S2: first children from the top of the gap stack.
    if (proceed_ref) {
        FirstChild fc{ref, c->gap_set, c->amr_first, c->n_gaps, NCH};
        if ((rc = compact_nowait(c, fc, idm))) return rc;   // its count is nR
        const int lo = c->n_gaps - NCH * nR, hi = c->n_gaps;
        k_fill_int<<<1, 1, 0, c->stream>>>(c->amr_small + S_GMAX, 1, INT_MIN);
        k_max_range<<<grid_for(hi - lo), NT, 0, c->stream>>>(c->gap_set, lo, hi, c->amr_small + S_GMAX);
        k_s2_1<<<grid_for(idm), NT, 0, c->stream>>>(c->amr_emap, nbr, ref, c->amr_first, nmb, Qmax, idm, nch);
    }
    // S3: 2:1 quality control of coarsening.  The largest new child ID (S2)
    // is read back with the recount of the marks (one wait for both).
    if (proceed_coarse) {
        k_q1_1<<<grid_for(idm), NT, 0, c->stream>>>(nch, nmb, Qmax, idm, ref);
        k_q1_2<<<grid_for(idm), NT, 0, c->stream>>>(nch, NCH, idm, ref);
        AGAL_CUDA(c, cudaMemsetAsync(c->amr_small, 0, sizeof(int) * 2, c->stream));
        k_count_marks<<<grid_for(idm), NT, 0, c->stream>>>(ref, idm, c->amr_small);
        if ((rc = read_small(c, h, 0, 3))) return rc;   // S_NR, S_NC, S_GMAX
        nC = h[S_NC];
        proceed_coarse = nC > 0;
        if (proceed_coarse) k_s2_2<<<grid_for(idm), NT, 0, c->stream>>>(c->amr_emap, nbr, ref, nmb, Qmax, idm, nch);
    } else if (proceed_ref) {
        if ((rc = read_small(c, h, S_GMAX, 1))) return rc;
        h[S_GMAX] = h[0];
    }
    if (proceed_ref && h[S_GMAX] + 1 > idm_wnew) idm_wnew = (int)std::min<long long>(h[S_GMAX] + 1, nmb);
    AGAL_CUDA(c, cudaGetLastError());
    if (!(proceed_ref || proceed_coarse)) {
        c->n_ref_last = 0;
        c->n_coarse_last = 0;
        return AGAL_OK;
    }
    // S4: add and remove blocks.
    k_add_remove<<<grid_for(idm), NT, 0, c->stream>>>(c->amr_first, nmb, c->dim, NCH, c->dx_cblock, idm, ref, nch,
                                                      c->cblock_level, c->cblock_f_X);
    AGAL_CUDA(c, cudaGetLastError());
    // The blocks leaving (S5) and joining (S6) each level, read back at once.
    int n_new[17], n_rem[17];
    for (int L = 0; L < 17; L++) n_new[L] = n_rem[L] = 0;
    if (proceed_coarse) {
        AGAL_CUDA(c, cudaMemsetAsync(c->amr_small + S_REM, 0, sizeof(int) * 17, c->stream));
        k_count_state<<<grid_for(idm_wnew), NT, 0, c->stream>>>(ref, c->cblock_level, idm_wnew, REF_REMOVE,
                                                                 c->amr_small + S_REM);
    }
    if (proceed_ref) {
        AGAL_CUDA(c, cudaMemsetAsync(c->amr_small + S_NEW, 0, sizeof(int) * 17, c->stream));
        k_count_state<<<grid_for(idm_wnew), NT, 0, c->stream>>>(ref, c->cblock_level, idm_wnew, REF_NEW,
                                                                 c->amr_small + S_NEW);
    }
    AGAL_CUDA(c, cudaGetLastError());
    if ((rc = read_small(c, h, S_NEW, S_REM + 17 - S_NEW))) return rc;
    for (int L = 0; L < 17; L++) {
        if (proceed_ref) n_new[L] = h[L];
        if (proceed_coarse) n_rem[L] = h[S_REM - S_NEW + L];
    }
    // S5: removed children leave the ID sets and return to the gap stack.
    int expect_keep[17], expect_merge[17];
    for (int L = 0; L < 17; L++) expect_keep[L] = expect_merge[L] = -1;
    if (proceed_coarse) {
        int prev = 0;
        for (int L = 1; L < ML; L++) {
            const int cnt = n_rem[L];
            if (cnt == 0) continue;
            RemovedAtLevel rl{ref, c->cblock_level, L, c->amr_b + prev};
            if ((rc = compact_nowait(c, rl, idm_wnew))) return rc;   // cnt blocks, counted above
            int *ids = c->id_set + (long long)L * nmb;
            const int n = c->n_ids[L];
            k_mark_removed_ids<<<grid_for(n), NT, 0, c->stream>>>(ids, n, ref);
            KeepIds ki{ids, c->amr_a};
            if ((rc = compact_nowait(c, ki, n))) return rc;   // n - cnt kept, checked at S7
            k_keep_total<<<1, 1, 0, c->stream>>>(c->amr_small, S_KEEP + L);
            k_copy_counted<<<grid_for(n), NT, 0, c->stream>>>(c->amr_a, ids, c->amr_small + S_KEEP + L, n);
            expect_keep[L] = n - cnt;
            c->n_ids[L] -= cnt;
            prev += cnt;
        }
        if (prev > 0)
            k_concat_reverse<<<grid_for(prev), NT, 0, c->stream>>>(c->gap_set, c->n_gaps - NCH * nR, c->amr_b, prev);
        c->n_gaps += prev;
        k_coarsen_s2<<<grid_for(idm), NT, 0, c->stream>>>(ref, nmb, Qmax, idm, nbr, nch);
        AGAL_CUDA(c, cudaGetLastError());
    }
    // S6: new children join the ID sets.
    if (proceed_ref) {
        for (int L = 1; L < ML; L++) {
            const int cnt = n_new[L];
            if (cnt == 0) continue;
            int *ids = c->id_set + (long long)L * nmb;
            const int n = c->n_ids[L];
            k_fill_int<<<grid_for(idm_wnew), NT, 0, c->stream>>>(c->amr_a, idm_wnew, 0);
            if (n > 0) k_scatter_member<<<grid_for(n), NT, 0, c->stream>>>(ids, n, c->amr_a);
            MergeLevel ml{c->amr_a, ref, c->cblock_level, L, ids};
            if ((rc = compact_nowait(c, ml, idm_wnew))) return rc;   // checked at S7
            k_keep_total<<<1, 1, 0, c->stream>>>(c->amr_small, S_MERGE + L);
            c->n_ids[L] += cnt;
            expect_merge[L] = c->n_ids[L];
        }
        c->n_gaps -= NCH * nR;
    }
    // S7: id_max per level.
    {
        Ints17 init, nn;
        for (int L = 0; L < 17; L++) {
            init.v[L] = INT_MIN;
            nn.v[L] = L < ML ? c->n_ids[L] : 0;
        }
        k_set_ints<<<1, 32, 0, c->stream>>>(c->amr_small + S_IDMAX, init);
        k_set_ints<<<1, 32, 0, c->stream>>>(c->amr_small + S_NIDS, nn);
        int nmax = 1;
        for (int L = 1; L < ML; L++) nmax = std::max(nmax, c->n_ids[L]);
        dim3 g(grid_for(nmax), ML - 1);
        k_level_max<<<g, NT, 0, c->stream>>>(c->id_set, nmb, c->amr_small + S_NIDS, c->amr_small + S_IDMAX);
        AGAL_CUDA(c, cudaGetLastError());
        // id_max and the S5 / S6 compaction sizes in one readback
        if ((rc = read_small(c, h, S_IDMAX, S_MERGE + 17 - S_IDMAX))) return rc;
        for (int L = 1; L < ML; L++) {
            if (expect_keep[L] >= 0 && h[S_KEEP - S_IDMAX + L] != expect_keep[L])
                return agal_set_err(c, AGAL_ERR_STATE, "ID set removal size mismatch");
            if (expect_merge[L] >= 0 && h[S_MERGE - S_IDMAX + L] != expect_merge[L])
                return agal_set_err(c, AGAL_ERR_STATE, "ID set merge size mismatch");
        }
        for (int L = 1; L < ML; L++) c->id_max[L] = h[L] + 1;
        int mx = c->id_max[0];
        for (int L = 1; L < ML; L++) mx = std::max(mx, c->id_max[L]);
        c->id_max[ML] = mx;
    }
    const int idmN = c->id_max[ML];
    k_masks_1<<<grid_for(idmN), NT, 0, c->stream>>>(ref, nch, nmb, Qmax, idmN, c->cblock_ID_mask);
    AGAL_CUDA(c, cudaGetLastError());
    for (int L = 0; L < ML - 1; L++)
        if ((rc = agal_les_refresh(c, L)) || (rc = agal_launch_interp(c, L, AGAL_INTERP_ADDED))) return rc;
    k_s3<<<grid_for(idm_wnew), NT, 0, c->stream>>>(ref, idm_wnew);
    AGAL_CUDA(c, cudaMemcpyAsync(c->amr_snap, ref, sizeof(int) * (size_t)idm_wnew, cudaMemcpyDeviceToDevice,
                                 c->stream));
    k_s4<<<grid_for(idm_wnew), NT, 0, c->stream>>>(c->amr_snap, nch, NCH, idm_wnew, ref);
    // S8: connectivity, boundaries, cell masks.
    k_connectivity<<<grid_for((long long)idmN * NCH), NT, 0, c->stream>>>(c->amr_emap, nch, nmb, c->dim, Qmax, NCH,
                                                                          idmN, nbr);
    k_boundaries<<<grid_for(idmN), NT, 0, c->stream>>>(nbr, c->cblock_ID_mask, nmb, Qmax, idmN, nch,
                                                       c->cblock_ID_onb);
    k_masks_2<<<grid_for((long long)idmN * c->MC), NT, 0, c->stream>>>(ref, nbr, nmb, c->dim, Qmax, c->MC, idmN,
                                                                        c->cells_ID_mask);
    k_fill_int<<<grid_for(idmN), NT, 0, c->stream>>>(c->amr_emap, idmN, -1);
    const int nf = (int)std::min<long long>(idm_wnew, nmb);
    k_fill_int<<<grid_for(nf), NT, 0, c->stream>>>(c->amr_first, nf, -1);
    AGAL_CUDA(c, cudaGetLastError());
    c->n_ref_last = nR;
    c->n_coarse_last = proceed_coarse ? nC : 0;
    return agal_build_meta(c);
}
