// Row-mapped form of the fused collide + boundary + stream step (variant 4).
//
// One thread owns one x-row of a cell-block: the four cells (I = 0..3, J, K)
// whose populations sit next to each other in every slot of the block-major
// layout F[b][s][c] (c = I + 4 J + 16 K).  So each slot of the row is ONE
// vector load (16 bytes in FP32, 8 bytes in FP16/BF16) instead of four scalar
// loads, and a warp's load of one slot covers whole 32-byte sectors of its
// blocks.  After the collision the row's post-collision values of direction p
// land, for c_x = 0, in one row of one destination block (same row shifted by
// (c_y, c_z), possibly in the y/z neighbour block): one vector store.  For
// c_x = +-1 three of the four cells shift inside the destination row (one
// aligned pair store and one scalar store) and the fourth crosses into the x
// neighbour of that block (one scalar store).  Versus one thread per cell this
// cuts the load/store instructions per cell by ~4x and ~2x, and the neighbour
// lookups and address arithmetic by ~4x (shared by the row).
//
// The arithmetic per cell is the shared collide_cell of step_common.cuh, so
// the populations are bit-identical to the other variants.  Closed links
// (missing neighbour block) bounce back into the cell's own slot p; on blocks
// with the boundary hook the bounced value is passed through bc_hook right
// after the collision (it needs the cell's velocity), exactly where push_cell
// applies it.  Blocks next to solid cells (geometry cases) take push_cell per
// cell (the per-cell solid-neighbour test), as do LES and FP64 contexts (run
// by variant 1 instead).  The reference's stream guard (f_pb > 0,
// solver_lbm_kernels.cu:620-628): a row with any non-positive post-collision
// value of a non-owning direction recomputes its cells' collisions from the
// input (bit for bit the same values) and records the refused links as
// push_cell does; k_stream_fixup / fused_fixup swaps them back.
#include <cuda_runtime.h>

#include <type_traits>

#include "ctx.h"
#include "lattice.cuh"
#include "step_common.cuh"
#include "storage.cuh"

namespace agal {
namespace {

// One slot of a row: four consecutive cells.
template <typename T> struct Row4;
template <> struct Row4<float> {
    using V = float4;
    __device__ static V load(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
    __device__ static void store(float *p, const V &v) { *reinterpret_cast<float4 *>(p) = v; }
    __device__ static float get(const V &v, int k) { return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w; }
    __device__ static void set2(V &v, int k, float a, float b)   // cells k, k + 1 (k even)
    {
        if (k == 0) { v.x = a; v.y = b; }
        else { v.z = a; v.w = b; }
    }
    // elements k, k + 1 of the row as one aligned pair for a pair store
    using P = float2;
    __device__ static P pair(const V &v, int k)
    {
        return k == 0 ? make_float2(v.x, v.y) : k == 1 ? make_float2(v.y, v.z) : make_float2(v.z, v.w);
    }
    __device__ static void store_pair(float *p, const P &x) { *reinterpret_cast<float2 *>(p) = x; }
    __device__ static void store_one(float *p, const V &v, int k) { *p = get(v, k); }
    // Warp exchange of a row's edge cell: cell 3 (for the right neighbour's
    // x-shift by +1) and cell 0 (for the left neighbour's shift by -1).
    using E = float;
    __device__ static E last(const V &v) { return v.w; }
    __device__ static E first(const V &v) { return v.x; }
    __device__ static V shift_in_left(const V &v, E l) { return make_float4(l, v.x, v.y, v.z); }
    __device__ static V shift_in_right(const V &v, E r) { return make_float4(v.y, v.z, v.w, r); }
};

// Half-precision rows (weight offsets): four 16-bit values in a uint2.
template <typename T> struct Row4Half {
    using V = uint2;
    __device__ static V load(const T *p) { return __ldg(reinterpret_cast<const uint2 *>(p)); }
    __device__ static void store(T *p, const V &v) { *reinterpret_cast<uint2 *>(p) = v; }
    __device__ static unsigned short bits(const V &v, int k)
    {
        const unsigned w = k < 2 ? v.x : v.y;
        return (unsigned short)((k & 1) ? (w >> 16) : (w & 0xFFFFu));
    }
    __device__ static float get(const V &v, int k)
    {
        if constexpr (std::is_same<T, __half>::value)
            return ST<T>::dec(__ushort_as_half(bits(v, k)));
        else
            return __bfloat162float(__ushort_as_bfloat16(bits(v, k)));
    }
    __device__ static unsigned pack(float a, float b)
    {
        if constexpr (std::is_same<T, __half>::value) {
            const __half2 h = __floats2half2_rn(a * kHalfScale, b * kHalfScale);
            return *reinterpret_cast<const unsigned *>(&h);
        } else {
            const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
            return *reinterpret_cast<const unsigned *>(&h);
        }
    }
    __device__ static void set2(V &v, int k, float a, float b)
    {
        if (k == 0) v.x = pack(a, b);
        else v.y = pack(a, b);
    }
    // cells k, k + 1 from already encoded values
    __device__ static void set2_bits(V &v, int k, T a, T b)
    {
        const unsigned w = (unsigned)*reinterpret_cast<const unsigned short *>(&a) |
                           ((unsigned)*reinterpret_cast<const unsigned short *>(&b) << 16);
        if (k == 0) v.x = w;
        else v.y = w;
    }
    using P = unsigned;
    __device__ static P pair(const V &v, int k)
    {
        return k == 0 ? v.x : k == 1 ? __byte_perm(v.x, v.y, 0x5432) : v.y;
    }
    __device__ static void store_pair(T *p, const P &x) { *reinterpret_cast<unsigned *>(p) = x; }
    __device__ static void store_one(T *p, const V &v, int k) { *reinterpret_cast<unsigned short *>(p) = bits(v, k); }
    // Exchanged words: the one holding cell 3 (high half) / cell 0 (low half).
    using E = unsigned;
    __device__ static E last(const V &v) { return v.y; }
    __device__ static E first(const V &v) { return v.x; }
    __device__ static V shift_in_left(const V &v, E l)
    {
        return make_uint2(__byte_perm(l, v.x, 0x5432), __byte_perm(v.x, v.y, 0x5432));
    }
    __device__ static V shift_in_right(const V &v, E r)
    {
        return make_uint2(__byte_perm(v.x, v.y, 0x5432), __byte_perm(v.y, r, 0x5432));
    }
};
template <> struct Row4<__half> : Row4Half<__half> {};
template <> struct Row4<__nv_bfloat16> : Row4Half<__nv_bfloat16> {};

// Threads per CTA and the register target.
template <int DIM, int Q, typename T> struct RowCfg {
    static constexpr int NT = (DIM == 2) ? 256 : 128;
    static constexpr int R = (DIM == 2) ? 4 : 16;              // rows per cell-block
    static constexpr int NB = NT / R;                           // cell-blocks per CTA
    // A warp holds the same XR rows of 32 / XR consecutive blocks, so that
    // x neighbours of a block sit in the same warp, XR lanes away: 2D all 4
    // rows of 8 blocks; 3D all 16 rows of 2 blocks (half of the 16 rows of 4
    // blocks measured 4% slower on the D3Q19 384^3 cavity: the 3D row step is
    // bound by its 128 registers, not by the stores).
    static constexpr int XR = (DIM == 2) ? 4 : 16;
    static constexpr int words = Q * (sizeof(T) == 4 ? 4 : 2);  // registers of the row's populations
    static constexpr int MINB = (DIM == 2) ? (sizeof(T) == 4 ? 3 : 4) : (words <= 40 ? 4 : words <= 80 ? 2 : 1);
};

// Boundary hook on the closed domain-boundary links of cell I of the row:
// the value that bounces back into the cell's own slot (push_cell's hook
// branch).
template <int DIM, int Q, typename C, bool OFF>
__device__ __forceinline__ void hook_closed(C (&g)[Q], int I, int J, int K, const int *nrow, int preset, C ux, C uy,
                                            C uz, C U)
{
#pragma unroll
    for (int p = 1; p < Q; p++) {
        const int cx = lat_c(DIM, 0, p), cy = lat_c(DIM, 1, p), cz = lat_c(DIM, 2, p);
        const int nb = nrow[nbr_slot(DIM, I + cx, J + cy, K + cz)];
        if (nb < 0 && nb != N_SKIPID) {
            const C wp = C(lat_w(Q, p));
            const C off = OFF ? wp : C(0);
            g[p] = bc_hook<C>(preset, nb, g[p] + off, ux, uy, uz, wp, cx, cy, cz, U) - off;
        }
    }
}

// push_cell's stream-guard records for cell t of block b (post-collision g).
template <int DIM, int Q, typename T>
__device__ __forceinline__ void guard_cell(const typename ST<T>::C (&g)[Q], int b, int t, const int *nrow,
                                           const StepArgs &a)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
#pragma unroll
    for (int p = 1; p < Q; p++) {
        if (lat_half(DIM, p)) continue;
        const int cx = lat_c(DIM, 0, p), cy = lat_c(DIM, 1, p), cz = lat_c(DIM, 2, p);
        const int nb = nrow[nbr_slot(DIM, I + cx, J + cy, K + cz)];
        if (nb < 0) continue;
        const C full = g[p] + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        if (full > C(0)) continue;
        const int nc = nbr_cell(DIM, I + cx, J + cy, K + cz);
        const int k = atomicAdd(a.fix_count, 1);
        if (k < a.fix_cap) {
            a.fix_list[2 * k] = (long long)nb * BLK + lat_pb(DIM, p) * MC + nc;
            a.fix_list[2 * k + 1] = (long long)b * BLK + p * MC + t;
        }
    }
}

template <int DIM, int Q, typename T, bool SOLID>
__global__ void __launch_bounds__(RowCfg<DIM, Q, T>::NT, RowCfg<DIM, Q, T>::MINB) k_step_row(const StepArgs a)
{
    using C = typename ST<T>::C;
    using RW = Row4<T>;
    using V = typename RW::V;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    constexpr int NT = RowCfg<DIM, Q, T>::NT, R = RowCfg<DIM, Q, T>::R, NB = RowCfg<DIM, Q, T>::NB;
    constexpr int W = Meta<DIM>::W;
    __shared__ int s_meta[NB][W];
    const int tid = threadIdx.x;
    constexpr int XR = RowCfg<DIM, Q, T>::XR, BPW = 32 / XR, SL = R / XR;
    const int warp = tid >> 5, lane = tid & 31;
    const int lb = (warp / SL) * BPW + lane / XR, r = (warp % SL) * XR + lane % XR;
    const int J = r & 3, K = (DIM == 3) ? (r >> 2) : 0;

    // Block IDs and metadata rows are written only by mesh passes, so they are
    // read before the wait on the predecessor (programmatic dependent launch).
    const int kap = blockIdx.x * NB + lb;
    const int b = (kap < a.n) ? __ldg(&a.ids[kap]) : -1;
    for (int i = r; i < W; i += R) s_meta[lb][i] = (b >= 0) ? __ldg(&a.meta[(long long)b * W + i]) : 0;
    pdl_wait();

    const unsigned seed = step_seed(a);
    const T *__restrict__ fin = static_cast<const T *>(a.fin);
    T *__restrict__ fo = static_cast<T *>(a.fout);
    const long long own = (long long)b * BLK + r * 4;   // element offset of slot 0 of this row
    V v[Q];
    if (b >= 0) {
#pragma unroll
        for (int s = 0; s < Q; s++) v[s] = RW::load(fin + own + s * MC);
    }
    __syncthreads();
    const int *nrow = s_meta[lb];
    const int fl = nrow[Meta<DIM>::FLAGS];
    const bool run = b >= 0 && !(fl & META_WALL);
    bool main = false;   // the row-wise path: collided here, streamed below
    if (run && !(fl & META_ACTIVE)) {
        // Inactive (refined solid) block: carried unchanged, as k_step does.
        if (SOLID) {
#pragma unroll
            for (int s = 0; s < Q; s++) RW::store(fo + own + s * MC, v[s]);
        }
    } else if (run && SOLID && (fl & META_NEARSOLID)) {
        // A solid cell in this block or a neighbour: per-cell push with the
        // solid-neighbour test.
        const bool hook = (fl & META_ONB) && a.bc_preset != AGAL_BC_NONE;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int t = r * 4 + k;
            if (__ldg(&a.cmask[(long long)b * MC + t]) == CELL_SOLID) {
#pragma unroll
                for (int s = 0; s < Q; s++) fo[own + s * MC + k] = fin[own + s * MC + k];
                continue;
            }
            C g[Q];
#pragma unroll
            for (int p = 0; p < Q; p++) g[p] = RW::get(v[lat_pb(DIM, p)], k);
            C ux, uy, uz;
            collide_cell<DIM, Q, T>(g, a, ux, uy, uz);
            push_cell<DIM, Q, T, true>(g, ux, uy, uz, b, t, nrow, hook, fo, a, seed);
        }
    } else if (run) {
        main = true;
        const bool hook = (fl & META_ONB) && a.bc_preset != AGAL_BC_NONE;
        bool bad = false;
        // Collide the row two cells at a time; v[p] then holds the
        // post-collision values of direction p (slot pb(p) was read first).
#pragma unroll
        for (int k = 0; k < 4; k += 2) {
            C g0[Q], g1[Q];
#pragma unroll
            for (int p = 0; p < Q; p++) {
                g0[p] = RW::get(v[lat_pb(DIM, p)], k);
                g1[p] = RW::get(v[lat_pb(DIM, p)], k + 1);
            }
            C ux0, uy0, uz0, ux1, uy1, uz1;
            collide_cell<DIM, Q, T>(g0, a, ux0, uy0, uz0);
            collide_cell<DIM, Q, T>(g1, a, ux1, uy1, uz1);
#pragma unroll
            for (int p = 1; p < Q; p++) {
                if (lat_half(DIM, p)) continue;
                const C w = ST<T>::OFF ? C(lat_w(Q, p)) : C(0);
                bad |= !(g0[p] + w > C(0));
                bad |= !(g1[p] + w > C(0));
            }
            if (hook) {
                hook_closed<DIM, Q, C, ST<T>::OFF>(g0, k, J, K, nrow, a.bc_preset, ux0, uy0, uz0, C(a.u_ref));
                hook_closed<DIM, Q, C, ST<T>::OFF>(g1, k + 1, J, K, nrow, a.bc_preset, ux1, uy1, uz1, C(a.u_ref));
            }
            if constexpr (sizeof(T) == 2) {
                if (a.sr) {
                    const unsigned r0 = sr_cell_of<DIM>(b, r * 4 + k, seed);
                    const unsigned r1 = sr_cell_of<DIM>(b, r * 4 + k + 1, seed);
#pragma unroll
                    for (int p = 0; p < Q; p++)
                        RW::set2_bits(v[p], k, enc_r<T>(g0[p], r0 * sr_dir(p), true),
                                      enc_r<T>(g1[p], r1 * sr_dir(p), true));
                } else {
#pragma unroll
                    for (int p = 0; p < Q; p++) RW::set2(v[p], k, g0[p], g1[p]);
                }
            } else {
#pragma unroll
                for (int p = 0; p < Q; p++) RW::set2(v[p], k, g0[p], g1[p]);
            }
        }
        if (bad) {
            // Rare: recompute the row's collisions from the input and record
            // the links the reference's guard refuses.
#pragma unroll 1
            for (int k = 0; k < 4; k++) {
                C g[Q];
#pragma unroll
                for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(fin[own + lat_pb(DIM, p) * MC + k]);
                C ux, uy, uz;
                collide_cell<DIM, Q, T>(g, a, ux, uy, uz);
                guard_cell<DIM, Q, T>(g, b, r * 4 + k, nrow, a);
            }
        }
    }

    // Stream of the row-wise path (all lanes take part in the exchanges).
    // Direction p goes to row (J + c_y, K + c_z) of the block in that y/z
    // neighbour slot, shifted by c_x; closed links bounce back into the
    // cell's own slot p.  For c_x = +1 the destination row's cell 0 comes
    // from cell 3 of the left neighbour's row: when that row belongs to lane
    // - XR of this warp and lands in the same destination block, it is
    // exchanged and the destination row is written whole (one aligned vector
    // store, full sectors), and the neighbour leaves its cell 3 out; likewise
    // for c_x = -1 with the right neighbour (lane + XR).  Rows at the warp's
    // edges, or next to a block on another path, keep the element-wise
    // stores.  Every element is written once either way.
    constexpr unsigned ALL = 0xffffffffu;
    const bool has_l = lane >= XR, has_r = lane + XR < 32;
    const int s0 = (DIM == 3) ? 12 : 3;   // slot of the (0, 0, 0) offset minus one: x - 1
    const int left_b = __shfl_up_sync(ALL, b, XR);
    const bool left_main = __shfl_up_sync(ALL, main, XR);
    const bool left_ok = main && has_l && left_main && nrow[s0] == left_b && left_b >= 0;
    // Every lane executes every exchange (never inside a short-circuit): a
    // lane that skipped one would leave the rest of the warp waiting.
    const bool right_left_ok = __shfl_down_sync(ALL, left_ok, XR);
    const bool right_ok = has_r && right_left_ok;
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const int cx = lat_c(DIM, 0, p), cy = lat_c(DIM, 1, p), cz = lat_c(DIM, 2, p);
        const int q = lat_pb(DIM, p);
        const int Jn = J + cy, Kn = K + cz;
        const int syz = (Jn < 0 ? 0 : Jn > 3 ? 6 : 3) + (DIM == 3 ? (Kn < 0 ? 0 : Kn > 3 ? 18 : 9) : 0);
        const int rn = (Jn & 3) + (DIM == 3 ? 4 * (Kn & 3) : 0);
        const int Byz = nrow[syz + 1];
        T *back = fo + own + p * MC;
        T *dst = fo + (long long)Byz * BLK + q * MC + rn * 4;
        if (cx == 0) {
            if (main) RW::store(Byz >= 0 ? dst : back, v[p]);
        } else if (cx > 0) {
            const int Bx = nrow[syz + 2];
            const typename RW::E lv = __shfl_up_sync(ALL, RW::last(v[p]), XR);
            const int lBx = __shfl_up_sync(ALL, Bx, XR);
            const bool full = left_ok && Byz >= 0 && lBx == Byz;
            const bool r_full = __shfl_down_sync(ALL, full, XR);
            const bool given = has_r && r_full;   // cell 3 written by lane + XR
            if (main) {
                if (Byz >= 0) {
                    if (full) {
                        RW::store(dst, RW::shift_in_left(v[p], lv));
                    } else {
                        RW::store_one(dst + 1, v[p], 0);
                        RW::store_pair(dst + 2, RW::pair(v[p], 1));
                    }
                } else {
                    RW::store_pair(back, RW::pair(v[p], 0));
                    RW::store_one(back + 2, v[p], 2);
                }
                if (!given) RW::store_one(Bx >= 0 ? fo + (long long)Bx * BLK + q * MC + rn * 4 : back + 3, v[p], 3);
            }
        } else {
            const int Bx = nrow[syz + 0];
            const typename RW::E rv = __shfl_down_sync(ALL, RW::first(v[p]), XR);
            const int rBx = __shfl_down_sync(ALL, Bx, XR);
            const bool full = right_ok && Byz >= 0 && rBx == Byz;
            const bool l_full = __shfl_up_sync(ALL, full, XR);
            const bool given = has_l && l_full;   // cell 0 written by lane - XR
            if (main) {
                if (Byz >= 0) {
                    if (full) {
                        RW::store(dst, RW::shift_in_right(v[p], rv));
                    } else {
                        RW::store_pair(dst, RW::pair(v[p], 1));
                        RW::store_one(dst + 2, v[p], 3);
                    }
                } else {
                    RW::store_one(back + 1, v[p], 1);
                    RW::store_pair(back + 2, RW::pair(v[p], 2));
                }
                if (!given) RW::store_one(Bx >= 0 ? fo + (long long)Bx * BLK + q * MC + rn * 4 + 3 : back, v[p], 0);
            }
        }
    }
    if (a.fix_ticket) fused_fixup<T>(a);
}

}  // namespace

template <int DIM, int Q, typename T>
int launch_step_row(agal_ctx *c, const StepArgs &a, int n)
{
    using Cfg = RowCfg<DIM, Q, T>;
    const unsigned grid = (unsigned)((n + Cfg::NB - 1) / Cfg::NB);
    if (c->geometry_init)
        AGAL_CUDA(c, launch_pdl(k_step_row<DIM, Q, T, true>, dim3(grid), dim3(Cfg::NT), 0, c->stream, a));
    else
        AGAL_CUDA(c, launch_pdl(k_step_row<DIM, Q, T, false>, dim3(grid), dim3(Cfg::NT), 0, c->stream, a));
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

#define AGAL_ROW_INST(D, Q, T) template int launch_step_row<D, Q, T>(agal_ctx *, const StepArgs &, int);
AGAL_ROW_INST(2, 9, float)
AGAL_ROW_INST(2, 9, __half)
AGAL_ROW_INST(2, 9, __nv_bfloat16)
AGAL_ROW_INST(3, 19, float)
AGAL_ROW_INST(3, 19, __half)
AGAL_ROW_INST(3, 19, __nv_bfloat16)
AGAL_ROW_INST(3, 27, float)
AGAL_ROW_INST(3, 27, __half)
AGAL_ROW_INST(3, 27, __nv_bfloat16)

}  // namespace agal
