// Tile form of the fused collide + boundary + stream step for the root level
// of 2D cases (variant 5).
//
// Why: the push step writes each post-collision value to its destination
// cell, and a cell-block's slot is only 16 cells (32 bytes in FP16), so a
// warp's store lands in many partly written sectors of many blocks.  On a
// B200 the L1-to-L2 request path, not DRAM, then bounds the step: FP16 takes
// as long as FP32 for half the bytes.  Here one CTA owns every output value of
// an 8 x 8 tile of cell-blocks and writes each block's Q x 16 slots as one
// contiguous run of 16-byte stores (whole 128-byte lines).
//
// Per CTA:
//  1. cp.async copies the tile's 64 cell-blocks and the 36 blocks around it
//     (whole blocks: contiguous runs of full lines) into shared memory.
//  2. Every cell of the tile and of its one-cell halo ring (34 x 34 cells) is
//     collided (collide_cell, the same arithmetic as every other variant);
//     the post-collision values f*_p go to shared memory, post[p][y][x].
//  3. Each output slot q of cell z is gathered: f*_{pb(q)}(z + c_q) over an
//     open link; f*_q(z) over a closed one (no block there), passed through
//     the boundary hook on a domain boundary (push_cell's bounce-back).  The
//     reference's stream guard (solver_lbm_kernels.cu:620-628: the swap of a
//     link is refused when the value on its non-owning side is not positive)
//     is a local choice here: a refused link keeps f*_q(z), which is what the
//     fix-up list of the push variants restores.  Tiles without a refused
//     link or a missing neighbour (almost all) take a select-free gather.
// The halo ring is recomputed by the neighbouring tiles (13% more
// collisions) and read from L2; DRAM traffic stays at one read and one write
// of each population.
//
// Requirements (else the launcher runs variant 4): a 2D case, the root level
// L0 holding the whole root grid (ids 0.. in x-fastest order, as every case
// does), root blocks per side a multiple of 8, no geometry, no LES, FP32,
// FP16 or BF16 storage.  The tile table (agal_build_tiles) lists per tile the
// 10 x 10 block IDs of the tile and its ring; ring entries are the neighbour
// table's entries of the adjacent tile block (boundary pseudo-IDs, periodic
// wrap), interior entries carry the block's on-boundary flag in bit 30.
#include <cuda_runtime.h>

#include <type_traits>

#include "ctx.h"
#include "lattice.cuh"
#include "mbar.cuh"
#include "step_common.cuh"
#include "storage.cuh"

namespace agal {
namespace {

constexpr int TB = 8;             // cell-blocks per tile side
constexpr int TC = 4 * TB;        // cells per tile side
constexpr int HB = TB + 2;        // blocks per side of the tile and its ring
constexpr int NH = HB * HB;       // 100 block IDs per tile
constexpr int NI = TB * TB;       // 64 tile blocks
constexpr int PX = TC + 8;        // plane row stride: cell x at column x + 4 (x = -1 .. 32)
constexpr int PY = TC + 2;        // plane rows: cell y at row y + 1
constexpr int PS = PY * PX + 20;  // plane stride (floats): 16-byte multiple, planes 4 banks apart
constexpr int NT = 288;           // 9 warps: 8 collide the tile's rows, 1 the ring
constexpr int ONB_BIT = 1 << 30;

template <typename T> struct TileSmem {
    static constexpr int BLKB = 9 * 16 * (int)sizeof(T);       // bytes of one cell-block (multiple of 16)
    static constexpr int OFF_PUSH = 0;                          // [9][PS] pushed post-collision values
    static constexpr int OFF_RAW = (OFF_PUSH + 9 * PS * 4 + 127) / 128 * 128;   // [NH][Q][16] staged blocks
    // [2][TC*TC] velocity for the boundary hook: in the staging buffer, which
    // boundary tiles release before their gather
    static constexpr int OFF_U = OFF_RAW;
    static constexpr int OFF_ID = OFF_RAW + NH * BLKB;          // [3][NH] block IDs of three tiles
    static constexpr int OFF_BAR = OFF_ID + 3 * NH * 4;         // mbarrier
    static constexpr int BYTES = OFF_BAR + 16;
    static_assert(BLKB % 16 == 0 && OFF_RAW % 128 == 0 && OFF_BAR % 8 == 0, "alignment");
    static_assert(2 * TC * TC * 4 <= NH * BLKB, "velocity fits the staging buffer");
};

// Four consecutive stored values (one row of a slot) decoded to FP32.
template <typename T> __device__ __forceinline__ void load_row4(const T *p, float (&o)[4]);
template <> __device__ __forceinline__ void load_row4<float>(const float *p, float (&o)[4])
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
template <> __device__ __forceinline__ void load_row4<__half>(const __half *p, float (&o)[4])
{
    const uint2 v = *reinterpret_cast<const uint2 *>(p);
    const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&v.y));
    o[0] = a.x * kHalfUnscale; o[1] = a.y * kHalfUnscale; o[2] = b.x * kHalfUnscale; o[3] = b.y * kHalfUnscale;
}
template <> __device__ __forceinline__ void load_row4<__nv_bfloat16>(const __nv_bfloat16 *p, float (&o)[4])
{
    const uint2 v = *reinterpret_cast<const uint2 *>(p);
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&v.y));
    o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// Eight encoded values (two rows of one slot) as one output write.
template <typename T> __device__ __forceinline__ void store_rows2(T *dst, const float (&v)[8]);
template <> __device__ __forceinline__ void store_rows2<float>(float *dst, const float (&v)[8])
{
    reinterpret_cast<float4 *>(dst)[0] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float4 *>(dst)[1] = make_float4(v[4], v[5], v[6], v[7]);
}
template <typename H2, typename T>
__device__ __forceinline__ void store_rows2_half(T *dst, const float (&v)[8])
{
    unsigned w[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        H2 h;
        if constexpr (std::is_same<T, __half>::value)
            h = __floats2half2_rn(v[2 * k] * kHalfScale, v[2 * k + 1] * kHalfScale);
        else
            h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
        w[k] = *reinterpret_cast<const unsigned *>(&h);
    }
    *reinterpret_cast<uint4 *>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
}
template <> __device__ __forceinline__ void store_rows2<__half>(__half *dst, const float (&v)[8])
{
    store_rows2_half<__half2>(dst, v);
}
template <> __device__ __forceinline__ void store_rows2<__nv_bfloat16>(__nv_bfloat16 *dst, const float (&v)[8])
{
    store_rows2_half<__nv_bfloat162>(dst, v);
}

// Eight already encoded half values as one 16-byte store.
template <typename T> __device__ __forceinline__ void store_encoded8(T *dst, const T (&h)[8])
{
    unsigned w[4];
#pragma unroll
    for (int k = 0; k < 4; k++)
        w[k] = (unsigned)*reinterpret_cast<const unsigned short *>(&h[2 * k]) |
               ((unsigned)*reinterpret_cast<const unsigned short *>(&h[2 * k + 1]) << 16);
    *reinterpret_cast<uint4 *>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
}

struct TileArgs {
    StepArgs s;
    const int *tiles;   // [n_tiles][NH]
    int n_tiles;
};

// Non-positive value on the non-owning side of some link of this cell (the
// stream guard may refuse a swap): any direction outside the half set.
template <typename T>
__device__ __forceinline__ bool guard_risk(const float (&g)[9])
{
    bool bad = false;
#pragma unroll
    for (int p = 1; p < 9; p++)
        if (!lat_half(2, p)) bad |= !(g[p] + (ST<T>::OFF ? float(lat_w(9, p)) : 0.f) > 0.f);
    return bad;
}

// Ring cell h of a tile (tile cell coordinates -1 .. 32): 0..31 left column
// (x = -1), 32..63 right (x = 32), 64..95 bottom row (y = -1), 96..127 top
// (y = 32), 128..131 the corners.
__device__ __forceinline__ void ring_cell(int h, int &hx, int &hy)
{
    if (h < 2 * TC) { hx = (h < TC) ? -1 : TC; hy = h & (TC - 1); }
    else if (h < 4 * TC) { hy = (h < 3 * TC) ? -1 : TC; hx = h & (TC - 1); }
    else { hx = (h & 1) ? TC : -1; hy = (h & 2) ? TC : -1; }
}
__device__ __forceinline__ int ring_block(int hx, int hy) { return ((hy + 4) >> 2) * HB + ((hx + 4) >> 2); }

// Persistent: CTA c handles tiles c, c + G, c + 2G, ... (G = grid size).
// While tile i is gathered and stored, the bulk copies of tile i+1's blocks
// land (boundary tiles, which keep the hook velocities in the staging
// buffer, issue them after their gather).
template <typename T>
__global__ void __maxnreg__(96) k_step_tile2d(const TileArgs ta)
{
    using C = typename ST<T>::C;
    using SM = TileSmem<T>;
    constexpr int Q = 9, MC = 16, BLK = Q * MC;
    constexpr bool OFF = ST<T>::OFF;
    extern __shared__ __align__(128) unsigned char smem[];
    float *push = reinterpret_cast<float *>(smem + SM::OFF_PUSH);
    T *raw = reinterpret_cast<T *>(smem + SM::OFF_RAW);
    float *su = reinterpret_cast<float *>(smem + SM::OFF_U);
    int *sid = reinterpret_cast<int *>(smem + SM::OFF_ID);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + SM::OFF_BAR);
    const StepArgs &a = ta.s;
    const int tid = threadIdx.x;
    const int G = gridDim.x;
    const T *__restrict__ fin = static_cast<const T *>(a.fin);
    T *__restrict__ fo = static_cast<T *>(a.fout);

    // Tile table rows: written by mesh passes only, so the first two are read
    // before the wait on the predecessor (programmatic dependent launch).
    int t = blockIdx.x;
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    if (tid < NH) {
        sid[tid] = __ldg(&ta.tiles[(long long)t * NH + tid]);
        if (t + G < ta.n_tiles) sid[NH + tid] = __ldg(&ta.tiles[(long long)(t + G) * NH + tid]);
    }
    __syncthreads();
    pdl_wait();
    const unsigned seed = step_seed(a);
    // The blocks of a tile and its ring: one bulk copy each (a contiguous
    // Q x 16 run); warp 0 counts them for the expected bytes.
    auto issue = [&](const int *ids) {
        if (tid < 32) {
            int cnt = 0;
#pragma unroll
            for (int k = 0; k < (NH + 31) / 32; k++) {
                const int idx = tid + 32 * k;
                cnt += __popc(__ballot_sync(0xffffffffu, idx < NH && ids[idx] >= 0));
            }
            if (tid == 0) mbar_arrive_expect_tx(bar, (unsigned)(cnt * SM::BLKB));
        }
        if (tid < NH && ids[tid] >= 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bulk_g2s(raw + (size_t)tid * BLK, fin + (size_t)(ids[tid] & ~ONB_BIT) * BLK, SM::BLKB, bar);
        }
    };
    issue(sid);

    // Per-thread constants of the gather: unit u = tid % 144 of a tile block
    // row (block bxo, slot q, row pair hh), two block rows per pass.
    const int half_sel = tid / 144, u = tid - half_sel * 144;
    const int bxo = u / 18, rem = u - bxo * 18;
    const int q = rem >> 1, hh = rem & 1;
    const int cxq = lat_c(2, 0, q), cyq = lat_c(2, 1, q), qb = lat_pb(2, q);
    const bool halfq = lat_half(2, q);
    const float wq = OFF ? float(lat_w(Q, q)) : 0.f;
    const int y0 = tid >> 3, bx0 = tid & 7;
    bool late_issue = false;   // the previous (boundary) tile left the next issue to this iteration

    for (int i = 0; t < ta.n_tiles; i++, t += G) {
        const int *ids = sid + (i % 3) * NH;
        if (late_issue) issue(ids);
        const bool landed = mbar_wait(bar, (unsigned)(i & 1), a.status);
        const int st = __syncthreads_or(((tid < NH && ids[tid] < 0) ? 1 : 0) | (landed ? 0 : 2));
        if (st & 2) {
            // A copy did not land in time (AGAL_ERR_TIMEOUT is recorded): wait
            // once more, bounded, so nothing is in flight when the CTA exits.
            mbar_wait(bar, (unsigned)(i & 1), a.status);
            return;
        }
        const bool missing = st & 1;

        // 1. Collide from the staged blocks: warps 0-7 a row of four tile
        //    cells each, warp 8 the 128 edge ring cells (four each) and the
        //    four corners (of which only the diagonal into the tile is kept).
        float gi[4][Q];
        float ui[4][2];
        float corner = 0.f;
        bool bad = false;
        if (tid < 256) {
            const T *src = raw + (size_t)(((y0 >> 2) + 1) * HB + bx0 + 1) * BLK + (y0 & 3) * 4;
            float row[Q][4];
#pragma unroll
            for (int s = 0; s < Q; s++) load_row4<T>(src + s * MC, row[s]);
#pragma unroll
            for (int k = 0; k < 4; k++) {
#pragma unroll
                for (int p = 0; p < Q; p++) gi[k][p] = row[lat_pb(2, p)][k];
                C ux, uy, uz;
                collide_cell<2, Q, T>(gi[k], a, ux, uy, uz);
                ui[k][0] = ux;
                ui[k][1] = uy;
                bad |= guard_risk<T>(gi[k]);
            }
        } else {
            const int j = tid - 256;
#pragma unroll
            for (int m = 0; m < 5; m++) {
                if (m == 4 && j >= 4) break;
                int hx, hy;
                ring_cell(m < 4 ? 4 * j + m : 128 + j, hx, hy);
                const int k = ring_block(hx, hy);
                if (ids[k] < 0) continue;
                const T *src = raw + (size_t)k * BLK + (hx & 3) + 4 * (hy & 3);
                float g[Q];
#pragma unroll
                for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(src[lat_pb(2, p) * MC]);
                C ux, uy, uz;
                collide_cell<2, Q, T>(g, a, ux, uy, uz);
                bad |= guard_risk<T>(g);
                if (m < 4) {
#pragma unroll
                    for (int p = 0; p < Q; p++) gi[m][p] = g[p];
                } else {
                    // the corner's diagonal towards the tile
                    const int pd = (hx < 0) ? ((hy < 0) ? 5 : 8) : ((hy < 0) ? 6 : 7);
#pragma unroll
                    for (int p = 5; p < Q; p++)
                        if (p == pd) corner = g[p];
                }
            }
        }
        // The staged blocks are consumed: the next tile's copies may start
        // (a boundary tile first keeps its velocities there).
        const int slow1 = __syncthreads_or(bad);
        late_issue = false;
        if (t + G < ta.n_tiles) {
            if (!missing) issue(sid + ((i + 1) % 3) * NH);
            else late_issue = true;
        }
        if (tid < 256) {
            // push f*_p of cell (x, y) to (x + c_p, y + c_p): plane p then
            // holds, at each cell, the value arriving there along p
#pragma unroll
            for (int p = 0; p < Q; p++) {
                const int cx = lat_c(2, 0, p), cy = lat_c(2, 1, p);
                float *dst = push + p * PS + (y0 + cy + 1) * PX + 4 + 4 * bx0 + cx;
                if (cx == 0) {
                    *reinterpret_cast<float4 *>(dst) = make_float4(gi[0][p], gi[1][p], gi[2][p], gi[3][p]);
                } else {
#pragma unroll
                    for (int k = 0; k < 4; k++) dst[k] = gi[k][p];
                }
            }
            if (missing) {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    su[y0 * TC + 4 * bx0 + k] = ui[k][0];
                    su[TC * TC + y0 * TC + 4 * bx0 + k] = ui[k][1];
                }
            }
        } else {
            const int j = tid - 256;
#pragma unroll
            for (int m = 0; m < 5; m++) {
                if (m == 4 && j >= 4) break;
                int hx, hy;
                ring_cell(m < 4 ? 4 * j + m : 128 + j, hx, hy);
                if (ids[ring_block(hx, hy)] < 0) continue;
                if (m < 4) {
#pragma unroll
                    for (int p = 1; p < Q; p++) {
                        const int tx = hx + lat_c(2, 0, p), ty = hy + lat_c(2, 1, p);
                        if (tx >= 0 && tx < TC && ty >= 0 && ty < TC) push[p * PS + (ty + 1) * PX + 4 + tx] = gi[m][p];
                    }
                } else {
                    const int pd = (hx < 0) ? ((hy < 0) ? 5 : 8) : ((hy < 0) ? 6 : 7);
                    push[pd * PS + (hy + lat_c(2, 1, pd) + 1) * PX + 4 + hx + lat_c(2, 0, pd)] = corner;
                }
            }
        }
        const int slow = __syncthreads_or(bad) | slow1 | (missing ? 1 : 0);

        // 2. Gather and write: output slot q of cell z is the value arriving
        //    along pb(q), push[pb(q)][z]; two rows of four cells per unit.
#pragma unroll 1
        for (int pass = 0; pass < TB / 2; pass++) {
            const int by = 2 * pass + half_sel;
            const int e = ids[(by + 1) * HB + bxo + 1];
            const int zx = 4 * bxo, zy = 4 * by + 2 * hh;
            const float *srow = push + qb * PS + (zy + 1) * PX + 4 + zx;
            float v[8];
            {
                const float4 r0 = *reinterpret_cast<const float4 *>(srow);
                const float4 r1 = *reinterpret_cast<const float4 *>(srow + PX);
                v[0] = r0.x; v[1] = r0.y; v[2] = r0.z; v[3] = r0.w;
                v[4] = r1.x; v[5] = r1.y; v[6] = r1.z; v[7] = r1.w;
            }
            // a value keeps the rounding key of the cell and direction it was
            // collided for: (z + c_q, pb(q)) when gathered, (z, q) when it
            // bounces back or its swap is refused
            bool mine[8] = {false, false, false, false, false, false, false, false};
            if (slow && q != 0) {
                const bool hook = (e & ONB_BIT) && a.bc_preset != AGAL_BC_NONE;
#pragma unroll
                for (int k = 0; k < 8; k++) {
                    const int x = zx + (k & 3), y = zy + (k >> 2);
                    const int nb = ids[ring_block(x + cxq, y + cyq)];
                    // f*_q(z): pushed along q to z + c_q
                    const float own = push[q * PS + (y + cyq + 1) * PX + 4 + x + cxq];
                    if (nb < 0) {
                        // closed link: bounce back, hooked on a domain boundary
                        float vv = own;
                        if (hook && nb != N_SKIPID) {
                            const int c = y * TC + x;
                            vv = bc_hook<C>(a.bc_preset, nb, own + wq, su[c], su[TC * TC + c], C(0),
                                            C(lat_w(Q, q)), cxq, cyq, 0, C(a.u_ref)) -
                                 wq;
                        }
                        v[k] = vv;
                        mine[k] = true;
                    } else {
                        const bool refused = halfq ? !(v[k] + wq > 0.f) : !(own + wq > 0.f);
                        if (refused) {
                            v[k] = own;
                            mine[k] = true;
                        }
                    }
                }
            }
            T *dst = fo + (long long)(e & ~ONB_BIT) * BLK + q * MC + hh * 8;
            if constexpr (sizeof(T) == 2) {
                if (a.sr) {
                    T h[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const int x = zx + (k & 3), y = zy + (k >> 2);
                        unsigned rnd;
                        if (mine[k]) {
                            rnd = sr_cell_of<2>(e & ~ONB_BIT, (x & 3) + 4 * (y & 3), seed) * sr_dir(q);
                        } else {
                            const int sx = x + cxq, sy = y + cyq;
                            rnd = sr_cell_of<2>(ids[ring_block(sx, sy)] & ~ONB_BIT, (sx & 3) + 4 * (sy & 3), seed) *
                                  sr_dir(qb);
                        }
                        h[k] = enc_r<T>(v[k], rnd, true);
                    }
                    store_encoded8<T>(dst, h);
                    continue;
                }
            }
            store_rows2<T>(dst, v);
        }
        // Tile i + 2's IDs go where tile i - 1's were; the planes, the
        // velocities and this tile's IDs stay untouched until every thread is
        // past its gather.
        if (tid < NH && t + 2 * G < ta.n_tiles)
            sid[((i + 2) % 3) * NH + tid] = __ldg(&ta.tiles[(long long)(t + 2 * G) * NH + tid]);
        __syncthreads();
    }
}

// Tile table: per tile the 10 x 10 block IDs of the tile and its ring.
__global__ void k_build_tiles2d(int nbx, int nby, long long nmb, const int *nbr, const int *onb, int *tiles)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int tx_n = nbx / TB, ty_n = nby / TB;
    if (g >= (long long)tx_n * ty_n * NH) return;
    const int tile = (int)(g / NH), pos = (int)(g % NH);
    const int i = pos % HB - 1, j = pos / HB - 1;                 // -1 .. 8
    const int ic = i < 0 ? 0 : (i >= TB ? TB - 1 : i), jc = j < 0 ? 0 : (j >= TB ? TB - 1 : j);
    const int bx = (tile % tx_n) * TB + ic, by = (tile / tx_n) * TB + jc;
    const int b = bx + nbx * by;                                   // root-grid ID (x fastest)
    int v;
    if (i == ic && j == jc) {
        v = b | (onb[b] == 1 ? ONB_BIT : 0);
    } else {
        const int S = (i - ic + 1) + 3 * (j - jc + 1);             // lexicographic neighbour slot
        v = nbr[b + (long long)lat_map(2, S) * nmb];
    }
    tiles[g] = v;
}

}  // namespace

// Opt the tile kernel into its dynamic shared memory and size its persistent
// grid (resident CTAs per SM x SMs), once per device; outside any stream
// capture.
template <typename T>
int prepare_step_tile(int *grid_out)
{
    static int grid[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return AGAL_ERR_CUDA;
    if (!grid[dev]) {
        if (cudaFuncSetAttribute(k_step_tile2d<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 TileSmem<T>::BYTES) != cudaSuccess ||
            cudaFuncSetAttribute(k_step_tile2d<T>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared) != cudaSuccess)
            return AGAL_ERR_CUDA;
        int per_sm = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_tile2d<T>, NT, TileSmem<T>::BYTES) !=
                cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return AGAL_ERR_CUDA;
        grid[dev] = (per_sm > 0 ? per_sm : 1) * sms;
    }
    if (grid_out) *grid_out = grid[dev];
    return AGAL_OK;
}

// Launch the tile step of the root level; returns AGAL_ERR_UNSUPPORTED when
// the case has no tile table (the caller runs another variant).
template <int DIM, int Q, typename T>
int launch_step_tile(agal_ctx *c, const StepArgs &a, int L)
{
    if constexpr (DIM != 2 || Q != 9 || std::is_same<T, double>::value) {
        return AGAL_ERR_UNSUPPORTED;
    } else {
        if (L != c->L0 || c->n_tiles <= 0 || c->nu_sgs) return AGAL_ERR_UNSUPPORTED;
        int grid = 0;
        if (prepare_step_tile<T>(&grid) != AGAL_OK)
            return agal_set_err(c, AGAL_ERR_CUDA, "cudaFuncSetAttribute(k_step_tile2d)");
        if (grid > c->n_tiles) grid = c->n_tiles;
        TileArgs ta{a, c->tiles, c->n_tiles};
        AGAL_CUDA(c, launch_pdl(k_step_tile2d<T>, dim3(grid), dim3(NT), (size_t)TileSmem<T>::BYTES, c->stream, ta));
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
}

#define AGAL_TILE_INST(D, Q, T) template int launch_step_tile<D, Q, T>(agal_ctx *, const StepArgs &, int);
AGAL_TILE_INST(2, 9, float)
AGAL_TILE_INST(2, 9, double)
AGAL_TILE_INST(2, 9, __half)
AGAL_TILE_INST(2, 9, __nv_bfloat16)
AGAL_TILE_INST(3, 19, float)
AGAL_TILE_INST(3, 19, double)
AGAL_TILE_INST(3, 19, __half)
AGAL_TILE_INST(3, 19, __nv_bfloat16)
AGAL_TILE_INST(3, 27, float)
AGAL_TILE_INST(3, 27, double)
AGAL_TILE_INST(3, 27, __half)
AGAL_TILE_INST(3, 27, __nv_bfloat16)

}  // namespace agal

// Build (or drop) the tile table for the root level; called after mesh
// changes (agal_build_meta).  Returns AGAL_OK when the tile step is not
// available (c->n_tiles stays 0).
int agal_build_tiles(agal_ctx *c)
{
    using namespace agal;
    c->n_tiles = 0;
    c->n_ptiles = agal_count_ptiles(c);
    if (c->dim != 2 || c->geometry_init) return AGAL_OK;
    const int nbx = c->Nx / 4, nby = c->Ny / 4;
    if (nbx % TB || nby % TB || c->n_ids[c->L0] != nbx * nby) return AGAL_OK;
    const int nt = (nbx / TB) * (nby / TB);
    if (!c->tiles) AGAL_CUDA(c, cudaMalloc(&c->tiles, sizeof(int) * (size_t)nt * NH));
    const long long tot = (long long)nt * NH;
    k_build_tiles2d<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(nbx, nby, c->nmb, c->cblock_ID_nbr,
                                                                         c->cblock_ID_onb, c->tiles);
    AGAL_CUDA(c, cudaGetLastError());
    if (prepare_step_tile<float>(nullptr) || prepare_step_tile<__half>(nullptr) ||
        prepare_step_tile<__nv_bfloat16>(nullptr))
        return agal_set_err(c, AGAL_ERR_CUDA, "cudaFuncSetAttribute(k_step_tile2d)");
    c->n_tiles = nt;
    return AGAL_OK;
}
