// Warp-specialised, persistent form of the fused collide + boundary + stream
// step, with the cell-blocks staged in shared memory by TMA bulk copies.
//
// Each CTA runs one producer warp and eight consumer warps over a ring of NS
// shared-memory stages.  A stage holds BPS cell-blocks: their populations
// (one contiguous Q x M_CBLOCK chunk per block in the block-major layout, so
// one cp.async.bulk per block), their neighbour rows and flags.  The producer
// fills stage s and arms its `full` mbarrier with the expected byte count;
// consumers wait on it, collide each cell from shared memory, push the
// results to global memory exactly as the plain kernel does, and arrive on
// the stage's `empty` mbarrier.  Loads for the next NS-1 stages stay in flight
// while the current one is computed, which the one-shot kernel cannot do.
//
// Every mbarrier wait is bounded (kWaitNs of wall clock); on expiry the
// thread records AGAL_ERR_TIMEOUT in the status word and leaves its loop, and
// the producer still waits (bounded) for the copies it issued before exiting,
// so no bulk copy is in flight when the CTA ends.  No multicast is used.
#include <cuda_runtime.h>

#include <cstdint>

#include "ctx.h"
#include "lattice.cuh"
#include "mbar.cuh"
#include "step_common.cuh"
#include "storage.cuh"

namespace agal {
namespace {

constexpr size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

// Stage geometry: ~20 KB of populations per stage (at most 64 blocks), 3 or
// 4 stages.  A stage holds, per block: populations, metadata row, block ID.
template <int DIM, int Q, typename T> struct TmaCfg {
    static constexpr int MC = Geo<DIM>::MC, BLK = Q * MC, W = Meta<DIM>::W;
    static constexpr int BLK_BYTES = BLK * (int)sizeof(T);   // multiple of 16 for every set/type
    static constexpr int META_BYTES = W * 4;                  // 48 / 112
    static constexpr int BPS_RAW = 20480 / BLK_BYTES;
    static constexpr int BPS = BPS_RAW < 1 ? 1 : (BPS_RAW > 64 ? 64 : BPS_RAW);
    static constexpr size_t POP = (size_t)BPS * BLK_BYTES;
    static constexpr size_t STAGE = align_up(POP + (size_t)BPS * META_BYTES + (size_t)BPS * 4, 128);
    static constexpr int NS = STAGE <= 24 * 1024 ? 4 : 3;
    static constexpr size_t BARS = 128;   // 2 * NS mbarriers, padded
    static constexpr size_t SMEM = BARS + NS * STAGE;
    static constexpr int CONSUMERS = 512;   // 16 consumer warps: enough to overlap smem latency
    static constexpr int THREADS = CONSUMERS + 32;
    static_assert(BLK_BYTES % 16 == 0 && META_BYTES % 16 == 0, "bulk copies need 16-byte multiples");
};

template <int DIM, int Q, typename T, bool SOLID>
__global__ void __launch_bounds__(TmaCfg<DIM, Q, T>::THREADS)
k_step_tma(const StepArgs a, int *status)
{
    using Cfg = TmaCfg<DIM, Q, T>;
    using C = typename ST<T>::C;
    constexpr int MC = Cfg::MC, BLK = Cfg::BLK, BPS = Cfg::BPS, NS = Cfg::NS, W = Cfg::W;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + NS;
    unsigned char *stages = smem + Cfg::BARS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nchunks = (a.n + BPS - 1) / BPS;
    const unsigned seed = step_seed(a);   // plain launch: the predecessor has completed

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], Cfg::CONSUMERS);
        }
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == Cfg::CONSUMERS / 32) {
        // ---------------- producer warp ----------------
        // Its only global loads are the block IDs, prefetched one chunk
        // ahead; populations and metadata rows arrive by bulk copy.
        const T *fin = static_cast<const T *>(a.fin);
        int bn[2] = {-1, -1};   // IDs of blocks lane and lane+32 of the next chunk
        auto fetch_ids = [&](int chunk) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int lb = lane + 32 * h;
                const int kap = chunk * BPS + lb;
                bn[h] = (lb < BPS && chunk < nchunks && kap < a.n) ? __ldg(&a.ids[kap]) : -1;
            }
        };
        fetch_ids(blockIdx.x);
        int k = 0;
        for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x, ++k) {
            const int s = k % NS;
            const unsigned ph = (unsigned)(k / NS) & 1u;
            const int b0 = bn[0], b1 = bn[1];
            fetch_ids(chunk + gridDim.x);
            if (!mbar_wait(&empty[s], ph ^ 1u, status)) break;
            unsigned char *st = stages + (size_t)s * Cfg::STAGE;
            T *pop = reinterpret_cast<T *>(st);
            int *meta = reinterpret_cast<int *>(st + Cfg::POP);
            int *blk = meta + BPS * W;
            if (lane < BPS) blk[lane] = b0;
            if (lane + 32 < BPS) blk[lane + 32] = b1;
            int valid = (b0 >= 0) + (b1 >= 0);
            for (int off = 16; off > 0; off >>= 1) valid += __shfl_xor_sync(0xffffffffu, valid, off);
            __syncwarp();
            if (lane == 0) mbar_arrive_expect_tx(&full[s], (unsigned)(valid * (Cfg::BLK_BYTES + Cfg::META_BYTES)));
            __syncwarp();
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int lb = lane + 32 * h;
                const int b = h ? b1 : b0;
                if (lb < BPS && b >= 0) {
                    bulk_g2s(pop + (size_t)lb * BLK, fin + (long long)b * BLK, Cfg::BLK_BYTES, &full[s]);
                    bulk_g2s(meta + lb * W, a.meta + (long long)b * W, Cfg::META_BYTES, &full[s]);
                }
            }
        }
        // Drain: the last phase armed on each stage must complete before exit.
        if (lane == 0) {
            for (int s = 0; s < NS && s < k; s++) {
                const int last = k - 1 - ((k - 1 - s) % NS);   // last chunk index using stage s
                mbar_wait(&full[s], (unsigned)(last / NS) & 1u, status);
            }
        }
    } else {
        // ---------------- consumer warps ----------------
        T *__restrict__ fo = static_cast<T *>(a.fout);
        int k = 0;
        for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x, ++k) {
            const int s = k % NS;
            const unsigned ph = (unsigned)(k / NS) & 1u;
            if (!mbar_wait(&full[s], ph, status)) break;
            const unsigned char *st = stages + (size_t)s * Cfg::STAGE;
            const T *pop = reinterpret_cast<const T *>(st);
            const int *meta = reinterpret_cast<const int *>(st + Cfg::POP);
            const int *blk = meta + BPS * W;
            for (int c = threadIdx.x; c < BPS * MC; c += Cfg::CONSUMERS) {
                const int lb = c / MC, t = c % MC;
                const int b = blk[lb];
                if (b < 0) continue;
                const int *row = meta + lb * W;
                const int fl = row[Meta<DIM>::FLAGS];
                if (fl & META_WALL) continue;
                // Solid cells and inactive blocks are left untouched by the
                // reference's in-place step: carry them over unchanged.
                if (SOLID && (!(fl & META_ACTIVE) || __ldg(&a.cmask[(long long)b * MC + t]) == CELL_SOLID)) {
#pragma unroll
                    for (int sl = 0; sl < Q; sl++)
                        fo[(long long)b * BLK + sl * MC + t] = pop[(size_t)lb * BLK + sl * MC + t];
                    continue;
                }
                if (!(fl & META_ACTIVE)) continue;
                C g[Q];
#pragma unroll
                for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(pop[(size_t)lb * BLK + lat_pb(DIM, p) * MC + t]);
                C ux, uy, uz;
                collide_cell<DIM, Q, T>(g, a, ux, uy, uz);
                const bool hook = (fl & META_ONB) && a.bc_preset != AGAL_BC_NONE;
                push_cell<DIM, Q, T, SOLID>(g, ux, uy, uz, b, t, row, hook, fo, a, seed);
            }
            mbar_arrive(&empty[s]);
        }
    }
}

// Kernel attributes and persistent grid size, set once per instantiation
// (outside any stream capture: agal_set_tuning / agal_autotune call it).
template <int DIM, int Q, typename T, bool SOLID> struct TmaLaunch {
    static inline int ctas_per_sm = -1;
    static inline int sms = 0;
    static int prepare(agal_ctx *c)
    {
        using Cfg = TmaCfg<DIM, Q, T>;
        if (ctas_per_sm >= 0) return AGAL_OK;
        AGAL_CUDA(c, cudaFuncSetAttribute(k_step_tma<DIM, Q, T, SOLID>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)Cfg::SMEM));
        int n = 0;
        AGAL_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step_tma<DIM, Q, T, SOLID>, Cfg::THREADS,
                                                                   Cfg::SMEM));
        AGAL_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device));
        ctas_per_sm = n > 0 ? n : 1;
        return AGAL_OK;
    }
};

template <int DIM, int Q, typename T, bool SOLID>
int launch_step_tma_t(agal_ctx *c, const StepArgs &a)
{
    using Cfg = TmaCfg<DIM, Q, T>;
    using Ln = TmaLaunch<DIM, Q, T, SOLID>;
    int rc = Ln::prepare(c);
    if (rc) return rc;
    const int sms = Ln::sms, ctas_per_sm = Ln::ctas_per_sm;
    const int nchunks = (a.n + Cfg::BPS - 1) / Cfg::BPS;
    const int grid = nchunks < sms * ctas_per_sm ? nchunks : sms * ctas_per_sm;
    if (grid <= 0) return AGAL_OK;
    k_step_tma<DIM, Q, T, SOLID><<<grid, Cfg::THREADS, Cfg::SMEM, c->stream>>>(a, c->d_status);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

template <int DIM, int Q, typename T>
int launch_step_tma(agal_ctx *c, const StepArgs &a)
{
    return c->geometry_init ? launch_step_tma_t<DIM, Q, T, true>(c, a) : launch_step_tma_t<DIM, Q, T, false>(c, a);
}

template <int DIM, int Q, typename T>
int prepare_step_tma(agal_ctx *c)
{
    int rc = TmaLaunch<DIM, Q, T, false>::prepare(c);
    return rc ? rc : TmaLaunch<DIM, Q, T, true>::prepare(c);
}

#define AGAL_TMA_INST(D, Q, T)                                                     \
    template int launch_step_tma<D, Q, T>(agal_ctx *, const StepArgs &); \
    template int prepare_step_tma<D, Q, T>(agal_ctx *);
AGAL_TMA_INST(2, 9, float)
AGAL_TMA_INST(2, 9, double)
AGAL_TMA_INST(2, 9, __half)
AGAL_TMA_INST(2, 9, __nv_bfloat16)
AGAL_TMA_INST(3, 19, float)
AGAL_TMA_INST(3, 19, double)
AGAL_TMA_INST(3, 19, __half)
AGAL_TMA_INST(3, 19, __nv_bfloat16)
AGAL_TMA_INST(3, 27, float)
AGAL_TMA_INST(3, 27, double)
AGAL_TMA_INST(3, 27, __half)
AGAL_TMA_INST(3, 27, __nv_bfloat16)

}  // namespace agal
