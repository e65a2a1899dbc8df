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
#include "step_common.cuh"
#include "storage.cuh"

namespace agal {
namespace {

constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *status)
{
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (true) {
        if (mbar_test(bar, parity)) return true;
        if (now_ns() - t0 > kWaitNs) {
            atomicExch(status, AGAL_ERR_TIMEOUT);
            return false;
        }
    }
}

// 1-D bulk copy global -> shared, completion counted on bar (no multicast).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

constexpr size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

}  // namespace

// Stage geometry: ~18-28 KB of populations per stage, 3 or 4 stages.
template <int DIM, int Q, typename T> struct TmaCfg {
    static constexpr int MC = Geo<DIM>::MC, QMAX = Geo<DIM>::QMAX, BLK = Q * MC;
    static constexpr int BLK_BYTES = BLK * (int)sizeof(T);   // multiple of 16 for every set/type
    static constexpr int BPS = (20480 / BLK_BYTES) > 0 ? (20480 / BLK_BYTES) : 1;
    static constexpr size_t POP = (size_t)BPS * BLK_BYTES;
    static constexpr size_t STAGE = align_up(POP + (size_t)BPS * QMAX * 4 + (size_t)BPS * 8, 128);
    static constexpr int NS = STAGE <= 24 * 1024 ? 4 : 3;
    static constexpr size_t BARS = 128;   // 2 * NS mbarriers, padded
    static constexpr size_t SMEM = BARS + NS * STAGE;
    static constexpr int CONSUMERS = 256;
    static constexpr int THREADS = CONSUMERS + 32;
    static_assert(BLK_BYTES % 16 == 0, "bulk copies need 16-byte multiples");
};

template <int DIM, int Q, typename T, bool SOLID>
__global__ void __launch_bounds__(TmaCfg<DIM, Q, T>::THREADS)
k_step_tma(const StepArgs a, int *status)
{
    using Cfg = TmaCfg<DIM, Q, T>;
    using C = typename ST<T>::C;
    constexpr int MC = Cfg::MC, QMAX = Cfg::QMAX, BLK = Cfg::BLK, BPS = Cfg::BPS, NS = Cfg::NS;
    constexpr int CENTER = center_slot(DIM);
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + NS;
    unsigned char *stages = smem + Cfg::BARS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nchunks = (a.n + BPS - 1) / BPS;

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
        const T *fin = static_cast<const T *>(a.fin);
        int k = 0;
        for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x, ++k) {
            const int s = k % NS;
            const unsigned ph = (unsigned)(k / NS) & 1u;
            if (!mbar_wait(&empty[s], ph ^ 1u, status)) break;
            unsigned char *st = stages + (size_t)s * Cfg::STAGE;
            T *pop = reinterpret_cast<T *>(st);
            int *nbr = reinterpret_cast<int *>(st + Cfg::POP);
            int *blk = nbr + BPS * QMAX;
            int *flg = blk + BPS;
            int valid = 0;
            for (int lb = lane; lb < BPS; lb += 32) {
                const int kap = chunk * BPS + lb;
                const int b = (kap < a.n) ? __ldg(&a.ids[kap]) : -1;
                int fl = 0;
                if (b >= 0) {
                    if (__ldg(&a.nbr_child[b]) < 0 || __ldg(&a.bmask[b]) != BLOCK_SOLID) fl |= 1;   // kernels.cu:236
                    if (__ldg(&a.onb[b]) == 1) fl |= 2;                                             // kernels.cu:736
                }
                blk[lb] = b;
                flg[lb] = fl;
                valid += (b >= 0);
            }
            for (int off = 16; off > 0; off >>= 1) valid += __shfl_xor_sync(0xffffffffu, valid, off);
            __syncwarp();
            for (int i = lane; i < BPS * QMAX; i += 32) {
                const int lb = i % BPS, S = i / BPS;
                const int b = blk[lb];
                int v = b;   // the centre slot is the block itself
                if (S != CENTER) {
                    const int m = __ldg((DIM == 2) ? &g_map2[S] : &g_map3[S]);
                    v = (b >= 0) ? __ldg(&a.nbr[b + (long long)m * a.nmb]) : N_SKIPID;
                }
                nbr[lb * QMAX + S] = v;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive_expect_tx(&full[s], (unsigned)(valid * Cfg::BLK_BYTES));
            __syncwarp();
            for (int lb = lane; lb < BPS; lb += 32) {
                const int b = blk[lb];
                if (b >= 0) bulk_g2s(pop + (size_t)lb * BLK, fin + (long long)b * BLK, Cfg::BLK_BYTES, &full[s]);
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
        const C omeg = C(a.omega);
        int k = 0;
        for (int chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x, ++k) {
            const int s = k % NS;
            const unsigned ph = (unsigned)(k / NS) & 1u;
            if (!mbar_wait(&full[s], ph, status)) break;
            const unsigned char *st = stages + (size_t)s * Cfg::STAGE;
            const T *pop = reinterpret_cast<const T *>(st);
            const int *nbr = reinterpret_cast<const int *>(st + Cfg::POP);
            const int *blk = nbr + BPS * QMAX;
            const int *flg = blk + BPS;
            for (int c = threadIdx.x; c < BPS * MC; c += Cfg::CONSUMERS) {
                const int lb = c / MC, t = c % MC;
                const int b = blk[lb], fl = flg[lb];
                if (b < 0 || !(fl & 1)) continue;
                if (SOLID && __ldg(&a.cmask[(long long)b * MC + t]) == CELL_SOLID) continue;
                C g[Q];
#pragma unroll
                for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(pop[(size_t)lb * BLK + lat_pb(DIM, p) * MC + t]);
                C ux, uy, uz;
                bgk_collide<DIM, Q, C, ST<T>::OFF>(g, omeg, ux, uy, uz);
                const bool hook = (fl & 2) && a.bc_preset != AGAL_BC_NONE;
                push_cell<DIM, Q, T, SOLID>(g, ux, uy, uz, b, t, nbr + lb * QMAX, hook, fo, a);
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
