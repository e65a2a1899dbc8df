// BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor cores (tcgen05).
//
//   D[M x N] = A[M x K] . B[N x K]^T        (A, B row-major, K contiguous)
//
// One CTA of 128 threads per 128-row tile of D and K slice, N <= 32 (one
// 128 x 32 FP32 accumulator in tensor memory, 32 columns).  K is walked in
// chunks of KC through two shared-memory stages: the four warps copy chunk
// k+1 of B with cp.async, and stage chunk k+1 of A through a loader functor
// (a row-major matrix with cp.async, or an implicit-GEMM gather that builds
// the columns from another array) (16 bytes per copy, rows past M or N
// zero-filled) into the tensor core's no-swizzle K-major
// layout (8-row x 16-byte core matrices; K-adjacent core matrices 128 B
// apart, 8-row groups KC x 2 B apart) while the tensor core multiplies chunk
// k; one thread issues KC/16 tcgen05.mma (kind::f16, M = 128, N = 32, K = 16)
// per chunk and commits them to the stage's mbarrier, whose completion frees
// the stage.  After the last chunk each warp reads its 32 accumulator lanes
// with tcgen05.ld and stores (one K slice) or atomically adds (split K) its
// rows of D.  Every mbarrier wait is bounded (2 s of %globaltimer): on expiry
// the status word gets AGAL_ERR_TIMEOUT, the tile is skipped, and the tensor
// memory is still freed.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../include/agal_b200.h"

namespace agal {
namespace umma {

constexpr int TM = 128;          // rows per CTA (tcgen05 M)
constexpr int TN = 32;           // accumulator columns (tcgen05 N)
constexpr int KC = 128;          // K elements per shared-memory chunk
constexpr int THREADS = 128;
constexpr size_t STAGE = (size_t)(TM + TN) * KC * 2;  // 40 KB
constexpr size_t SMEM = 2 * STAGE;                     // two stages
constexpr unsigned long long kWaitNs = 2000000000ull;

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity)
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

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *status)
{
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_try(bar, parity)) {
        if (now_ns() - t0 > kWaitNs) {
            atomicExch(status, AGAL_ERR_TIMEOUT);
            return false;
        }
    }
    return true;
}

// Shared-memory matrix descriptor, no swizzle, K-major (tcgen05 format:
// start >> 4 in bits 0-13, leading byte offset >> 4 in 16-29, stride byte
// offset >> 4 in 32-45, version 1 in bits 46-47, layout 0 in bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(const void *p, unsigned lbo_bytes, unsigned sbo_bytes)
{
    const uint64_t a = (smem_u32(p) >> 4) & 0x3FFFu;
    const uint64_t l = (lbo_bytes >> 4) & 0x3FFFu;
    const uint64_t s = (sbo_bytes >> 4) & 0x3FFFu;
    return a | (l << 16) | (s << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9, 10-12 = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in
// bits 24-28.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Byte offset of element (row r, k) of a chunk in the core-matrix layout.
__device__ __forceinline__ unsigned core_off(int r, int kg)
{
    // kg = k / 8 (one 16-byte row of a core matrix)
    return (unsigned)(((r >> 3) * (KC / 8) + kg) * 128 + (r & 7) * 16);
}

__device__ __forceinline__ void cp_async16(unsigned dst, const void *src, bool valid)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// A operand staged from a row-major BF16 matrix [M][K] with cp.async.
struct DenseA {
    const __nv_bfloat16 *A;
    int M, K;
    // Chunk of columns [kc, kc + 8 g8) of rows m0.. into the stage sA.
    __device__ void operator()(unsigned char *sA, int m0, int kc, int g8, int tid) const
    {
        for (int i = tid; i < TM * g8; i += THREADS) {
            const int r = i / g8, kg = i % g8;
            const bool ok = m0 + r < M;
            cp_async16(smem_u32(sA + core_off(r, kg)), A + (size_t)(ok ? m0 + r : 0) * K + kc + kg * 8, ok);
        }
    }
};

template <class ALoad>
__global__ void __launch_bounds__(THREADS) k_gemm_bf16(const ALoad aload, const __nv_bfloat16 *__restrict__ B,
                                                       float *__restrict__ D, int M, int N, int K, int ldd,
                                                       int kslice, int *status)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t s_taddr;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TM;
    const int k_begin = blockIdx.y * kslice, k_end = min(K, k_begin + kslice);
    const int nchunks = (k_end - k_begin + KC - 1) / KC;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_taddr)),
                     "r"(TN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < 2; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[s])), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = s_taddr;

    // cp.async copies of chunk c into stage c & 1 (rows past M / N zero-filled)
    auto load = [&](int c) {
        unsigned char *sA = smem + (size_t)(c & 1) * STAGE;
        unsigned char *sB = sA + (size_t)TM * KC * 2;
        const int kc = k_begin + c * KC;
        const int g8 = min(KC, k_end - kc) / 8;
        aload(sA, m0, kc, g8, tid);
        for (int i = tid; i < TN * g8; i += THREADS) {
            const int r = i / g8, kg = i % g8;
            const bool ok = r < N;
            cp_async16(smem_u32(sB + core_off(r, kg)), B + (size_t)(ok ? r : 0) * K + kc + kg * 8, ok);
        }
        cp_async_commit();
    };

    bool ok = true;
    if (nchunks > 0) load(0);
    for (int it = 0; it < nchunks; it++) {
        // the stage chunk it+1 goes to was read by the MMAs of chunk it-1
        if (it >= 1) ok = mbar_wait_bounded(&mbar[(it - 1) & 1], (unsigned)(((it - 1) >> 1) & 1), status) && ok;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        if (it + 1 < nchunks) {
            load(it + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned char *sA = smem + (size_t)(it & 1) * STAGE;
            const unsigned char *sB = sA + (size_t)TM * KC * 2;
            const int kw = min(KC, k_end - (k_begin + it * KC));   // multiple of 16
            for (int s = 0; s < kw / 16; s++) {
                const uint64_t ad = smem_desc(sA + s * 256, 128, KC * 16);
                const uint64_t bd = smem_desc(sB + s * 256, 128, KC * 16);
                const uint32_t acc = (it > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(taddr), "l"(ad), "l"(bd), "r"(IDESC), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mbar[it & 1]))
                         : "memory");
        }
    }
    cp_async_wait<0>();   // nothing left in flight on an early exit
    if (ok && nchunks > 0)
        ok = mbar_wait_bounded(&mbar[(nchunks - 1) & 1], (unsigned)(((nchunks - 1) >> 1) & 1), status);
    tc_fence_after();
    ok = __syncthreads_and(ok);

    if (ok && nchunks > 0) {
        uint32_t v[32];
        const uint32_t src = taddr + ((uint32_t)(warp * 32) << 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
            "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
              "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
              "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
            : "r"(src)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int row = m0 + warp * 32 + lane;
        if (row < M) {
            if (gridDim.y == 1) {
#pragma unroll
                for (int j = 0; j < TN; j++)
                    if (j < N) D[(size_t)row * ldd + j] = __uint_as_float(v[j]);
            } else {
#pragma unroll
                for (int j = 0; j < TN; j++)
                    if (j < N) atomicAdd(&D[(size_t)row * ldd + j], __uint_as_float(v[j]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(TN) : "memory");
}

// D = A . B^T for M rows (any), N <= 32, K a multiple of 16, the A operand
// staged by aload (DenseA: a row-major matrix; or an implicit-GEMM gather that
// builds the columns in shared memory).  A long K with few row tiles is split
// over CTAs (K slices of a multiple of KC) whose partial tiles are added
// atomically into D, which is zeroed first; that needs ldd == N (D contiguous).
template <class ALoad>
inline cudaError_t gemm_bf16_with(const ALoad &aload, const __nv_bfloat16 *B, float *D, int M, int N, int K, int ldd,
                                  int *status, cudaStream_t s)
{
    if (M <= 0) return cudaSuccess;
    if (N < 1 || N > TN || K <= 0 || K % 16) return cudaErrorInvalidValue;
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || !attr[dev]) {
        const cudaError_t e =
            cudaFuncSetAttribute(k_gemm_bf16<ALoad>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attr[dev] = true;
    }
    const int mt = (M + TM - 1) / TM;
    int splits = 1;
    if (ldd == N && mt < 148 && K > 4 * KC) splits = std::min((K + 4 * KC - 1) / (4 * KC), std::max(1, 296 / mt));
    const int kslice = ((K + splits - 1) / splits + KC - 1) / KC * KC;
    splits = (K + kslice - 1) / kslice;
    if (splits > 1) {
        const cudaError_t e = cudaMemsetAsync(D, 0, sizeof(float) * (size_t)M * ldd, s);
        if (e != cudaSuccess) return e;
    }
    k_gemm_bf16<ALoad><<<dim3((unsigned)mt, (unsigned)splits), THREADS, SMEM, s>>>(aload, B, D, M, N, K, ldd, kslice,
                                                                                   status);
    return cudaGetLastError();
}

inline cudaError_t gemm_bf16(const __nv_bfloat16 *A, const __nv_bfloat16 *B, float *D, int M, int N, int K, int ldd,
                             int *status, cudaStream_t s)
{
    return gemm_bf16_with(DenseA{A, M, K}, B, D, M, N, K, ldd, status, s);
}

}  // namespace umma
}  // namespace agal
