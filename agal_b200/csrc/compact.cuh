// Ordered (stable) stream compaction on the device.
//
// Each CTA takes a contiguous chunk of SCAN_T x SCAN_I indices and counts its
// flagged ones; the per-CTA counts are scanned in one CTA; a second pass
// emits every flagged index with its rank, warp-shuffle scans keeping index
// order.  Used by the refine/coarsen pass (block-ID ordered lists, as
// thrust::copy_if produces them) and by the geometry set-up (ray-filtered
// faces, wall-block slots).
#pragma once

#include <cuda_runtime.h>

namespace agal {
namespace cmp {
namespace {   // internal linkage: one copy per translation unit

constexpr int SCAN_T = 512;
constexpr int SCAN_I = 8;
constexpr int SCAN_CHUNK = SCAN_T * SCAN_I;

// Number of per-CTA partial counts a compaction over n indices needs.
inline int parts_for(long long n) { return (int)((n + SCAN_CHUNK - 1) / SCAN_CHUNK); }

// Exclusive CTA-wide scan of v (SCAN_T threads); *total receives the sum.
__device__ __forceinline__ int cta_exscan(int v, int *s_warp, int *total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = (lane < SCAN_T / 32) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_T / 32) s_warp[lane] = w;
    }
    __syncthreads();
    *total = s_warp[SCAN_T / 32 - 1];
    return (wid ? s_warp[wid - 1] : 0) + x - v;
}

template <class F>
__global__ void __launch_bounds__(SCAN_T) k_cmp_count(const F f, int n, int *parts)
{
    __shared__ int s_warp[SCAN_T / 32];
    const long long base = (long long)blockIdx.x * SCAN_CHUNK + (long long)threadIdx.x * SCAN_I;
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; k++) {
        const long long i = base + k;
        if (i < n && f.pred((int)i)) cnt++;
    }
    int total;
    cta_exscan(cnt, s_warp, &total);
    if (threadIdx.x == 0) parts[blockIdx.x] = total;
}

// Exclusive scan of the per-CTA counts in one CTA; total into *out.
__global__ void __launch_bounds__(SCAN_T) k_cmp_scan(int *parts, int np, int *out)
{
    __shared__ int s_warp[SCAN_T / 32];
    int carry = 0;
    for (int base = 0; base < np; base += SCAN_T) {
        const int i = base + threadIdx.x;
        const int v = (i < np) ? parts[i] : 0;
        int total;
        const int ex = cta_exscan(v, s_warp, &total);
        if (i < np) parts[i] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = carry;
}

template <class F>
__global__ void __launch_bounds__(SCAN_T) k_cmp_emit(const F f, int n, const int *parts)
{
    __shared__ int s_warp[SCAN_T / 32];
    const long long base = (long long)blockIdx.x * SCAN_CHUNK + (long long)threadIdx.x * SCAN_I;
    bool fl[SCAN_I];
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < SCAN_I; k++) {
        const long long i = base + k;
        fl[k] = i < n && f.pred((int)i);
        cnt += fl[k];
    }
    int total;
    int r = parts[blockIdx.x] + cta_exscan(cnt, s_warp, &total);
#pragma unroll
    for (int k = 0; k < SCAN_I; k++)
        if (fl[k]) f.emit((int)(base + k), r++);
}

// Ordered compaction over [0, n): f.emit(i, rank) for every i with f.pred(i),
// the count into *d_total (device).  parts holds parts_for(n) ints.  The
// predicate must not read what emit writes.  Asynchronous on stream s.
template <class F>
cudaError_t compact_async(cudaStream_t s, int *parts, int *d_total, const F &f, int n)
{
    if (n <= 0) return cudaMemsetAsync(d_total, 0, sizeof(int), s);
    const int np = parts_for(n);
    k_cmp_count<F><<<np, SCAN_T, 0, s>>>(f, n, parts);
    k_cmp_scan<<<1, SCAN_T, 0, s>>>(parts, np, d_total);
    k_cmp_emit<F><<<np, SCAN_T, 0, s>>>(f, n, parts);
    return cudaGetLastError();
}

}  // namespace
}  // namespace cmp
}  // namespace agal
