// Population storage types.
//
// FP32 and FP64 store f_p as is.  FP16 and BF16 store the offset
// g_p = f_p - w_p from the lattice weight (rho = 1, u = 0 gives g = 0), which
// keeps the stored magnitude at O(|u|) and the relative rounding error of
// half precision small; arithmetic is done in FP32 on g.  FP16 stores
// g * 2^10 (below).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

namespace agal {

template <typename T> struct ST;
template <> struct ST<float> {
    using C = float;
    static constexpr bool OFF = false;
    __host__ __device__ static C dec(float v) { return v; }
    __host__ __device__ static float enc(C v) { return v; }
};
template <> struct ST<double> {
    using C = double;
    static constexpr bool OFF = false;
    __host__ __device__ static C dec(double v) { return v; }
    __host__ __device__ static double enc(C v) { return v; }
};
// FP16 offsets are stored times kHalfScale = 2^10 (exact either way): the
// offsets of a flow with |u| <= 0.1 lie within about 1e-7..1e-1, which then
// falls in FP16's normal range (2^-14..65504) with its full 11-bit precision
// instead of the fixed 2^-24 spacing of its subnormals.
constexpr float kHalfScale = 1024.0f;
constexpr float kHalfUnscale = 1.0f / 1024.0f;
template <> struct ST<__half> {
    using C = float;
    static constexpr bool OFF = true;
    __host__ __device__ static C dec(__half v) { return __half2float(v) * kHalfUnscale; }
    __host__ __device__ static __half enc(C v) { return __float2half_rn(v * kHalfScale); }
};
template <> struct ST<__nv_bfloat16> {
    using C = float;
    static constexpr bool OFF = true;
    __host__ __device__ static C dec(__nv_bfloat16 v) { return __bfloat162float(v); }
    __host__ __device__ static __nv_bfloat16 enc(C v) { return __float2bfloat16_rn(v); }
};

// Stochastic rounding of the half-precision offsets (agal_params
// half_rounding).  Adding a uniform random integer below the target format's
// last mantissa bit to the FP32 bit pattern and truncating those bits rounds
// the magnitude up with probability equal to the discarded fraction (sign and
// magnitude are separate, so the value stays unbiased; a carry into the
// exponent gives the next binade, the right upper neighbour).  The result is
// exactly representable, so the final conversion does not round again.  FP16
// offsets are stored scaled by kHalfScale, which keeps them in FP16's normal
// range, where the 13 truncated bits are the whole difference.
//
// Random bits: one hash per cell (its element index in the pool and the
// launch seed), times an odd constant per direction.
__device__ __forceinline__ unsigned sr_cell(long long cell, unsigned seed)
{
    unsigned x = (unsigned)cell * 0x9E3779B1u + seed;
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}
__host__ __device__ constexpr unsigned sr_dir(int p) { return 0x9E3779B9u * (2u * (unsigned)p + 1u); }

// Encode a computed value for storage: stochastic rounding for the half
// types when sr is set (rnd: 32 random bits), the plain conversion otherwise.
template <typename T>
__device__ __forceinline__ T enc_r(typename ST<T>::C v, unsigned rnd, bool sr)
{
    if constexpr (std::is_same<T, __half>::value) {
        if (!sr) return ST<T>::enc(v);
        const unsigned u = (__float_as_uint(v * kHalfScale) + (rnd >> 19)) & ~0x1FFFu;
        return __float2half_rn(__uint_as_float(u));
    } else if constexpr (std::is_same<T, __nv_bfloat16>::value) {
        if (!sr) return ST<T>::enc(v);
        const unsigned u = (__float_as_uint(v) + (rnd >> 16)) & 0xFFFF0000u;
        return __float2bfloat16_rn(__uint_as_float(u));
    } else {
        return ST<T>::enc(v);
    }
}

}  // namespace agal
