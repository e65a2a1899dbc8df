// Population storage types.
//
// FP32 and FP64 store f_p as is.  FP16 and BF16 store the offset
// g_p = f_p - w_p from the lattice weight (rho = 1, u = 0 gives g = 0), which
// keeps the stored magnitude at O(|u|) and the relative rounding error of
// half precision small; arithmetic is done in FP32 on g.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

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
template <> struct ST<__half> {
    using C = float;
    static constexpr bool OFF = true;
    __host__ __device__ static C dec(__half v) { return __half2float(v); }
    __host__ __device__ static __half enc(C v) { return __float2half_rn(v); }
};
template <> struct ST<__nv_bfloat16> {
    using C = float;
    static constexpr bool OFF = true;
    __host__ __device__ static C dec(__nv_bfloat16 v) { return __bfloat162float(v); }
    __host__ __device__ static __nv_bfloat16 enc(C v) { return __float2bfloat16_rn(v); }
};

}  // namespace agal
