// Run Fn<DIM, Q, storage type>::run(c, args...) for the context's velocity
// set and population storage.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "ctx.h"

namespace agal {

template <template <int, int, typename> class Fn, typename... Args>
int dispatch(agal_ctx *c, Args... args)
{
    switch (c->Q) {
    case 9:
        switch (c->storage) {
        case AGAL_STORE_FP32: return Fn<2, 9, float>::run(c, args...);
        case AGAL_STORE_FP64: return Fn<2, 9, double>::run(c, args...);
        case AGAL_STORE_FP16: return Fn<2, 9, __half>::run(c, args...);
        case AGAL_STORE_BF16: return Fn<2, 9, __nv_bfloat16>::run(c, args...);
        }
        break;
    case 19:
        switch (c->storage) {
        case AGAL_STORE_FP32: return Fn<3, 19, float>::run(c, args...);
        case AGAL_STORE_FP64: return Fn<3, 19, double>::run(c, args...);
        case AGAL_STORE_FP16: return Fn<3, 19, __half>::run(c, args...);
        case AGAL_STORE_BF16: return Fn<3, 19, __nv_bfloat16>::run(c, args...);
        }
        break;
    case 27:
        switch (c->storage) {
        case AGAL_STORE_FP32: return Fn<3, 27, float>::run(c, args...);
        case AGAL_STORE_FP64: return Fn<3, 27, double>::run(c, args...);
        case AGAL_STORE_FP16: return Fn<3, 27, __half>::run(c, args...);
        case AGAL_STORE_BF16: return Fn<3, 27, __nv_bfloat16>::run(c, args...);
        }
        break;
    }
    return agal_set_err(c, AGAL_ERR_UNSUPPORTED, "velocity set / storage combination not built");
}

}  // namespace agal
