// Population transfers between the device's block-major storage and the
// reference's slot-major FP64 layout (cells_f_F[s][b * M_CBLOCK + c], absolute
// values; mesh.h:379), converted on the device.
//
// A kernel decodes (or encodes) a chunk of blocks into a fixed device staging
// buffer, and one strided copy (cudaMemcpy2DAsync, rows = slots) moves the
// chunk to or from the caller's host array, so a dump or load costs the PCIe
// transfer of the FP64 array and no host-side loop.  Each block is read from
// the buffer its level currently steps in (cur[level]); loads write both
// buffers.
#include <cuda_runtime.h>

#include <algorithm>

#include "ctx.h"
#include "dispatch.cuh"
#include "lattice.cuh"
#include "storage.cuh"

namespace agal {
namespace {

constexpr long long kStageDoubles = 8ll << 20;   // 64 MiB of staging

struct XferArgs {
    const void *F0, *F1;
    void *W0, *W1;
    const int *lev, *ref;
    unsigned cur_mask;   // bit L = buffer of level L
    int max_levels;
    long long b0, ncell;
    int Q, MC, dim;
    double *stage;       // [Q][ncell]
};

template <typename T>
__global__ void k_f_to_ref(const XferArgs a)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)a.Q * a.ncell) return;
    const int s = (int)(g / a.ncell);
    const long long cell = g - (long long)s * a.ncell;
    const long long b = a.b0 + cell / a.MC;
    const int lv = a.lev[b];
    const int L = (a.ref[b] != REF_INACTIVE && lv >= 0 && lv < a.max_levels) ? lv : 0;
    const T *F = static_cast<const T *>(((a.cur_mask >> L) & 1u) ? a.F1 : a.F0);
    const T v = F[(b * a.Q + s) * a.MC + cell % a.MC];
    // slot s holds f_{pb(s)}, and w_{pb(s)} == w_s
    a.stage[g] = (double)ST<T>::dec(v) + (ST<T>::OFF ? lat_w(a.Q, s) : 0.0);
}

template <typename T>
__global__ void k_ref_to_f(const XferArgs a)
{
    using C = typename ST<T>::C;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)a.Q * a.ncell) return;
    const int s = (int)(g / a.ncell);
    const long long cell = g - (long long)s * a.ncell;
    const long long b = a.b0 + cell / a.MC;
    const T v = ST<T>::enc((C)(a.stage[g] - (ST<T>::OFF ? lat_w(a.Q, s) : 0.0)));
    const long long dst = (b * a.Q + s) * a.MC + cell % a.MC;
    static_cast<T *>(a.W0)[dst] = v;
    static_cast<T *>(a.W1)[dst] = v;
}

int stage_buffer(agal_ctx *c, long long *chunk_blocks)
{
    if (!c->xfer) AGAL_CUDA(c, cudaMalloc(&c->xfer, sizeof(double) * (size_t)kStageDoubles));
    *chunk_blocks = std::max(1ll, kStageDoubles / ((long long)c->Q * c->MC));
    return AGAL_OK;
}

template <int DIM, int Q, typename T> struct RunToHost {
    // blocks [0, nb) -> host[s * pitch + b * MC + c]
    static int run(agal_ctx *c, long long nb, long long pitch, double *host)
    {
        long long chunk = 0;
        int rc = stage_buffer(c, &chunk);
        if (rc) return rc;
        XferArgs a{};
        a.F0 = c->F[0];
        a.F1 = c->F[1];
        a.lev = c->cblock_level;
        a.ref = c->cblock_ID_ref;
        for (int L = 0; L < c->max_levels && L < 32; L++) a.cur_mask |= (unsigned)(c->cur[L] & 1) << L;
        a.max_levels = c->max_levels;
        a.Q = Q;
        a.MC = Geo<DIM>::MC;
        a.dim = DIM;
        a.stage = static_cast<double *>(c->xfer);
        for (long long b0 = 0; b0 < nb; b0 += chunk) {
            a.b0 = b0;
            a.ncell = std::min(chunk, nb - b0) * a.MC;
            const long long tot = (long long)Q * a.ncell;
            k_f_to_ref<T><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(a);
            AGAL_CUDA(c, cudaGetLastError());
            AGAL_CUDA(c, cudaMemcpy2DAsync(host + b0 * a.MC, sizeof(double) * (size_t)pitch, a.stage,
                                           sizeof(double) * (size_t)a.ncell, sizeof(double) * (size_t)a.ncell, Q,
                                           cudaMemcpyDeviceToHost, c->stream));
        }
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
        return AGAL_OK;
    }
};

template <int DIM, int Q, typename T> struct RunFromHost {
    // host[s * pitch + b * MC + c] -> blocks [0, nb) of both buffers
    static int run(agal_ctx *c, long long nb, long long pitch, const double *host)
    {
        long long chunk = 0;
        int rc = stage_buffer(c, &chunk);
        if (rc) return rc;
        XferArgs a{};
        a.W0 = c->F[0];
        a.W1 = c->F[1];
        a.Q = Q;
        a.MC = Geo<DIM>::MC;
        a.dim = DIM;
        a.stage = static_cast<double *>(c->xfer);
        for (long long b0 = 0; b0 < nb; b0 += chunk) {
            a.b0 = b0;
            a.ncell = std::min(chunk, nb - b0) * a.MC;
            AGAL_CUDA(c, cudaMemcpy2DAsync(a.stage, sizeof(double) * (size_t)a.ncell, host + b0 * a.MC,
                                           sizeof(double) * (size_t)pitch, sizeof(double) * (size_t)a.ncell, Q,
                                           cudaMemcpyHostToDevice, c->stream));
            const long long tot = (long long)Q * a.ncell;
            k_ref_to_f<T><<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(a);
            AGAL_CUDA(c, cudaGetLastError());
        }
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
        return AGAL_OK;
    }
};

}  // namespace
}  // namespace agal

int agal_f_to_host(agal_ctx *c, long long nb, long long pitch, double *host)
{
    return agal::dispatch<agal::RunToHost>(c, nb, pitch, host);
}

int agal_f_from_host(agal_ctx *c, long long nb, long long pitch, const double *host)
{
    return agal::dispatch<agal::RunFromHost>(c, nb, pitch, host);
}
