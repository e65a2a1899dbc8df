// Learned refinement predictor: a small convolutional network over per-block
// fields that predicts the refine / coarsen marks of the next regrid, trained
// on the GPU on snapshots labelled by the plain criterion (no reference
// counterpart: the reference has the plain vorticity / Q criterion only).
//
// Network, per block of P = 4^d cells, zero padding at the block faces:
//   x0 [P x 8]  channels (rho - 1)/U^2, u/U, v/U, w/U, 2^L |curl u|/U (per
//               coarse cell), level/(ML-1), refined flag, 1  (U = u_ref)
//   h1 = relu(conv3^d(x0; 8 -> 32) + b1)
//   h2 = relu(conv3^d(h1; 32 -> 32) + b2)
//   z  = mean over cells of conv3^d(h2; 32 -> 2) + b3   (refine, coarsen logits)
// Each convolution is an im2col gather (BF16, column = tap * C + channel) and
// a tcgen05 GEMM with FP32 accumulation (umma_gemm.cuh); the backward pass is
// the same GEMMs on transposed operands plus col2im gathers; Adam updates FP32
// master weights, from which the BF16 copies are taken.  Loss: binary cross
// entropy of both logits against the percentile rule's decisions at the next
// regrid (a leaf block's value above the upper quantile; a block's value
// below the lower one), over the blocks that still exist there, the rare
// positive class weighted.  A block's marks follow from those decisions and
// the rule's admissibility (unrefined and eligible to refine, refined to
// coarsen).
//
// In the solver (S_CRITERION = AGAL_CRITERION_LEARNED, agal_learn_attach) a
// regrid applies the marks the network predicted at the previous regrid;
// every judge_every-th regrid also runs the plain percentile criterion as
// judge, counts the blocks it marks for refinement that the network missed,
// and refines those too.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "ctx.h"
#include "dispatch.cuh"
#include "lattice.cuh"
#include "storage.cuh"
#include "umma_gemm.cuh"

using bf16 = __nv_bfloat16;

namespace agal {
namespace learn {

constexpr int C0 = 8;    // input channels
constexpr int CH = 32;   // hidden channels
constexpr int NO = 2;    // outputs: refine, coarsen

__host__ __device__ constexpr int taps(int dim) { return dim == 2 ? 9 : 27; }
__host__ __device__ constexpr int cells(int dim) { return dim == 2 ? 16 : 64; }
inline int pad16(int x) { return (x + 15) / 16 * 16; }

// Neighbour cell of cell c along tap t inside a 4^d block, -1 outside.
__device__ __forceinline__ int tap_cell(int dim, int c, int t)
{
    const int I = c & 3, J = (c >> 2) & 3, K = (dim == 3) ? (c >> 4) : 0;
    const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = (dim == 3) ? t / 9 - 1 : 0;
    const int i = I + dx, j = J + dy, k = K + dz;
    if (i < 0 || i > 3 || j < 0 || j > 3 || k < 0 || k > 3) return -1;
    return i + 4 * j + 16 * k;
}

// Implicit-GEMM A operand of a convolution: the im2col column block [kc, kc +
// 8 g8) of rows m0.. built directly in the GEMM's shared-memory stage from
// the layer input H [rows][cin] (FP32): each 16-byte core-matrix row is 8
// channels of one tap of one cell, i.e. 32 contiguous bytes of H, converted
// to BF16 as k_im2col converts them (zero outside the block and past the
// taps), so the product is the same bit for bit without the columns ever
// reaching global memory.
struct GatherA {
    const float *H;
    int M, cin, dim, P, ntaps;
    __device__ void operator()(unsigned char *sA, int m0, int kc, int g8, int tid) const
    {
        for (int i = tid; i < umma::TM * g8; i += umma::THREADS) {
            const int r = i / g8, kg = i % g8;
            const int row = m0 + r, k0 = kc + kg * 8;
            const int t = k0 / cin, ch = k0 - t * cin;
            uint4 w = make_uint4(0u, 0u, 0u, 0u);
            if (row < M && t < ntaps) {
                const int cell = row % P;
                const int nc = tap_cell(dim, cell, t);
                if (nc >= 0) {
                    const float4 *src = reinterpret_cast<const float4 *>(H + ((size_t)(row - cell + nc) * cin + ch));
                    const float4 a = __ldg(src), b = __ldg(src + 1);
                    auto pk = [](float x, float y) {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(x, y);
                        return *reinterpret_cast<const unsigned *>(&h);
                    };
                    w = make_uint4(pk(a.x, a.y), pk(a.z, a.w), pk(b.x, b.y), pk(b.z, b.w));
                }
            }
            *reinterpret_cast<uint4 *>(sA + umma::core_off(r, kg)) = w;
        }
    }
};

// ---- features --------------------------------------------------------------
struct FeatArgs {
    const int *ids;
    int n;
    const void *F0, *F1;
    int cur[16];
    const int *level, *ref;
    int ml;
    double u_ref;
    float *X;   // [n * P][C0]
};

template <int DIM, int Q, typename T>
__global__ void k_features(const FeatArgs a)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    __shared__ float su[3][MC];
    const int j = blockIdx.x, t = threadIdx.x;
    if (j >= a.n) return;
    const int b = a.ids[j];
    const int L = a.level[b];
    const T *f = static_cast<const T *>(a.cur[L] ? a.F1 : a.F0) + (long long)b * BLK + t;
    C r = 0, x = 0, y = 0, z = 0;
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const C fp = ST<T>::dec(f[lat_pb(DIM, p) * MC]) + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        r += fp;
        x += C(lat_c(DIM, 0, p)) * fp;
        y += C(lat_c(DIM, 1, p)) * fp;
        if (DIM == 3) z += C(lat_c(DIM, 2, p)) * fp;
    }
    const float U = (float)a.u_ref;
    const float u = (float)(x / r) / U, v = (float)(y / r) / U, w = (DIM == 3) ? (float)(z / r) / U : 0.f;
    su[0][t] = u;
    su[1][t] = v;
    su[2][t] = w;
    __syncthreads();
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    // In-block differences: central inside, one-sided at the faces.
    auto d = [&](int comp, int axis) {
        const int pos = axis == 0 ? I : (axis == 1 ? J : K);
        const int step = axis == 0 ? 1 : (axis == 1 ? 4 : 16);
        const int lo = pos > 0 ? t - step : t, hi = pos < 3 ? t + step : t;
        return (su[comp][hi] - su[comp][lo]) / (float)((pos > 0 ? 1 : 0) + (pos < 3 ? 1 : 0));
    };
    float om;
    if (DIM == 2) {
        om = fabsf(d(1, 0) - d(0, 1));
    } else {
        const float ox = d(2, 1) - d(1, 2), oy = d(0, 2) - d(2, 0), oz = d(1, 0) - d(0, 1);
        om = sqrtf(ox * ox + oy * oy + oz * oz);
    }
    float *o = a.X + ((long long)j * MC + t) * C0;
    o[0] = (float)(r - C(1)) / (U * U);
    o[1] = u;
    o[2] = v;
    o[3] = w;
    o[4] = om * (float)(1 << L);   // per coarse cell, the units the percentile rule compares in
    o[5] = (float)L / (float)(a.ml > 1 ? a.ml - 1 : 1);
    o[6] = (a.ref[b] == REF_REFINED || a.ref[b] == REF_REFINED_WCHILD) ? 1.f : 0.f;
    o[7] = 1.f;
}

template <int DIM, int Q, typename T> struct RunFeatures {
    static int run(agal_ctx *c, const int *ids, int n, float *X, cudaStream_t s)
    {
        FeatArgs a{};
        a.ids = ids;
        a.n = n;
        a.F0 = c->F[0];
        a.F1 = c->F[1];
        for (int L = 0; L < c->max_levels && L < 16; L++) a.cur[L] = c->cur[L];
        a.level = c->cblock_level;
        a.ref = c->cblock_ID_ref;
        a.ml = c->max_levels;
        a.u_ref = c->P.u_ref != 0.0 ? c->P.u_ref : 0.05;
        a.X = X;
        if (n > 0) k_features<DIM, Q, T><<<n, Geo<DIM>::MC, 0, s>>>(a);
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
};

// ---- layer kernels -----------------------------------------------------------
// im2col: out[row][tap * Cin + ch] = in[row of the tap's cell][ch] (BF16),
// zero outside the block and in the padding columns up to Kp.
__global__ void k_im2col(const float *in, int rows, int dim, int cin, int kp, bf16 *out)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)rows * kp) return;
    const int row = (int)(g / kp), col = (int)(g % kp);
    const int P = cells(dim), t = col / cin, ch = col % cin;
    float v = 0.f;
    if (t < taps(dim)) {
        const int nc = tap_cell(dim, row % P, t);
        if (nc >= 0) v = in[((long long)(row - row % P) + nc) * cin + ch];
    }
    out[g] = __float2bfloat16_rn(v);
}

// col2im (gather): dH[row][ch] = sum over taps of dX[row'][tap * C + ch] with
// row' the cell whose tap reaches this cell.
__global__ void k_col2im(const float *dX, int rows, int dim, int c, int kp, float *dH)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)rows * c) return;
    const int row = (int)(g / c), ch = (int)(g % c);
    const int P = cells(dim), cell = row % P, base = row - cell;
    float s = 0.f;
    for (int t = 0; t < taps(dim); t++) {
        // the cell whose tap t lands here is the neighbour along the opposite tap
        const int src = tap_cell(dim, cell, taps(dim) - 1 - t);
        if (src >= 0) s += dX[((long long)base + src) * kp + t * c + ch];
    }
    dH[g] = s;
}

__global__ void k_bias_relu(const float *Y, const float *b, int rows, int c, float *H)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)rows * c) return;
    H[g] = fmaxf(Y[g] + b[g % c], 0.f);
}

// dY = dH * [H > 0], FP32 and BF16 copies.
__global__ void k_relu_back(const float *dH, const float *H, int rows, int c, float *dY, bf16 *dYb)
{
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= (long long)rows * c) return;
    const float v = H[g] > 0.f ? dH[g] : 0.f;
    dY[g] = v;
    dYb[g] = __float2bfloat16_rn(v);
}

// out[c][r] = in[r][c] for a rows x cols matrix (BF16 or FP32 source), rows of
// out padded to ld (>= rows, zero beyond rows).
template <typename S>
__global__ void k_transpose_bf16(const S *in, int rows, int cols, int ld, bf16 *out)
{
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        float v = 0.f;
        if (r < rows && c < cols) {
            if constexpr (sizeof(S) == 2) v = __bfloat162float(in[(long long)r * cols + c]);
            else v = (float)in[(long long)r * cols + c];
        }
        tile[i][threadIdx.x] = v;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (c < cols && r < ld) out[(long long)c * ld + r] = __float2bfloat16_rn(tile[threadIdx.x][i]);
    }
}

// Block pooling, sigmoid cross entropy and its gradient.  z[j][k] = mean over
// the block's cells of Z + b3[k]; loss over valid blocks (weight wt), the
// positive class of output k weighted by pw[k]:
//   l = wt (pw y softplus(-z) + (1 - y) softplus(z)),
//   dl/dz = wt (sigmoid(z) (pw y + 1 - y) - pw y).
__global__ void k_pool_loss(const float *Z, const float *b3, int n, int P, const float *Y, const float *Wt,
                            float pw0, float pw1, float inv_count, float *logits, float *dZrow, bf16 *dZb, int dzld,
                            float *loss, float *db3)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int k = 0; k < NO; k++) {
        float s = 0.f;
        for (int c = 0; c < P; c++) s += Z[((long long)j * P + c) * NO + k];
        const float z = s / (float)P + b3[k];
        logits[j * NO + k] = z;
        if (!Y) continue;
        const float y = Y[j * NO + k], wt = Wt[j], pw = k == 0 ? pw0 : pw1;
        const float p = 1.f / (1.f + expf(-z));
        const float sp = log1pf(expf(-fabsf(z)));   // softplus(z) = max(z, 0) + sp, softplus(-z) = max(-z, 0) + sp
        const float l = wt * (pw * y * (fmaxf(-z, 0.f) + sp) + (1.f - y) * (fmaxf(z, 0.f) + sp));
        const float g = wt * (p * (pw * y + 1.f - y) - pw * y) * inv_count;
        atomicAdd(loss, l * inv_count);
        atomicAdd(&db3[k], g);
        for (int c = 0; c < P; c++) {
            const long long r = (long long)j * P + c;
            dZrow[r * NO + k] = g / (float)P;
            dZb[r * dzld + k] = __float2bfloat16_rn(g / (float)P);
        }
    }
}

// Column sums (bias gradients) of a rows x c FP32 matrix, one thread per column.
__global__ void k_colsum(const float *A, int rows, int c, float *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= c) return;
    float s = 0.f;
    for (int r = 0; r < rows; r++) s += A[(long long)r * c + k];
    out[k] += s;
}

// grad[n][k] += gT[k][n] (weight gradients come out of the GEMM transposed).
__global__ void k_add_transposed(const float *gT, int K, int N, int kp, float *grad)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N * kp) return;
    const int n = g / kp, k = g % kp;
    if (k < K) grad[g] += gT[(long long)k * N + n];
}

__global__ void k_adam(float *w, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_to_bf16(const float *in, int n, bf16 *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

// lvl[j] = level of block ids[j].
__global__ void k_gather_level(const int *ids, int n, const int *level, int *lvl)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) lvl[j] = level[ids[j]];
}

// Marks from predicted logits with the plain criterion's admissibility rules
// (solver_lbm_criterion.cu:560-592): refinement of unrefined, eligible blocks
// below MAX_LEVELS_INTERIOR-1, coarsening of refined blocks.
// A block predicted at the previous regrid counts if it still sits on the
// level it had then.  write = 0 only sets the refinement flags.
__global__ void k_apply_marks(const int *ids, const int *lvl0, int n, const float *logits, float thr_r, float thr_c,
                              int *ref,
                              const int *nbr, long long nmb, int qmax, const int *level, int mli, int *flag,
                              int only_refine, int write)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int b = ids[j];
    const int r = ref[b];
    const bool same = level[b] == lvl0[j];
    bool eligible = true;
    for (int q = 0; q < qmax; q++)
        if (nbr[b + (long long)q * nmb] == N_SKIPID) eligible = false;
    const bool up = same && logits[j * NO] > thr_r, down = same && logits[j * NO + 1] > thr_c;
    if (flag) flag[j] = up ? 1 : 0;
    if (!write) return;
    if (r == REF_UNREFINED && eligible && level[b] < mli - 1 && up) ref[b] = REF_MARK_REFINE;
    if (!only_refine && r == REF_REFINED && down) ref[b] = REF_MARK_COARSEN;
}

// Judge: plain refinement marks the network did not predict.
__global__ void k_judge(const int *ids, int n, const int *pred_flag, const int *ref, int *counts)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int r = ref[ids[j]];
    if (r == REF_MARK_REFINE) {
        atomicAdd(&counts[0], 1);
        if (!pred_flag[j]) atomicAdd(&counts[1], 1);
    }
}

// Labels over a horizon of H regrids: refine if the rule decides to refine
// at any of them, coarsen only if it decides to coarsen at all of them, and
// weight 1 only for a block that keeps its level through all of them.
__global__ void k_label_acc(float *Y, float *Wt, const float *Yn, const float *Wn, int n, int first)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    if (first) {
        Y[2 * j] = Yn[2 * j];
        Y[2 * j + 1] = Yn[2 * j + 1];
        Wt[j] = Wn[j];
    } else {
        Y[2 * j] = fmaxf(Y[2 * j], Yn[2 * j]);
        Y[2 * j + 1] = fminf(Y[2 * j + 1], Yn[2 * j + 1]);
        Wt[j] = Wt[j] * Wn[j];
    }
}

unsigned gridn(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

}  // namespace learn
}  // namespace agal

using namespace agal;
using namespace agal::learn;

struct agal_learn {
    int dim = 2, P = 16, T = 9, K1 = 72, K1p = 80, K2 = 288;
    size_t oW1 = 0, ob1 = 0, oW2 = 0, ob2 = 0, oW3 = 0, ob3 = 0, np = 0;
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // FP32 master weights, grads, Adam moments
    bf16 *W1b = nullptr, *W2b = nullptr, *W3b = nullptr;            // [N][K]
    bf16 *W2t = nullptr, *W3t = nullptr;                            // [K2][32], [K2][16]
    long long adam_t = 0;
    float pw[NO] = {1.f, 1.f};                                      // positive-class weights of the loss
    struct Snap {
        int n = 0;
        float *X = nullptr;                  // [n * P][C0]
        int *ids = nullptr, *lvl = nullptr;  // block IDs and their levels at the snapshot
        float *Y = nullptr, *Wt = nullptr;   // labels [n][2], weights [n]
        float *D = nullptr;                  // the rule's decisions on the snapshot's own state [n][2]
        int got = 0;                         // regrids of the horizon folded into Y so far
        bool labelled = false;
    };
    std::vector<Snap> snaps;
    // work buffers, sized for cap rows
    long long cap = 0;
    bf16 *X1b = nullptr, *X2b = nullptr, *X3b = nullptr, *Xt = nullptr, *dYt = nullptr, *dYb = nullptr, *dZb = nullptr;
    float *Y = nullptr, *H1 = nullptr, *H2 = nullptr, *Z = nullptr, *dZ = nullptr, *dX = nullptr, *dH = nullptr,
          *dY = nullptr, *gT = nullptr, *logits = nullptr, *scal = nullptr;
    int *flags = nullptr, *status = nullptr, *counts = nullptr;
    cudaStream_t s = nullptr;
    // solver coupling
    int judge_every = 4;
    // 0: a snapshot is taken after a regrid and labelled by the next one, and
    // the prediction made after a regrid is applied at the next.  h >= 1
    // (look-ahead): a snapshot is taken at a regrid before its refinement
    // pass and labelled by that regrid and the next h - 1, and the
    // prediction is made and applied at the same regrid.
    int horizon = 0;
    int implicit = 1;                        // inference convolutions as implicit GEMMs
    float *lab_Y = nullptr, *lab_W = nullptr;   // one regrid's decisions, folded into the labels
    long long lab_cap = 0;
    long long regrids = 0, judged = 0, plain_refine = 0, missed = 0;
    float thr[NO] = {0.f, 0.f};              // logit thresholds of the two outputs (0 = probability 1/2)
    int pred_n = 0;                          // prediction made at the last regrid
    int *pred_ids = nullptr, *pred_lvl = nullptr;
    float *pred_X = nullptr, *pred_logits = nullptr;
    long long pred_cap = 0;
    std::string err;
};

namespace {

int lerr(agal_learn *m, int code, const std::string &msg)
{
    if (m) m->err = msg;
    return code;
}

#define LCUDA(m, call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) return lerr((m), e_ == cudaErrorMemoryAllocation ? AGAL_ERR_OOM : AGAL_ERR_CUDA, \
                                           std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename X>
cudaError_t grow(X **p, long long n)
{
    if (*p) cudaFree(*p);
    *p = nullptr;
    return cudaMalloc(p, sizeof(X) * (size_t)std::max(n, 1LL));
}

int ensure(agal_learn *m, long long rows)
{
    const long long rp = pad16((int)std::min<long long>(rows, 1LL << 30));
    if (rp <= m->cap) return AGAL_OK;
    const long long c = std::max(rp, m->cap * 3 / 2);
    const int kmax = std::max(m->K2, m->K1p);
    LCUDA(m, grow(&m->X1b, c * m->K1p));
    LCUDA(m, grow(&m->X2b, c * m->K2));
    LCUDA(m, grow(&m->X3b, c * m->K2));
    LCUDA(m, grow(&m->Xt, c * kmax));
    LCUDA(m, grow(&m->dYt, c * CH));
    LCUDA(m, grow(&m->dYb, c * CH));
    LCUDA(m, grow(&m->dZb, c * 16));
    LCUDA(m, grow(&m->Y, c * CH));
    LCUDA(m, grow(&m->H1, c * CH));
    LCUDA(m, grow(&m->H2, c * CH));
    LCUDA(m, grow(&m->Z, c * NO));
    LCUDA(m, grow(&m->dZ, c * NO));
    LCUDA(m, grow(&m->dX, c * m->K2));
    LCUDA(m, grow(&m->dH, c * CH));
    LCUDA(m, grow(&m->dY, c * CH));
    LCUDA(m, grow(&m->logits, c / m->P * NO + NO));
    LCUDA(m, grow(&m->flags, c / m->P + 1));
    m->cap = c;
    return AGAL_OK;
}

int upload_bf16(agal_learn *m, cudaStream_t s)
{
    k_to_bf16<<<gridn(CH * m->K1p), 256, 0, s>>>(m->w + m->oW1, CH * m->K1p, m->W1b);
    k_to_bf16<<<gridn(CH * m->K2), 256, 0, s>>>(m->w + m->oW2, CH * m->K2, m->W2b);
    k_to_bf16<<<gridn(NO * m->K2), 256, 0, s>>>(m->w + m->oW3, NO * m->K2, m->W3b);
    const dim3 tb(32, 8);
    k_transpose_bf16<float><<<dim3((m->K2 + 31) / 32, 1), tb, 0, s>>>(m->w + m->oW2, CH, m->K2, CH, m->W2t);
    k_transpose_bf16<float><<<dim3((m->K2 + 31) / 32, 1), tb, 0, s>>>(m->w + m->oW3, NO, m->K2, 16, m->W3t);
    LCUDA(m, cudaGetLastError());
    return AGAL_OK;
}

int gemm(agal_learn *m, const bf16 *A, const bf16 *B, float *D, int M, int N, int K, int ldd, cudaStream_t s)
{
    LCUDA(m, umma::gemm_bf16(A, B, D, M, N, K, ldd, m->status, s));
    return AGAL_OK;
}

// Convolution of the layer input H [rows][cin] by the BF16 weights B [N][K]:
// D = im2col(H) . B^T, the columns gathered inside the GEMM.
int conv_gemm(agal_learn *m, const float *H, int cin, int rows, const bf16 *B, float *D, int N, int K, int ldd,
              cudaStream_t s)
{
    const GatherA ga{H, rows, cin, m->dim, m->P, taps(m->dim)};
    LCUDA(m, umma::gemm_bf16_with(ga, B, D, rows, N, K, ldd, m->status, s));
    return AGAL_OK;
}

// Transposed BF16 copy of a rows x cols matrix into [cols][ld] (ld >= rows).
template <typename S>
void transpose(const S *in, int rows, int cols, int ld, bf16 *out, cudaStream_t s)
{
    k_transpose_bf16<S><<<dim3((cols + 31) / 32, (ld + 31) / 32), dim3(32, 8), 0, s>>>(in, rows, cols, ld, out);
}

// Forward pass of n blocks (features X0) on stream s, logits to m->logits;
// with labels, the loss (added to m->scal[0]) and the gradients (added to m->g).
int forward(agal_learn *m, const float *X0, int n, const float *Ylab, const float *Wt, float inv_count, cudaStream_t s)
{
    if (n <= 0) return AGAL_OK;
    const int P = m->P, rows = n * P, rp = pad16(rows), K1p = m->K1p, K2 = m->K2;
    int rc = ensure(m, rows);
    if (rc) return rc;
    if (!Ylab && m->implicit) {
        // Inference: the three convolutions as implicit GEMMs (no columns in
        // global memory); bit for bit the path below.
        if ((rc = conv_gemm(m, X0, C0, rows, m->W1b, m->Y, CH, K1p, CH, s))) return rc;
        k_bias_relu<<<gridn((long long)rows * CH), 256, 0, s>>>(m->Y, m->w + m->ob1, rows, CH, m->H1);
        if ((rc = conv_gemm(m, m->H1, CH, rows, m->W2b, m->Y, CH, K2, CH, s))) return rc;
        k_bias_relu<<<gridn((long long)rows * CH), 256, 0, s>>>(m->Y, m->w + m->ob2, rows, CH, m->H2);
        if ((rc = conv_gemm(m, m->H2, CH, rows, m->W3b, m->Z, NO, K2, NO, s))) return rc;
        k_pool_loss<<<gridn(n, 128), 128, 0, s>>>(m->Z, m->w + m->ob3, n, P, nullptr, nullptr, m->pw[0], m->pw[1],
                                                  inv_count, m->logits, m->dZ, m->dZb, 16, m->scal, m->g + m->ob3);
        LCUDA(m, cudaGetLastError());
        return AGAL_OK;
    }
    k_im2col<<<gridn((long long)rows * K1p), 256, 0, s>>>(X0, rows, m->dim, C0, K1p, m->X1b);
    if ((rc = gemm(m, m->X1b, m->W1b, m->Y, rows, CH, K1p, CH, s))) return rc;
    k_bias_relu<<<gridn((long long)rows * CH), 256, 0, s>>>(m->Y, m->w + m->ob1, rows, CH, m->H1);
    k_im2col<<<gridn((long long)rows * K2), 256, 0, s>>>(m->H1, rows, m->dim, CH, K2, m->X2b);
    if ((rc = gemm(m, m->X2b, m->W2b, m->Y, rows, CH, K2, CH, s))) return rc;
    k_bias_relu<<<gridn((long long)rows * CH), 256, 0, s>>>(m->Y, m->w + m->ob2, rows, CH, m->H2);
    k_im2col<<<gridn((long long)rows * K2), 256, 0, s>>>(m->H2, rows, m->dim, CH, K2, m->X3b);
    if ((rc = gemm(m, m->X3b, m->W3b, m->Z, rows, NO, K2, NO, s))) return rc;
    if (Ylab) LCUDA(m, cudaMemsetAsync(m->dZb, 0, sizeof(bf16) * (size_t)rp * 16, s));
    k_pool_loss<<<gridn(n, 128), 128, 0, s>>>(m->Z, m->w + m->ob3, n, P, Ylab, Wt, m->pw[0], m->pw[1], inv_count,
                                         m->logits, m->dZ, m->dZb, 16, m->scal, m->g + m->ob3);
    LCUDA(m, cudaGetLastError());
    if (!Ylab) return AGAL_OK;
    // ---- backward ----
    // dW3^T [K2 x 2] = X3^T . dZ
    transpose<bf16>(m->X3b, rows, K2, rp, m->Xt, s);
    transpose<float>(m->dZ, rows, NO, rp, m->dYt, s);
    if ((rc = gemm(m, m->Xt, m->dYt, m->gT, K2, NO, rp, NO, s))) return rc;
    k_add_transposed<<<gridn(NO * K2), 256, 0, s>>>(m->gT, K2, NO, K2, m->g + m->oW3);
    // dX3 = dZ . W3 (N tiled by 32), then back to the cells of h2
    for (int n0 = 0; n0 < K2; n0 += umma::TN)
        if ((rc = gemm(m, m->dZb, m->W3t + (size_t)n0 * 16, m->dX + n0, rows, std::min(umma::TN, K2 - n0), 16, K2, s)))
            return rc;
    k_col2im<<<gridn((long long)rows * CH), 256, 0, s>>>(m->dX, rows, m->dim, CH, K2, m->dH);
    k_relu_back<<<gridn((long long)rows * CH), 256, 0, s>>>(m->dH, m->H2, rows, CH, m->dY, m->dYb);
    k_colsum<<<1, CH, 0, s>>>(m->dY, rows, CH, m->g + m->ob2);
    // dW2^T [K2 x 32] = X2^T . dY2
    transpose<bf16>(m->X2b, rows, K2, rp, m->Xt, s);
    transpose<bf16>(m->dYb, rows, CH, rp, m->dYt, s);
    if ((rc = gemm(m, m->Xt, m->dYt, m->gT, K2, CH, rp, CH, s))) return rc;
    k_add_transposed<<<gridn(CH * K2), 256, 0, s>>>(m->gT, K2, CH, K2, m->g + m->oW2);
    // dX2 = dY2 . W2, back to h1
    for (int n0 = 0; n0 < K2; n0 += umma::TN)
        if ((rc = gemm(m, m->dYb, m->W2t + (size_t)n0 * CH, m->dX + n0, rows, std::min(umma::TN, K2 - n0), CH, K2, s)))
            return rc;
    k_col2im<<<gridn((long long)rows * CH), 256, 0, s>>>(m->dX, rows, m->dim, CH, K2, m->dH);
    k_relu_back<<<gridn((long long)rows * CH), 256, 0, s>>>(m->dH, m->H1, rows, CH, m->dY, m->dYb);
    k_colsum<<<1, CH, 0, s>>>(m->dY, rows, CH, m->g + m->ob1);
    // dW1^T [K1p x 32] = X1^T . dY1
    transpose<bf16>(m->X1b, rows, K1p, rp, m->Xt, s);
    transpose<bf16>(m->dYb, rows, CH, rp, m->dYt, s);
    if ((rc = gemm(m, m->Xt, m->dYt, m->gT, K1p, CH, rp, CH, s))) return rc;
    k_add_transposed<<<gridn(CH * K1p), 256, 0, s>>>(m->gT, m->K1, CH, K1p, m->g + m->oW1);
    LCUDA(m, cudaGetLastError());
    return AGAL_OK;
}

int check_status(agal_learn *m, cudaStream_t s)
{
    int st = 0;
    LCUDA(m, cudaMemcpyAsync(&st, m->status, sizeof(int), cudaMemcpyDeviceToHost, s));
    LCUDA(m, cudaStreamSynchronize(s));
    if (st) return lerr(m, st, "tensor-core GEMM wait timed out");
    return AGAL_OK;
}

int total_blocks(const agal_ctx *c)
{
    int tot = 0;
    for (int L = 0; L < c->max_levels; L++) tot += c->n_ids[L];
    return tot;
}

// IDs of every active block of the case (level by level, ID-set order) and
// their levels into ids / lvl (capacity >= total_blocks), on stream s.
int collect_blocks(agal_learn *m, agal_ctx *c, int *ids, int *lvl, cudaStream_t s)
{
    int off = 0;
    for (int L = 0; L < c->max_levels; L++) {
        const int k = c->n_ids[L];
        if (k > 0)
            LCUDA(m, cudaMemcpyAsync(ids + off, c->id_set + (size_t)L * c->nmb, sizeof(int) * k,
                                     cudaMemcpyDeviceToDevice, s));
        off += k;
    }
    if (off > 0) k_gather_level<<<gridn(off), 256, 0, s>>>(ids, off, c->cblock_level, lvl);
    LCUDA(m, cudaGetLastError());
    return AGAL_OK;
}

int features(agal_learn *m, agal_ctx *c, const int *ids, int n, float *X, cudaStream_t s)
{
    const int rc = dispatch<RunFeatures>(c, ids, n, X, s);
    if (rc) return lerr(m, rc, c->err);
    return AGAL_OK;
}

// Labelled snapshot k: 1 / (2 * sum of weights), 0 when nothing is weighted.
int snapshot_norm(agal_learn *m, int k, float *inv)
{
    const auto &sn = m->snaps[k];
    std::vector<float> wt(std::max(sn.n, 1), 0.f);
    if (sn.n > 0) LCUDA(m, cudaMemcpy(wt.data(), sn.Wt, sizeof(float) * sn.n, cudaMemcpyDeviceToHost));
    double cnt = 0;
    for (int j = 0; j < sn.n; j++) cnt += wt[j];
    *inv = cnt > 0 ? (float)(1.0 / (cnt * NO)) : 0.f;
    return AGAL_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" int agal_learn_gemm_bf16(const uint16_t *A, const uint16_t *B, float *D, int M, int N, int K)
{
    // D[M x N] = A[M x K] . B[N x K]^T on host buffers (BF16 bit patterns in,
    // FP32 out) through the tcgen05 kernel; a test hook of the layers' GEMM.
    if (!A || !B || !D || M <= 0 || N < 1 || N > umma::TN || K <= 0 || K % 16) return AGAL_ERR_PARAM;
    bf16 *dA = nullptr, *dB = nullptr;
    float *dD = nullptr;
    int *st = nullptr;
    int rc = AGAL_OK, hs = 0;
    if (cudaMalloc(&dA, sizeof(uint16_t) * (size_t)M * K) != cudaSuccess ||
        cudaMalloc(&dB, sizeof(uint16_t) * (size_t)N * K) != cudaSuccess ||
        cudaMalloc(&dD, sizeof(float) * (size_t)M * N) != cudaSuccess || cudaMalloc(&st, sizeof(int)) != cudaSuccess) {
        rc = AGAL_ERR_OOM;
    } else if (cudaMemcpy(dA, A, sizeof(uint16_t) * (size_t)M * K, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(dB, B, sizeof(uint16_t) * (size_t)N * K, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemset(st, 0, sizeof(int)) != cudaSuccess ||
               umma::gemm_bf16(dA, dB, dD, M, N, K, N, st, 0) != cudaSuccess ||
               cudaDeviceSynchronize() != cudaSuccess ||
               cudaMemcpy(D, dD, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost) != cudaSuccess ||
               cudaMemcpy(&hs, st, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        rc = AGAL_ERR_CUDA;
    } else if (hs) {
        rc = hs;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(st);
    return rc;
}

extern "C" int agal_learn_create(int dim, unsigned long long seed, agal_learn **out)
{
    if (!out || (dim != 2 && dim != 3)) return AGAL_ERR_PARAM;
    *out = nullptr;
    agal_learn *m = new agal_learn();
    m->dim = dim;
    m->P = cells(dim);
    m->T = taps(dim);
    m->K1 = m->T * C0;
    m->K1p = pad16(m->K1);
    m->K2 = m->T * CH;
    m->oW1 = 0;
    m->ob1 = m->oW1 + (size_t)CH * m->K1p;
    m->oW2 = m->ob1 + CH;
    m->ob2 = m->oW2 + (size_t)CH * m->K2;
    m->oW3 = m->ob2 + CH;
    m->ob3 = m->oW3 + (size_t)NO * m->K2;
    m->np = m->ob3 + NO;
    // He-uniform initial weights (padding columns of W1 stay zero), zero biases.
    std::vector<float> h(m->np, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](size_t o, int nout, int k, int kp) {
        const float a = std::sqrt(6.0f / (float)k);
        std::uniform_real_distribution<float> u(-a, a);
        for (int r = 0; r < nout; r++)
            for (int q = 0; q < k; q++) h[o + (size_t)r * kp + q] = u(rng);
    };
    fill(m->oW1, CH, m->K1, m->K1p);
    fill(m->oW2, CH, m->K2, m->K2);
    fill(m->oW3, NO, m->K2, m->K2);
    bool ok = cudaStreamCreateWithFlags(&m->s, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&m->w, sizeof(float) * m->np) == cudaSuccess && cudaMalloc(&m->g, sizeof(float) * m->np) == cudaSuccess &&
         cudaMalloc(&m->m, sizeof(float) * m->np) == cudaSuccess && cudaMalloc(&m->v, sizeof(float) * m->np) == cudaSuccess &&
         cudaMalloc(&m->W1b, sizeof(bf16) * CH * m->K1p) == cudaSuccess &&
         cudaMalloc(&m->W2b, sizeof(bf16) * CH * m->K2) == cudaSuccess &&
         cudaMalloc(&m->W3b, sizeof(bf16) * NO * m->K2) == cudaSuccess &&
         cudaMalloc(&m->W2t, sizeof(bf16) * m->K2 * CH) == cudaSuccess &&
         cudaMalloc(&m->W3t, sizeof(bf16) * m->K2 * 16) == cudaSuccess &&
         cudaMalloc(&m->gT, sizeof(float) * std::max(m->K2, m->K1p) * CH) == cudaSuccess &&
         cudaMalloc(&m->scal, sizeof(float) * 4) == cudaSuccess && cudaMalloc(&m->status, sizeof(int)) == cudaSuccess &&
         cudaMalloc(&m->counts, sizeof(int) * 4) == cudaSuccess;
    ok = ok && cudaMemcpy(m->w, h.data(), sizeof(float) * m->np, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(m->m, 0, sizeof(float) * m->np) == cudaSuccess && cudaMemset(m->v, 0, sizeof(float) * m->np) == cudaSuccess &&
         cudaMemset(m->g, 0, sizeof(float) * m->np) == cudaSuccess && cudaMemset(m->status, 0, sizeof(int)) == cudaSuccess;
    if (!ok || upload_bf16(m, m->s) != AGAL_OK || cudaStreamSynchronize(m->s) != cudaSuccess) {
        cudaGetLastError();
        agal_learn_destroy(m);
        return AGAL_ERR_CUDA;
    }
    *out = m;
    return AGAL_OK;
}

extern "C" int agal_learn_destroy(agal_learn *m)
{
    if (!m) return AGAL_ERR_PARAM;
    if (m->s) cudaStreamSynchronize(m->s);
    for (auto &sn : m->snaps) {
        cudaFree(sn.X); cudaFree(sn.ids); cudaFree(sn.lvl); cudaFree(sn.Y); cudaFree(sn.Wt); cudaFree(sn.D);
    }
    void *ps[] = {m->w, m->g, m->m, m->v, m->W1b, m->W2b, m->W3b, m->W2t, m->W3t, m->X1b, m->X2b, m->X3b, m->Xt,
                  m->dYt, m->dYb, m->dZb, m->Y, m->H1, m->H2, m->Z, m->dZ, m->dX, m->dH, m->dY, m->gT, m->logits,
                  m->scal, m->flags, m->status, m->counts, m->pred_ids, m->pred_lvl, m->pred_X, m->pred_logits,
                  m->lab_Y, m->lab_W};
    for (void *p : ps)
        if (p) cudaFree(p);
    if (m->s) cudaStreamDestroy(m->s);
    delete m;
    return AGAL_OK;
}

extern "C" const char *agal_learn_last_error(const agal_learn *m) { return m ? m->err.c_str() : ""; }

extern "C" int agal_learn_num_params(const agal_learn *m, long long *n)
{
    if (!m || !n) return AGAL_ERR_PARAM;
    *n = (long long)m->np;
    return AGAL_OK;
}

// Parameters in the order W1 [32][K1p] (zero padding columns), b1 [32], W2
// [32][K2], b2 [32], W3 [2][K2], b3 [2], with K1p = 16 ceil(T 8 / 16), K2 =
// 32 T, T = 3^d taps (column = tap * C + channel, tap = (dx+1) + 3 (dy+1) +
// 9 (dz+1)).
extern "C" int agal_learn_get_params(agal_learn *m, float *out, long long n)
{
    if (!m || !out || n != (long long)m->np) return AGAL_ERR_PARAM;
    LCUDA(m, cudaStreamSynchronize(m->s));
    LCUDA(m, cudaMemcpy(out, m->w, sizeof(float) * m->np, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

extern "C" int agal_learn_set_params(agal_learn *m, const float *in, long long n)
{
    if (!m || !in || n != (long long)m->np) return AGAL_ERR_PARAM;
    LCUDA(m, cudaStreamSynchronize(m->s));
    LCUDA(m, cudaMemcpy(m->w, in, sizeof(float) * m->np, cudaMemcpyHostToDevice));
    const int rc = upload_bf16(m, m->s);
    if (rc) return rc;
    LCUDA(m, cudaStreamSynchronize(m->s));
    return AGAL_OK;
}

extern "C" int agal_learn_set_class_weights(agal_learn *m, double refine, double coarsen)
{
    if (!m || !(refine > 0.0) || !(coarsen > 0.0)) return AGAL_ERR_PARAM;
    m->pw[0] = (float)refine;
    m->pw[1] = (float)coarsen;
    return AGAL_OK;
}

// Snapshot of the case's current state: features of every active block, and
// (multi-level cases) the percentile rule's decisions on this same state.
extern "C" int agal_learn_record(agal_learn *m, agal_ctx *c)
{
    if (!m || !c || c->dim != m->dim) return AGAL_ERR_PARAM;
    agal_learn::Snap sn;
    sn.n = total_blocks(c);
    const size_t nb = (size_t)std::max(sn.n, 1);
    auto fail = [&](int rc) {
        cudaFree(sn.ids); cudaFree(sn.lvl); cudaFree(sn.X); cudaFree(sn.Y); cudaFree(sn.Wt); cudaFree(sn.D);
        return rc;
    };
    if (cudaMalloc(&sn.ids, sizeof(int) * nb) != cudaSuccess || cudaMalloc(&sn.lvl, sizeof(int) * nb) != cudaSuccess ||
        cudaMalloc(&sn.X, sizeof(float) * nb * m->P * C0) != cudaSuccess ||
        cudaMalloc(&sn.Y, sizeof(float) * nb * NO) != cudaSuccess || cudaMalloc(&sn.Wt, sizeof(float) * nb) != cudaSuccess ||
        cudaMalloc(&sn.D, sizeof(float) * nb * NO) != cudaSuccess)
        return fail(lerr(m, AGAL_ERR_OOM, "snapshot allocation failed"));
    int rc = collect_blocks(m, c, sn.ids, sn.lvl, c->stream);
    if (!rc) rc = features(m, c, sn.ids, sn.n, sn.X, c->stream);
    if (!rc && cudaMemsetAsync(sn.D, 0, sizeof(float) * nb * NO, c->stream) != cudaSuccess)
        rc = lerr(m, AGAL_ERR_CUDA, "snapshot decisions reset failed");
    if (!rc && c->crit) {
        for (int L = 0; L < c->max_levels && !rc; L++)
            if ((rc = agal_launch_refresh(c, L))) rc = lerr(m, rc, c->err);
        if (!rc && (rc = agal_percentile_decisions(c, 1, sn.ids, nullptr, sn.n, sn.D, nullptr))) rc = lerr(m, rc, c->err);
    }
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = lerr(m, AGAL_ERR_CUDA, "snapshot features failed");
    if (rc) return fail(rc);
    m->snaps.push_back(sn);
    return AGAL_OK;
}

// Labels of the unlabelled snapshots: the decisions of the percentile
// rule's last run on the case (a block above the upper quantile, below the
// lower one), for each snapshot's blocks that still exist on the same level,
// folded over the next `horizon` regrids after the snapshot (k_label_acc).
extern "C" int agal_learn_label(agal_learn *m, agal_ctx *c)
{
    if (!m || !c) return AGAL_ERR_PARAM;
    if (!c->crit) return lerr(m, AGAL_ERR_STATE, "labels need the percentile rule of a multi-level case");
    for (auto it = m->snaps.rbegin(); it != m->snaps.rend(); ++it) {
        if (it->labelled) break;   // older snapshots are complete
        if (it->n > m->lab_cap) {
            LCUDA(m, cudaStreamSynchronize(c->stream));
            LCUDA(m, grow(&m->lab_Y, 2LL * it->n));
            LCUDA(m, grow(&m->lab_W, (long long)it->n));
            m->lab_cap = it->n;
        }
        const int rc = agal_percentile_decisions(c, 0, it->ids, it->lvl, it->n, m->lab_Y, m->lab_W);
        if (rc) return lerr(m, rc, c->err);
        if (it->n > 0)
            k_label_acc<<<gridn(it->n), 256, 0, c->stream>>>(it->Y, it->Wt, m->lab_Y, m->lab_W, it->n, it->got == 0);
        LCUDA(m, cudaGetLastError());
        if (++it->got >= std::max(m->horizon, 1)) it->labelled = true;
    }
    LCUDA(m, cudaStreamSynchronize(c->stream));
    return AGAL_OK;
}

extern "C" int agal_learn_set_horizon(agal_learn *m, int horizon)
{
    if (!m || horizon < 0 || horizon > 64) return AGAL_ERR_PARAM;
    for (const auto &sn : m->snaps)
        if (!sn.labelled && sn.got > 0) return lerr(m, AGAL_ERR_STATE, "horizon changed while snapshots are being labelled");
    m->horizon = horizon;
    return AGAL_OK;
}

// Inference convolutions as implicit GEMMs (1, the default: the columns are
// gathered inside the GEMM) or through materialised im2col columns (0).
// Both give the same logits bit for bit.
extern "C" int agal_learn_set_implicit(agal_learn *m, int on)
{
    if (!m) return AGAL_ERR_PARAM;
    m->implicit = on ? 1 : 0;
    return AGAL_OK;
}

extern "C" int agal_learn_counts(const agal_learn *m, long long *out)
{
    // {snapshots, labelled snapshots, regrids seen, judged regrids, plain
    //  refinement marks at judged regrids, of those missed by the network}
    if (!m || !out) return AGAL_ERR_PARAM;
    long long lab = 0;
    for (const auto &sn : m->snaps) lab += sn.labelled ? 1 : 0;
    out[0] = (long long)m->snaps.size();
    out[1] = lab;
    out[2] = m->regrids;
    out[3] = m->judged;
    out[4] = m->plain_refine;
    out[5] = m->missed;
    return AGAL_OK;
}

extern "C" int agal_learn_snapshot_decisions(agal_learn *m, int k, float *D)
{
    if (!m || k < 0 || k >= (int)m->snaps.size() || !D) return AGAL_ERR_PARAM;
    const auto &sn = m->snaps[k];
    if (sn.n > 0) LCUDA(m, cudaMemcpy(D, sn.D, sizeof(float) * (size_t)sn.n * NO, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

// Loss and gradients of snapshot k at the current weights (gradient check).
extern "C" int agal_learn_gradients(agal_learn *m, int k, float *grad, long long n, double *loss)
{
    if (!m || k < 0 || k >= (int)m->snaps.size() || !m->snaps[k].labelled || (grad && n != (long long)m->np))
        return AGAL_ERR_PARAM;
    const auto &sn = m->snaps[k];
    float inv = 0.f;
    int rc = snapshot_norm(m, k, &inv);
    if (rc) return rc;
    LCUDA(m, cudaMemsetAsync(m->g, 0, sizeof(float) * m->np, m->s));
    LCUDA(m, cudaMemsetAsync(m->scal, 0, sizeof(float) * 4, m->s));
    if ((rc = forward(m, sn.X, sn.n, sn.Y, sn.Wt, inv, m->s))) return rc;
    if ((rc = check_status(m, m->s))) return rc;
    float l = 0.f;
    LCUDA(m, cudaMemcpy(&l, m->scal, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l;
    if (grad) LCUDA(m, cudaMemcpy(grad, m->g, sizeof(float) * m->np, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

// Features / labels / weights of snapshot k (host copies; sizes from n_blocks).
extern "C" int agal_learn_snapshot(agal_learn *m, int k, int *n_blocks, float *X, float *Y, float *Wt)
{
    if (!m || k < 0 || k >= (int)m->snaps.size() || !n_blocks) return AGAL_ERR_PARAM;
    const auto &sn = m->snaps[k];
    *n_blocks = sn.n;
    if (sn.n == 0) return AGAL_OK;
    if (X) LCUDA(m, cudaMemcpy(X, sn.X, sizeof(float) * (size_t)sn.n * m->P * C0, cudaMemcpyDeviceToHost));
    if (Y) LCUDA(m, cudaMemcpy(Y, sn.Y, sizeof(float) * (size_t)sn.n * NO, cudaMemcpyDeviceToHost));
    if (Wt) LCUDA(m, cudaMemcpy(Wt, sn.Wt, sizeof(float) * (size_t)sn.n, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

// Adam over the labelled snapshots [first, last), one snapshot per step, in
// a seeded random order per epoch; mean loss of the last epoch to *loss.
extern "C" int agal_learn_train(agal_learn *m, int first, int last, int epochs, double lr, unsigned long long seed,
                                double *loss)
{
    if (!m || epochs < 0 || first < 0 || last > (int)m->snaps.size() || first > last) return AGAL_ERR_PARAM;
    std::vector<int> order;
    std::vector<float> inv;
    for (int k = first; k < last; k++) {
        if (!m->snaps[k].labelled || m->snaps[k].n == 0) continue;
        float x = 0.f;
        const int rc = snapshot_norm(m, k, &x);
        if (rc) return rc;
        if (x <= 0.f) continue;
        order.push_back(k);
        inv.push_back(x);
    }
    std::mt19937_64 rng(seed);
    double last_loss = 0.0;
    for (int e = 0; e < epochs; e++) {
        std::vector<size_t> perm(order.size());
        for (size_t i = 0; i < perm.size(); i++) perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        LCUDA(m, cudaMemsetAsync(m->scal, 0, sizeof(float) * 4, m->s));
        for (size_t i : perm) {
            const auto &sn = m->snaps[order[i]];
            LCUDA(m, cudaMemsetAsync(m->g, 0, sizeof(float) * m->np, m->s));
            int rc = forward(m, sn.X, sn.n, sn.Y, sn.Wt, inv[i], m->s);
            if (rc) return rc;
            m->adam_t++;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1.f - std::pow(b1, (float)m->adam_t), c2 = 1.f - std::pow(b2, (float)m->adam_t);
            k_adam<<<gridn((long long)m->np), 256, 0, m->s>>>(m->w, m->g, m->m, m->v, (int)m->np, (float)lr, b1, b2,
                                                             1e-8f, c1, c2);
            if ((rc = upload_bf16(m, m->s))) return rc;
        }
        float l = 0.f;
        LCUDA(m, cudaMemcpyAsync(&l, m->scal, sizeof(float), cudaMemcpyDeviceToHost, m->s));
        int rc = check_status(m, m->s);
        if (rc) return rc;
        last_loss = order.empty() ? 0.0 : (double)l / (double)order.size();
    }
    if (loss) *loss = last_loss;
    return AGAL_OK;
}

// Logits of snapshot k's blocks at the current weights: out [n][2].
extern "C" int agal_learn_predict_snapshot(agal_learn *m, int k, float *out)
{
    if (!m || k < 0 || k >= (int)m->snaps.size() || !out) return AGAL_ERR_PARAM;
    const auto &sn = m->snaps[k];
    if (sn.n == 0) return AGAL_OK;
    int rc = forward(m, sn.X, sn.n, nullptr, nullptr, 0.f, m->s);
    if (rc) return rc;
    if ((rc = check_status(m, m->s))) return rc;
    LCUDA(m, cudaMemcpy(out, m->logits, sizeof(float) * (size_t)sn.n * NO, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

// ---- coupling with the solution-based refinement ---------------------------
// mode 1: collect - every regrid labels the previous snapshot with the plain
//         marks and records a new one after the refine/coarsen pass;
// mode 2: predict - the marks of a regrid are the network's prediction from
//         the state after the previous regrid; every judge_every-th regrid
//         the percentile rule also runs, its refinement marks the network
//         missed are counted and applied too.
extern "C" int agal_learn_attach(agal_ctx *c, agal_learn *m, int mode, int judge_every, double threshold)
{
    if (!c) return AGAL_ERR_PARAM;
    if (!m || mode == 0) {
        c->learner = nullptr;
        c->learn_mode = 0;
        return AGAL_OK;
    }
    if (m->dim != c->dim || (mode != 1 && mode != 2) || judge_every < 1 || !(threshold > 0.0 && threshold < 1.0))
        return AGAL_ERR_PARAM;
    c->learner = m;
    c->learn_mode = mode;
    m->judge_every = judge_every;
    m->thr[0] = m->thr[1] = (float)std::log(threshold / (1.0 - threshold));
    m->pred_n = 0;
    return AGAL_OK;
}

extern "C" int agal_learn_set_thresholds(agal_learn *m, double refine, double coarsen)
{
    if (!m || !(refine > 0.0 && refine < 1.0) || !(coarsen > 0.0 && coarsen < 1.0)) return AGAL_ERR_PARAM;
    m->thr[0] = (float)std::log(refine / (1.0 - refine));
    m->thr[1] = (float)std::log(coarsen / (1.0 - coarsen));
    return AGAL_OK;
}

static int predict_now(agal_learn *m, agal_ctx *c);

// Marks of a regrid (called by agal_refine_with_solution instead of the
// criterion while a learner is attached).
int agal_learn_marks(agal_ctx *c)
{
    agal_learn *m = c->learner;
    int rc;
    if (c->learn_mode == 1) {
        if ((rc = agal_launch_criterion(c))) return rc;
        // look-ahead: this regrid's state is a snapshot, its first label the
        // rule's decisions now
        if (m->horizon > 0 && (rc = agal_learn_record(m, c))) return agal_set_err(c, rc, "learned predictor: " + m->err);
        if ((rc = agal_learn_label(m, c))) return agal_set_err(c, rc, "learned predictor: " + m->err);
        return AGAL_OK;
    }
    const bool judge = m->pred_n == 0 || (m->regrids % m->judge_every) == 0;
    m->regrids++;
    if (judge) {
        if ((rc = agal_launch_criterion(c))) return rc;
        m->judged++;
    }
    // look-ahead: predict from this regrid's state and apply it now
    if (m->horizon > 0 && (rc = predict_now(m, c))) return rc;
    if (m->pred_n > 0) {
        // flags of the predicted refinements, on a judged regrid the count of
        // the plain refinement marks the network missed, then the predicted
        // marks (refinements only on a judged regrid: the union with the
        // plain marks, whose coarsening marks stand)
        if (judge) AGAL_CUDA(c, cudaMemsetAsync(m->counts, 0, sizeof(int) * 4, c->stream));
        k_apply_marks<<<gridn(m->pred_n, 128), 128, 0, c->stream>>>(
            m->pred_ids, m->pred_lvl, m->pred_n, m->pred_logits, m->thr[0], m->thr[1], c->cblock_ID_ref, c->cblock_ID_nbr, c->nmb,
            c->Qmax, c->cblock_level, c->P.MAX_LEVELS_INTERIOR, m->flags, 0, 0);
        if (judge)
            k_judge<<<gridn(m->pred_n, 128), 128, 0, c->stream>>>(m->pred_ids, m->pred_n, m->flags, c->cblock_ID_ref,
                                                             m->counts);
        k_apply_marks<<<gridn(m->pred_n, 128), 128, 0, c->stream>>>(
            m->pred_ids, m->pred_lvl, m->pred_n, m->pred_logits, m->thr[0], m->thr[1], c->cblock_ID_ref, c->cblock_ID_nbr, c->nmb,
            c->Qmax, c->cblock_level, c->P.MAX_LEVELS_INTERIOR, nullptr, judge ? 1 : 0, 1);
        AGAL_CUDA(c, cudaGetLastError());
        if (judge) {
            // the judged regrids also surface a timed-out tensor-core wait of
            // the predictions made since the last one
            int h[4] = {0, 0, 0, 0}, st = 0;
            AGAL_CUDA(c, cudaMemcpyAsync(h, m->counts, sizeof(int) * 4, cudaMemcpyDeviceToHost, c->stream));
            AGAL_CUDA(c, cudaMemcpyAsync(&st, m->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
            if (st) return agal_set_err(c, st, "learned predictor: tensor-core GEMM wait timed out");
            m->plain_refine += h[0];
            m->missed += h[1];
        }
    }
    return AGAL_OK;
}

// After the refine/coarsen pass: record a snapshot (collect mode) or predict
// the next regrid's marks from the new state (predict mode, asynchronous on
// the case's stream).
int agal_learn_after_regrid(agal_ctx *c)
{
    agal_learn *m = c->learner;
    if (m->horizon > 0) return AGAL_OK;   // look-ahead: snapshots and predictions happen at the regrid
    if (c->learn_mode == 1) {
        const int rc = agal_learn_record(m, c);
        return rc ? agal_set_err(c, rc, "learned predictor: " + m->err) : AGAL_OK;
    }
    return predict_now(m, c);
}

// Features and forward pass of every active block of the case's current
// state, asynchronous on its stream; the logits become the prediction that
// the next call of k_apply_marks applies.
static int predict_now(agal_learn *m, agal_ctx *c)
{
    int rc;
    const int n = total_blocks(c);
    if (n > m->pred_cap) {
        const long long cap = std::max<long long>(n, m->pred_cap * 3 / 2);
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
        AGAL_CUDA(c, grow(&m->pred_ids, cap));
        AGAL_CUDA(c, grow(&m->pred_lvl, cap));
        AGAL_CUDA(c, grow(&m->pred_X, cap * m->P * C0));
        AGAL_CUDA(c, grow(&m->pred_logits, cap * NO));
        m->pred_cap = cap;
    }
    rc = collect_blocks(m, c, m->pred_ids, m->pred_lvl, c->stream);
    if (!rc) rc = features(m, c, m->pred_ids, n, m->pred_X, c->stream);
    if (!rc) rc = forward(m, m->pred_X, n, nullptr, nullptr, 0.f, c->stream);
    if (!rc && n > 0 &&
        cudaMemcpyAsync(m->pred_logits, m->logits, sizeof(float) * NO * n, cudaMemcpyDeviceToDevice, c->stream) !=
            cudaSuccess)
        rc = lerr(m, AGAL_ERR_CUDA, "prediction copy failed");
    if (rc) return agal_set_err(c, rc, "learned predictor: " + m->err);
    m->pred_n = n;
    return AGAL_OK;
}
