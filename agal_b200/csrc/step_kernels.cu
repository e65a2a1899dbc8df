// Per-level LBM kernels: initial conditions, the fused collide + boundary +
// stream step, macro refresh and FP64 mass/momentum sums.
//
// Population layout (block-major): F[b][s][c] = slot s of cell c of block b,
// so one block's Q x M_CBLOCK values are contiguous and every load of a
// cell's own populations is (block base + compile-time offset).  Slot s of a
// cell holds f_{pb(s)}: the reference's post-stream convention
// (solver_lbm_kernels.cu:67, 251).  agal_dump / agal_load convert to and from
// the reference's slot-major array cells_f_F[s][n_maxcells].
//
// The fused step replaces the reference's sequence
//   Cu_RefreshVariables -> Cu_Collide -> Cu_ImposeBC -> Cu_Stream
// (solver_lbm_kernels.cu:112, 206, 693, 534), which reads and writes the
// populations in place four times per step, by ONE pass that reads the Q
// populations of a cell from buffer A and pushes the Q post-collision values
// to their destination cells in buffer B.  Buffer B then holds exactly what
// the reference's in-place swap leaves behind: slot pb(p) of cell x + c_p
// holds f*_p(x) when the link is open; when it is closed (domain boundary,
// missing same-level neighbour, solid neighbour cell) slot p of x holds
// f*_p(x), passed through the boundary hook for a domain boundary.
// Algorithmic traffic: 2 * Q * sizeof(storage) bytes per cell update.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "ctx.h"
#include "lattice.cuh"
#include "storage.cuh"
#include "step_common.cuh"
#include "dispatch.cuh"

namespace agal {

// The step of chunk `cta` of the level's block list (CPT x 256 / M_CBLOCK
// blocks), given the CTA's shared metadata rows.
template <int DIM, int Q, typename T, int CPT, bool SOLID>
__device__ __forceinline__ void step_body(const StepArgs &a, int cta, int (*s_meta)[Meta<DIM>::W])
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    constexpr int NB = 256 / MC;           // cell-blocks per CTA and round
    constexpr int W = Meta<DIM>::W;
    const int tid = threadIdx.x;
    const int lb = tid / MC, t = tid % MC;

    // Round h of this thread is cell t of the CTA's cell-block h * NB + lb:
    // with several rounds a thread holds the same cell of several blocks, so
    // that every warp-wide load and push still covers whole rows of a block.
    // The block IDs and their metadata rows are written only by the mesh
    // passes, never by a kernel that lets this one launch early, so they are
    // read before the wait for the predecessor (the prologue of programmatic
    // dependent launch); the populations after it.
    int b[CPT];
#pragma unroll
    for (int h = 0; h < CPT; h++) {
        const int kap = (cta * CPT + h) * NB + lb;
        b[h] = (kap < a.n) ? __ldg(&a.ids[kap]) : -1;
        for (int i = t; i < W; i += MC)
            s_meta[h * NB + lb][i] = (b[h] >= 0) ? __ldg(&a.meta[(long long)b[h] * W + i]) : 0;
    }
    const T *__restrict__ f0 = static_cast<const T *>(a.fin) + t;
    pdl_wait();
    const unsigned seed = step_seed(a);

    // Load: slot pb(p) holds f_p (offset form g_p for half storage).
    C g[CPT][Q];
#pragma unroll
    for (int h = 0; h < CPT; h++)
        if (b[h] >= 0)
#pragma unroll
            for (int p = 0; p < Q; p++) g[h][p] = ST<T>::dec(__ldg(f0 + (long long)b[h] * BLK + lat_pb(DIM, p) * MC));
    __syncthreads();
    T *__restrict__ fo = static_cast<T *>(a.fout);
#pragma unroll
    for (int h = 0; h < CPT; h++) {
        const int *nrow = s_meta[h * NB + lb];
        const int fl = nrow[Meta<DIM>::FLAGS];
        if (b[h] < 0 || (fl & META_WALL)) continue;
        // The reference steps in place and leaves solid cells and inactive
        // blocks (refined solid blocks) untouched, so whatever a grid average
        // or an interpolation wrote there stays and feeds the next transfer:
        // carry those cells into the output buffer unchanged.
        const long long base = (long long)b[h] * BLK + t;
        auto carry = [&]() {
#pragma unroll
            for (int sl = 0; sl < Q; sl++) fo[base + sl * MC] = f0[base - t + sl * MC];
        };
        if (!(fl & META_ACTIVE)) {
            if (SOLID) carry();
            continue;
        }
        if (SOLID && __ldg(&a.cmask[(long long)b[h] * MC + t]) == CELL_SOLID) {
            if (a.macro) store_macros<DIM, Q, C, ST<T>::OFF>(g[h], a.macro, a.nmc, (long long)b[h] * MC + t);
            carry();
            continue;
        }
        const bool hook = (fl & META_ONB) && a.bc_preset != AGAL_BC_NONE;
        C ux, uy, uz;
        if (a.macro) store_macros<DIM, Q, C, ST<T>::OFF>(g[h], a.macro, a.nmc, (long long)b[h] * MC + t);
        collide_at<DIM, Q, T>(g[h], a, (long long)b[h] * MC + t, ux, uy, uz);
        push_cell<DIM, Q, T, SOLID>(g[h], ux, uy, uz, b[h], t, nrow, hook, fo, a, seed);
    }
}

template <int DIM, int Q, typename T, int CPT, bool SOLID>
__global__ void __launch_bounds__(256, (StepOcc<DIM, Q, T, CPT>::value))
k_step(const StepArgs a)
{
    __shared__ int s_meta[CPT * (256 / Geo<DIM>::MC)][Meta<DIM>::W];
    step_body<DIM, Q, T, CPT, SOLID>(a, blockIdx.x, s_meta);
    if (a.fix_ticket) fused_fixup<T>(a);
}

// Batched form: one persistent kernel over the chunks of many cases' block
// lists (a global work list).  Chunk w belongs to case i with
// start[i] <= w < start[i + 1] and is stepped with that case's arguments A[i];
// each case's chunks are the chunks k_step would give it alone, so every
// case's populations are those of advancing it alone.
template <int DIM, int Q, typename T, bool SOLID>
__global__ void __launch_bounds__(256, (StepOcc<DIM, Q, T, 1>::value))
k_step_batch(const StepArgs *__restrict__ A, const int *__restrict__ start, int n_cases)
{
    __shared__ int s_meta[256 / Geo<DIM>::MC][Meta<DIM>::W];
    const int total = start[n_cases];
    int i = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        while (start[i + 1] <= w) i++;   // w only grows: the case index only moves forward
        const StepArgs a = A[i];
        step_body<DIM, Q, T, 1, SOLID>(a, w - start[i], s_meta);
        __syncthreads();                 // the metadata rows are refilled for the next chunk
    }
}

// ---------------------------------------------------------------------------
// Initial conditions (Cu_SetInitialConditions, kernels.cu:15-77); writes both
// buffers so that cells never written by a step (solid cells) agree.
struct IcArgs {
    const int *ids;
    int n;
    void *f0, *f1;
    long long nmb;
    const int *cmask;
    const float *fX;
    double dxL, u_ref, noise;
    unsigned long long seed;
    int ic_preset, L;
};

__host__ __device__ inline double ic_noise(unsigned long long seed, int L, long long ix, long long iy,
                                           long long iz, int comp)
{
    unsigned long long z = seed ^ ((unsigned long long)(unsigned)L << 56) ^
                           ((unsigned long long)(ix & 0xFFFFF) << 36) ^
                           ((unsigned long long)(iy & 0xFFFFF) << 16) ^ ((unsigned long long)(iz & 0xFFFF)) ^
                           ((unsigned long long)comp << 60);
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

template <int DIM, int Q, typename T>
__global__ void k_set_ic(const IcArgs a)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long kap = gid / MC;
    const int t = (int)(gid % MC);
    if (kap >= a.n) return;
    const int b = a.ids[kap];
    if (b < 0) return;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    C rho = C(1), u = C(0), v = C(0), w = C(0);
    if (a.ic_preset == AGAL_IC_UNIFORM) {
        u = C(a.u_ref);
        if (a.noise != 0.0) {
            const double amp = a.noise * a.u_ref;
            const long long ix = llrint((double)a.fX[b] / a.dxL) + I;
            const long long iy = llrint((double)a.fX[b + a.nmb] / a.dxL) + J;
            const long long iz = (DIM == 3) ? llrint((double)a.fX[b + 2 * a.nmb] / a.dxL) + K : 0;
            u = C(a.u_ref + amp * ic_noise(a.seed, a.L, ix, iy, iz, 0));
            v = C(amp * ic_noise(a.seed, a.L, ix, iy, iz, 1));
            if (DIM == 3) w = C(amp * ic_noise(a.seed, a.L, ix, iy, iz, 2));
        }
    }
    const C udotu = u * u + v * v + w * w;
    const bool solid = a.cmask[(long long)b * MC + t] == CELL_SOLID;
    T *f0 = static_cast<T *>(a.f0) + (long long)b * BLK + t;
    T *f1 = static_cast<T *>(a.f1) + (long long)b * BLK + t;
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const C cu = C(lat_c(DIM, 0, p)) * u + C(lat_c(DIM, 1, p)) * v + C(lat_c(DIM, 2, p)) * w;
        const C wp = C(lat_w(Q, p));
        C val;
        if (solid) val = C(-1) - (ST<T>::OFF ? wp : C(0));
        else if (!ST<T>::OFF) val = rho * wp * (C(1) + C(3) * cu + C(4.5) * cu * cu - C(1.5) * udotu);
        else val = wp * ((rho - C(1)) + rho * (C(3) * cu + C(4.5) * cu * cu - C(1.5) * udotu));
        f0[lat_pb(DIM, p) * MC] = ST<T>::enc(val);
        f1[lat_pb(DIM, p) * MC] = ST<T>::enc(val);
    }
}

// ---------------------------------------------------------------------------
// Macros of one level from its current buffer (Cu_RefreshVariables,
// kernels.cu:112-159), into the macro array [dim+1][n_maxcells].
struct MacroArgs {
    const int *ids;
    int n;
    const void *f;
    void *macro;
    long long nmc;
};

template <int DIM, int Q, typename T>
__global__ void k_refresh(const MacroArgs a)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long kap = gid / MC;
    const int t = (int)(gid % MC);
    if (kap >= a.n) return;
    const int b = a.ids[kap];
    if (b < 0) return;
    const T *f = static_cast<const T *>(a.f) + (long long)b * BLK + t;
    C rho = 0, u = 0, v = 0, w = 0;
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const C fp = ST<T>::dec(f[lat_pb(DIM, p) * MC]) + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        rho += fp;
        u += C(lat_c(DIM, 0, p)) * fp;
        v += C(lat_c(DIM, 1, p)) * fp;
        if (DIM == 3) w += C(lat_c(DIM, 2, p)) * fp;
    }
    u /= rho;
    v /= rho;
    if (DIM == 3) w /= rho;
    C *m = static_cast<C *>(a.macro);
    const long long cell = (long long)b * MC + t;
    m[cell] = rho;
    m[a.nmc + cell] = u;
    m[2 * a.nmc + cell] = v;
    if (DIM == 3) m[3 * a.nmc + cell] = w;
}

// ---------------------------------------------------------------------------
// Eddy viscosity of the LES models (Cu_ComputeEddyViscosity,
// solver_lbm_kernels_les.cu:460-600): per block, the velocity of the current
// populations (the reference refreshes its macros right before, one-level
// meshes), a one-cell halo extrapolated from the block itself with the
// fourth-order rule 4 d1 - 6 d2 + 4 d3 - d4 (util_math.h:28-110), central
// differences (d+ - d-) / (2 dx), then the model (les.cu:13-250).
template <typename C>
__device__ __forceinline__ C les_model(int model, int dim, C dx, C ux, C uy, C uz, C vx, C vy, C vz, C wx, C wy,
                                       C wz)
{
    const C dx2 = r_mul(dx, dx);
    // strain rate S = (grad u + grad u^T) / 2 and its squared norm
    const C Sxy = r_mul(C(0.5), r_add(uy, vx)), Sxz = r_mul(C(0.5), r_add(uz, wx)),
            Syz = r_mul(C(0.5), r_add(vz, wy));
    C F2 = r_add(r_add(r_mul(ux, ux), r_mul(C(2), r_mul(Sxy, Sxy))), r_mul(vy, vy));
    if (dim == 3)
        F2 = r_add(r_add(r_add(F2, r_mul(C(2), r_mul(Sxz, Sxz))), r_mul(C(2), r_mul(Syz, Syz))), r_mul(wz, wz));
    if (model == 1) {   // Smagorinsky, C_s = 0.1
        return F2 > C(0) ? r_mul(r_mul(C(0.1 * 0.1), dx2), sqrt(r_mul(C(2), F2))) : C(0);
    }
    if (model == 2) {   // WALE, C_w = 0.325
        // g = grad u . grad u, its traceless symmetric part Sd
        const C gxx = r_add(r_add(r_mul(ux, ux), r_mul(uy, vx)), r_mul(uz, wx));
        const C gxy = r_add(r_add(r_mul(ux, uy), r_mul(uy, vy)), r_mul(uz, wy));
        const C gxz = r_add(r_add(r_mul(ux, uz), r_mul(uy, vz)), r_mul(uz, wz));
        const C gyx = r_add(r_add(r_mul(vx, ux), r_mul(vy, vx)), r_mul(vz, wx));
        const C gyy = r_add(r_add(r_mul(vx, uy), r_mul(vy, vy)), r_mul(vz, wy));
        const C gyz = r_add(r_add(r_mul(vx, uz), r_mul(vy, vz)), r_mul(vz, wz));
        const C gzx = r_add(r_add(r_mul(wx, ux), r_mul(wy, vx)), r_mul(wz, wx));
        const C gzy = r_add(r_add(r_mul(wx, uy), r_mul(wy, vy)), r_mul(wz, wy));
        const C gzz = r_add(r_add(r_mul(wx, uz), r_mul(wy, vz)), r_mul(wz, wz));
        const C gkk = dim == 3 ? r_add(r_add(gxx, gyy), gzz) : r_add(gxx, gyy);
        const C third = r_mul(C(1.0 / 3.0), gkk);
        const C Dxx = r_add(gxx, -third), Dyy = r_add(gyy, -third), Dzz = r_add(gzz, -third);
        const C Dxy = r_mul(C(0.5), r_add(gxy, gyx)), Dxz = r_mul(C(0.5), r_add(gxz, gzx)),
                Dyz = r_mul(C(0.5), r_add(gyz, gzy));
        C F1 = r_add(r_add(r_mul(Dxx, Dxx), r_mul(C(2), r_mul(Dxy, Dxy))), r_mul(Dyy, Dyy));
        if (dim == 3)
            F1 = r_add(r_add(r_add(F1, r_mul(C(2), r_mul(Dxz, Dxz))), r_mul(C(2), r_mul(Dyz, Dyz))), r_mul(Dzz, Dzz));
        if (!(F1 > C(0) && F2 > C(0))) return C(0);
        const C num = r_mul(r_mul(C(0.325 * 0.325), dx2), r_mul(F1, sqrt(F1)));
        const C den = r_add(r_mul(r_mul(F2, F2), sqrt(F2)), r_mul(F1, sqrt(sqrt(F1))));
        return r_div(num, den);
    }
    // Vreman, c = 2.5 * 0.17^2: B = grad u^T grad u
    const C Bxx = r_add(r_add(r_mul(ux, ux), r_mul(uy, uy)), r_mul(uz, uz));
    const C Bxy = r_add(r_add(r_mul(ux, vx), r_mul(uy, vy)), r_mul(uz, vz));
    const C Bxz = r_add(r_add(r_mul(ux, wx), r_mul(uy, wy)), r_mul(uz, wz));
    const C Byy = r_add(r_add(r_mul(vx, vx), r_mul(vy, vy)), r_mul(vz, vz));
    const C Byz = r_add(r_add(r_mul(vx, wx), r_mul(vy, wy)), r_mul(vz, wz));
    const C Bzz = r_add(r_add(r_mul(wx, wx), r_mul(wy, wy)), r_mul(wz, wz));
    C Bb = r_add(r_mul(Bxx, Byy), -r_mul(Bxy, Bxy));
    if (dim == 3)
        Bb = r_add(r_add(r_add(Bb, r_add(r_mul(Bxx, Bzz), -r_mul(Bxz, Bxz))), r_mul(Byy, Bzz)), -r_mul(Byz, Byz));
    C aa = r_add(r_add(r_mul(ux, ux), r_mul(vx, vx)), r_add(r_mul(uy, uy), r_mul(vy, vy)));
    if (dim == 3)
        aa = r_add(aa, r_add(r_add(r_add(r_mul(wx, wx), r_mul(wy, wy)), r_add(r_mul(uz, uz), r_mul(vz, vz))),
                             r_mul(wz, wz)));
    if (!(aa > C(0))) return C(0);
    Bb = r_div(Bb, aa);
    return Bb > C(0) ? r_mul(r_mul(C(0.17 * 0.17 * 2.5), dx2), sqrt(Bb)) : C(0);
}

struct EddyArgs {
    const int *ids;
    int n;
    const int *nbr_child, *bmask;
    const void *f;
    void *nu_sgs;
    double dx;
    int model;
    const void *macro;   // multi-level: velocity from the macro rows [dim+1][nmc] instead of f
    long long nmc;
};

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(Geo<DIM>::MC) k_eddy(const EddyArgs a)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    constexpr int H = 6, HV = (DIM == 3) ? H * H * H : H * H;   // block plus a one-cell halo
    __shared__ C s[3][HV];
    const int b = a.ids[blockIdx.x];
    // Cu_ComputeEddyViscosity (solver_lbm_kernels_les.cu:313-323): listed
    // blocks that are leaves or not inside a solid (uniform per CTA)
    if (b < 0 || !(a.nbr_child[b] < 0 || a.bmask[b] != BLOCK_SOLID)) return;
    const int t = threadIdx.x;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    auto at = [&](int i, int j, int k) { return (i + 1) + H * (j + 1) + (DIM == 3 ? H * H * (k + 1) : 0); };
    if (a.macro) {
        // solver_lbm_kernels_les.cu:502-507: the macro rows as they stand
        const C *mr = static_cast<const C *>(a.macro) + (long long)b * MC + t;
        for (int d = 0; d < 3; d++) s[d][at(I, J, K)] = d < DIM ? mr[(d + 1) * a.nmc] : C(0);
    } else {
        const T *f = static_cast<const T *>(a.f) + (long long)b * BLK + t;
        C rho = 0, m[3] = {0, 0, 0};
#pragma unroll
        for (int p = 0; p < Q; p++) {
            const C fp = ST<T>::dec(f[lat_pb(DIM, p) * MC]) + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
            rho += fp;
#pragma unroll
            for (int d = 0; d < DIM; d++) m[d] += C(lat_c(DIM, d, p)) * fp;
        }
        for (int d = 0; d < 3; d++) s[d][at(I, J, K)] = d < DIM ? m[d] / rho : C(0);
    }
    __syncthreads();
    auto ext = [](C d1, C d2, C d3, C d4) {
        return r_add(r_add(r_add(r_mul(C(4), d1), r_mul(C(-6), d2)), r_mul(C(4), d3)), -d4);
    };
    for (int d = 0; d < DIM; d++) {
        C *u = s[d];
        if (I == 0) {
            u[at(-1, J, K)] = ext(u[at(0, J, K)], u[at(1, J, K)], u[at(2, J, K)], u[at(3, J, K)]);
            u[at(4, J, K)] = ext(u[at(3, J, K)], u[at(2, J, K)], u[at(1, J, K)], u[at(0, J, K)]);
        }
        if (J == 0) {
            u[at(I, -1, K)] = ext(u[at(I, 0, K)], u[at(I, 1, K)], u[at(I, 2, K)], u[at(I, 3, K)]);
            u[at(I, 4, K)] = ext(u[at(I, 3, K)], u[at(I, 2, K)], u[at(I, 1, K)], u[at(I, 0, K)]);
        }
        if (DIM == 3 && K == 0) {
            u[at(I, J, -1)] = ext(u[at(I, J, 0)], u[at(I, J, 1)], u[at(I, J, 2)], u[at(I, J, 3)]);
            u[at(I, J, 4)] = ext(u[at(I, J, 3)], u[at(I, J, 2)], u[at(I, J, 1)], u[at(I, J, 0)]);
        }
    }
    __syncthreads();
    const C dx = C(a.dx), two_dx = r_mul(C(2), dx);
    C gr[3][3] = {};   // gr[component][axis]
    for (int d = 0; d < DIM; d++) {
        gr[d][0] = r_div(r_add(s[d][at(I + 1, J, K)], -s[d][at(I - 1, J, K)]), two_dx);
        gr[d][1] = r_div(r_add(s[d][at(I, J + 1, K)], -s[d][at(I, J - 1, K)]), two_dx);
        if (DIM == 3) gr[d][2] = r_div(r_add(s[d][at(I, J, K + 1)], -s[d][at(I, J, K - 1)]), two_dx);
    }
    static_cast<C *>(a.nu_sgs)[(long long)b * MC + t] =
        les_model<C>(a.model, DIM, dx, gr[0][0], gr[0][1], gr[0][2], gr[1][0], gr[1][1], gr[1][2], gr[2][0],
                     gr[2][1], gr[2][2]);
}

// ---------------------------------------------------------------------------
// FP64 mass and momentum of the leaf fluid cells of one level; one partial
// per CTA, summed in a fixed order by k_sum_partials (deterministic).
struct MassArgs {
    const int *ids;
    int n;
    const void *f;
    const int *nbr_child, *cmask;
    double vol;
    double *partial;   // [gridDim.x][4]
};

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(256) k_mass(const MassArgs a)
{
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    __shared__ double s[4][256];
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long kap = gid / MC;
    const int t = (int)(gid % MC);
    double m = 0, mx = 0, my = 0, mz = 0;
    if (kap < a.n) {
        const int b = a.ids[kap];
        if (b >= 0 && a.nbr_child[b] < 0) {
            if (a.cmask[(long long)b * MC + t] != CELL_SOLID) {
                const T *f = static_cast<const T *>(a.f) + (long long)b * BLK + t;
#pragma unroll
                for (int p = 0; p < Q; p++) {
                    const double fp = (double)ST<T>::dec(f[lat_pb(DIM, p) * MC]) + (ST<T>::OFF ? lat_w(Q, p) : 0.0);
                    m += fp;
                    mx += lat_c(DIM, 0, p) * fp;
                    my += lat_c(DIM, 1, p) * fp;
                    mz += lat_c(DIM, 2, p) * fp;
                }
            }
        }
    }
    s[0][threadIdx.x] = m * a.vol;
    s[1][threadIdx.x] = mx * a.vol;
    s[2][threadIdx.x] = my * a.vol;
    s[3][threadIdx.x] = mz * a.vol;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int k = 0; k < 4; k++) s[k][threadIdx.x] += s[k][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x < 4) a.partial[blockIdx.x * 4 + threadIdx.x] = s[threadIdx.x][0];
}

// One CTA per component (gridDim.x = 4): strided partial sums, then a
// fixed-shape tree, so the result does not depend on scheduling.
__global__ void __launch_bounds__(256) k_sum_partials(const double *partial, int n, double *out)
{
    __shared__ double s[256];
    const int k = blockIdx.x;
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) acc += partial[(long long)i * 4 + k];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int st = 128; st > 0; st >>= 1) {
        if (threadIdx.x < st) s[threadIdx.x] += s[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = s[0];
}

// ---------------------------------------------------------------------------
// Step metadata rows (Meta<DIM>) of every block from the mesh arrays: the
// neighbour table in lexicographic slot order (util.h:100-101 map) and the
// flags of kernels.cu:236 (collide/stream) and :736 (boundary hook).
template <int DIM>
__global__ void k_build_meta(long long nmb, const int *nbr, const int *nbr_child, const int *bmask,
                             const int *onb, const int *onb_solid, const int *blk_solid, int *meta)
{
    constexpr int W = Meta<DIM>::W, QMAX = Geo<DIM>::QMAX;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nmb * W) return;
    const long long b = g / W;
    const int i = (int)(g % W);
    int v = 0;
    if (i < QMAX) {
        v = (i == center_slot(DIM)) ? (int)b : nbr[b + (long long)((DIM == 2) ? g_map2[i] : g_map3[i]) * nmb];
    } else if (i == Meta<DIM>::FLAGS) {
        if (nbr_child[b] < 0 || bmask[b] != BLOCK_SOLID) v |= META_ACTIVE;
        if (onb[b] == 1) v |= META_ONB;
        for (int k = 0; k < QMAX; k++)
            if (nbr[b + (long long)k * nmb] < 0) v |= META_CLOSED;
        if (onb_solid && onb[b] == 1 && onb_solid[b] >= 0) v |= META_WALL;
        if (blk_solid) {
            // A solid cell in the block or in a block of its neighbourhood:
            // the row-mapped step tests solid neighbours cell by cell there.
            bool near = blk_solid[b] != 0;
            for (int k = 0; k < QMAX && !near; k++) {
                const int nb = nbr[b + (long long)k * nmb];
                near = nb >= 0 && nb < nmb && blk_solid[nb] != 0;
            }
            if (near) v |= META_NEARSOLID;
        }
    }
    meta[g] = v;
}

// 1 per block holding a solid cell (any block of the pool).
template <int DIM>
__global__ void k_block_solid(long long nmb, const int *cmask, int *blk_solid)
{
    constexpr int MC = Geo<DIM>::MC;
    const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nmb) return;
    int s = 0;
    for (int t = 0; t < MC; t++) s |= (cmask[b * MC + t] == CELL_SOLID);
    blk_solid[b] = s;
}


// TMA-staged persistent variant (step_tma.cu).
template <int DIM, int Q, typename T>
int launch_step_tma(agal_ctx *c, const StepArgs &a);
template <int DIM, int Q, typename T>
int prepare_step_tma(agal_ctx *c);

template <int DIM, int Q, typename T> struct RunPrepare {
    static int run(agal_ctx *c) { return prepare_step_tma<DIM, Q, T>(c); }
};

template <int DIM, int Q, typename T, int CPT>
int launch_step(agal_ctx *c, const StepArgs &a, int n)
{
    constexpr int BPC = 256 / (Geo<DIM>::MC / CPT);
    const unsigned grid = (unsigned)((n + BPC - 1) / BPC);
    if (c->geometry_init)
        AGAL_CUDA(c, launch_pdl(k_step<DIM, Q, T, CPT, true>, dim3(grid), dim3(256), 0, c->stream, a));
    else
        AGAL_CUDA(c, launch_pdl(k_step<DIM, Q, T, CPT, false>, dim3(grid), dim3(256), 0, c->stream, a));
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

// Row-mapped variant (step_row.cu); built for FP32 and the half types (FP64
// contexts run variant 1 for it).
template <int DIM, int Q, typename T>
int launch_step_row(agal_ctx *c, const StepArgs &a, int n);
template <int DIM, int Q, typename T>
int launch_row_or_cell(agal_ctx *c, const StepArgs &a, int n)
{
    if constexpr (std::is_same<T, double>::value) return launch_step<DIM, Q, T, 1>(c, a, n);
    else return launch_step_row<DIM, Q, T>(c, a, n);
}
// Root-level tile step of 2D cases (step_tile.cu); AGAL_ERR_UNSUPPORTED when
// the case or level has no tile table.
template <int DIM, int Q, typename T>
int launch_step_tile(agal_ctx *c, const StepArgs &a, int L);
template <int DIM, int Q, typename T>
int launch_step_ptile(agal_ctx *c, const StepArgs &a, int L);

// Swap back the pushed entries of every link whose swap the reference's
// stream guard refuses (recorded by push_cell), then clear the list for the
// next step.  One CTA; the list is usually empty.  A list longer than its
// capacity leaves AGAL_ERR_STATE in the status word (reported by agal_sync).
template <typename T>
__global__ void __launch_bounds__(1024) k_stream_fixup(T *fo, int *count, const long long *list, int cap, int *status)
{
    pdl_wait();
    const int n = *count;
    const int m = n < cap ? n : cap;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const long long x = list[2 * i], y = list[2 * i + 1];
        const T vx = fo[x];
        fo[x] = fo[y];
        fo[y] = vx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n > cap) atomicCAS(status, 0, AGAL_ERR_STATE);
        *count = 0;
    }
}

// Batched fix-up: CTA i applies case i's list (A[i]); k_stream_fixup per case.
template <typename T>
__global__ void __launch_bounds__(1024) k_stream_fixup_batch(const StepArgs *__restrict__ A)
{
    const StepArgs &a = A[blockIdx.x];
    T *fo = static_cast<T *>(a.fout);
    const int n = *a.fix_count;
    const int m = n < a.fix_cap ? n : a.fix_cap;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const long long x = a.fix_list[2 * i], y = a.fix_list[2 * i + 1];
        const T vx = fo[x];
        fo[x] = fo[y];
        fo[y] = vx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n > a.fix_cap) atomicCAS(a.status, 0, AGAL_ERR_STATE);
        *a.fix_count = 0;
    }
}

template <int DIM, int Q, typename T> struct StepBatch {
    // One persistent launch over the chunks of n cases (dev_start[n] of them),
    // then the fix-ups of every case.  Grid: resident CTAs per SM x SMs.
    static int run(cudaStream_t s, const StepArgs *dev_args, const int *dev_start, int n, int total, bool solid,
                   bool fixup)
    {
        if (total > 0) {
            auto kern = solid ? k_step_batch<DIM, Q, T, true> : k_step_batch<DIM, Q, T, false>;
            int dev = 0, sms = 0, per_sm = 0;
            if (cudaGetDevice(&dev) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0) != cudaSuccess)
                return AGAL_ERR_CUDA;
            const int grid = std::min(total, std::max(per_sm, 1) * sms);
            kern<<<grid, 256, 0, s>>>(dev_args, dev_start, n);
        }
        if (fixup && n > 0) k_stream_fixup_batch<T><<<n, 1024, 0, s>>>(dev_args);
        return cudaGetLastError() == cudaSuccess ? AGAL_OK : AGAL_ERR_CUDA;
    }
};

template <int DIM, int Q, typename T> struct RunStep {
    // flip = false launches the kernel from the current buffer into the
    // other one without making it current (used by the autotuner: the step is
    // a pure function of the current buffer, so the state is unchanged).
    static int run(agal_ctx *c, int L, int cpt = 0, bool flip = true)
    {
        const int n = c->n_ids[L];
        if (n <= 0) {
            if (flip) c->cur[L] = 1 - c->cur[L];   // an empty level keeps the parity bookkeeping
            return AGAL_OK;
        }
        StepArgs a;
        a.ids = c->id_set + (long long)L * c->nmb;
        a.n = n;
        a.fin = c->F[c->cur[L]];
        a.fout = c->F[1 - c->cur[L]];
        a.meta = c->meta;
        a.cmask = c->cells_ID_mask;
        a.omega = c->dxf[L] / c->tau[L];
        if (sizeof(typename ST<T>::C) == 4) a.omega = (double)((float)c->dxf[L] / (float)c->tau[L]);
        a.u_ref = c->P.u_ref;
        a.bc_preset = c->P.bc_preset;
        a.mrt = (Q == 19 && c->P.collision == AGAL_MRT) ? 1 : 0;
        {
            const double sv[5] = {c->P.s1, c->P.s2, c->P.s3, c->P.s5, c->P.s6};
            for (int k = 0; k < 5; k++) a.s[k] = (sizeof(typename ST<T>::C) == 4) ? (double)(float)sv[k] : sv[k];
        }
        a.fix_count = c->fix_count;
        a.fix_list = c->fix_list;
        a.fix_cap = c->fix_cap;
        a.status = c->d_status;
        if (cpt <= 0) cpt = c->step_cpt;
        // The tile step covers the root level of 2D cases; elsewhere the row
        // variant takes its place.
        const bool tile = cpt == 5 && !std::is_same<T, double>::value && L == c->L0 && c->n_tiles > 0 && !c->nu_sgs;
        if (cpt == 5 && !tile) cpt = 4;
        // The push-tile step likewise; elsewhere one cell per thread.
        const bool ptile =
            cpt == 6 && !std::is_same<T, double>::value && L == c->L0 && c->n_ptiles > 0 && !c->nu_sgs;
        if (cpt == 6 && !ptile) cpt = 1;
        // Small one-shot grids apply the fix-ups in their last CTA (saves a
        // launch of a few µs per sub-step); large grids, the persistent
        // variant and levels with a wall step use the separate kernel.  The
        // tile step resolves refused swaps itself (no list).
        const bool wall = agal_wall_active(c) && (int)c->wall_n.size() > L && c->wall_n[L] > 0;
        const bool fused = cpt != 3 && !tile && !wall && n <= AGAL_FUSED_FIXUP_BLOCKS;
        a.fix_ticket = fused ? c->fix_count + 1 : nullptr;
        a.nu_sgs = c->nu_sgs;
        a.macro = agal_les_macros(c) ? c->macro : nullptr;
        a.nmc = c->nmc;
        a.sr = (c->storage == AGAL_STORE_FP16 || c->storage == AGAL_STORE_BF16) &&
               c->P.half_rounding == AGAL_ROUND_STOCHASTIC;
        a.sr_ctr = c->d_sr;
        a.sr_salt = (unsigned)c->sr_salt;
        a.nu = (sizeof(typename ST<T>::C) == 4) ? (double)(float)c->P.v0 : c->P.v0;
        a.dxL = (sizeof(typename ST<T>::C) == 4) ? (double)(float)c->dxf[L] : c->dxf[L];
        if (c->rec) {
            // Batch recording: the batched kernel steps this case with the
            // one-cell-per-thread body; its fix-ups follow in one batched launch.
            a.fix_ticket = nullptr;
            const int rc = agal_record_step(c, L, &a, sizeof(a), agal_step_batch_key(c), n, a.fin, a.fout);
            if (rc) return rc;
            if (flip) c->cur[L] = 1 - c->cur[L];
            c->sr_salt++;
            return AGAL_OK;
        }
        if (c->nu_sgs) {
            // The eddy viscosity of the current populations; the persistent
            // and row-mapped variants have no per-cell relaxation rate, so
            // LES steps one cell per thread.
            if (cpt >= 3) cpt = 1;
            EddyArgs e{a.ids, n, c->cblock_ID_nbr_child, c->cblock_ID_mask, a.fin, c->nu_sgs, a.dxL, c->P.S_LES,
                       a.macro, c->nmc};
            k_eddy<DIM, Q, T><<<n, Geo<DIM>::MC, 0, c->stream>>>(e);
            AGAL_CUDA(c, cudaGetLastError());
        }
        int rc = AGAL_OK;
        if (tile) {
            rc = launch_step_tile<DIM, Q, T>(c, a, L);
            if (rc == AGAL_ERR_UNSUPPORTED) return agal_set_err(c, rc, "tile step not available");
            if (rc) return rc;
            if (flip) c->cur[L] = 1 - c->cur[L];
            c->sr_salt++;
            return AGAL_OK;
        }
        rc = (cpt == 6)   ? launch_step_ptile<DIM, Q, T>(c, a, L)
             : (cpt == 4) ? launch_row_or_cell<DIM, Q, T>(c, a, n)
             : (cpt == 3) ? launch_step_tma<DIM, Q, T>(c, a)
             : (cpt == 2) ? launch_step<DIM, Q, T, 2>(c, a, n)
                          : launch_step<DIM, Q, T, 1>(c, a, n);
        if (rc) return rc;
        if (const int rw = agal_launch_wall_step(c, L, a.fin, a.fout)) return rw;
        if (!fused)
            AGAL_CUDA(c, launch_pdl(k_stream_fixup<T>, dim3(1), dim3(1024), 0, c->stream, static_cast<T *>(a.fout),
                                    c->fix_count, c->fix_list, c->fix_cap, c->d_status));
        AGAL_CUDA(c, cudaGetLastError());
        if (flip) c->cur[L] = 1 - c->cur[L];
        c->sr_salt++;
        return AGAL_OK;
    }
};

// Autotuner of the step kernel: times every variant (1: one cell per thread,
// 2: two cells per thread, 3: TMA-staged persistent pipeline, 4: one row of
// four cells per thread, 5: root-level tile step, 6: root-level push tiles)
// on level L's current state, writing only the scratch buffer.
template <int DIM, int Q, typename T> struct RunTune {
    static int run(agal_ctx *c, int L, int reps, float *ms_out)
    {
        if (c->n_ids[L] <= 0) return AGAL_OK;
        cudaEvent_t e0, e1;
        AGAL_CUDA(c, cudaEventCreate(&e0));
        AGAL_CUDA(c, cudaEventCreate(&e1));
        float best = 1e30f;
        int best_cpt = 1;
        for (int cpt = 1; cpt <= AGAL_STEP_VARIANTS; cpt++) {
            int rc = RunStep<DIM, Q, T>::run(c, L, cpt, false);   // warm-up
            if (rc) return rc;
            AGAL_CUDA(c, cudaEventRecord(e0, c->stream));
            for (int r = 0; r < reps; r++)
                if ((rc = RunStep<DIM, Q, T>::run(c, L, cpt, false))) return rc;
            AGAL_CUDA(c, cudaEventRecord(e1, c->stream));
            AGAL_CUDA(c, cudaEventSynchronize(e1));
            float ms = 0.f;
            AGAL_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
            ms /= (float)reps;
            if (ms_out) ms_out[cpt - 1] = ms;
            if (ms < best) { best = ms; best_cpt = cpt; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c->step_cpt = best_cpt;
        return AGAL_OK;
    }
};

template <int DIM, int Q, typename T> struct RunIc {
    static int run(agal_ctx *c, int L)
    {
        const int n = c->n_ids[L];
        if (n <= 0) return AGAL_OK;
        IcArgs a;
        a.ids = c->id_set + (long long)L * c->nmb;
        a.n = n;
        a.f0 = c->F[0];
        a.f1 = c->F[1];
        a.nmb = c->nmb;
        a.cmask = c->cells_ID_mask;
        a.fX = c->cblock_f_X;
        a.dxL = c->dxf[L];
        a.u_ref = c->P.u_ref;
        a.noise = c->P.ic_noise;
        a.seed = c->P.seed;
        a.ic_preset = c->P.ic_preset;
        a.L = L;
        const long long cells = (long long)n * Geo<DIM>::MC;
        k_set_ic<DIM, Q, T><<<(unsigned)((cells + 255) / 256), 256, 0, c->stream>>>(a);
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
};

template <int DIM, int Q, typename T> struct RunRefresh {
    static int run(agal_ctx *c, int L)
    {
        const int n = c->n_ids[L];
        if (n <= 0) return AGAL_OK;
        MacroArgs a;
        a.ids = c->id_set + (long long)L * c->nmb;
        a.n = n;
        a.f = c->F[c->cur[L]];
        a.macro = c->macro;
        a.nmc = c->nmc;
        const long long cells = (long long)n * Geo<DIM>::MC;
        k_refresh<DIM, Q, T><<<(unsigned)((cells + 255) / 256), 256, 0, c->stream>>>(a);
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
};

template <int DIM, int Q, typename T> struct RunMass {
    // Enqueue the sums and the copy of the four results to host_out.
    static int run(agal_ctx *c, double *host_out)
    {
        // Partials of all levels, laid out level after level.
        long long total = 0;
        std::vector<long long> grids(c->max_levels);
        for (int L = 0; L < c->max_levels; L++) {
            grids[L] = ((long long)c->n_ids[L] * Geo<DIM>::MC + 255) / 256;
            total += grids[L];
        }
        if (total > c->red_len) {
            if (c->red) cudaFree(c->red);
            c->red = nullptr;
            AGAL_CUDA(c, cudaMalloc(&c->red, sizeof(double) * 4 * (size_t)total));
            c->red_len = (int)total;
        }
        long long off = 0;
        for (int L = 0; L < c->max_levels; L++) {
            if (grids[L] == 0) continue;
            MassArgs a;
            a.ids = c->id_set + (long long)L * c->nmb;
            a.n = c->n_ids[L];
            a.f = c->F[c->cur[L]];
            a.nbr_child = c->cblock_ID_nbr_child;
            a.cmask = c->cells_ID_mask;
            a.vol = std::ldexp(1.0, -L * DIM);
            a.partial = c->red + 4 * off;
            k_mass<DIM, Q, T><<<(unsigned)grids[L], 256, 0, c->stream>>>(a);
            AGAL_CUDA(c, cudaGetLastError());
            off += grids[L];
        }
        if (total == 0) {
            AGAL_CUDA(c, cudaMemsetAsync(c->red_out, 0, 4 * sizeof(double), c->stream));
        } else {
            k_sum_partials<<<4, 256, 0, c->stream>>>(c->red, (int)total, c->red_out);
            AGAL_CUDA(c, cudaGetLastError());
        }
        AGAL_CUDA(c, cudaMemcpyAsync(host_out, c->red_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        return AGAL_OK;
    }
};

// ---------------------------------------------------------------------------
// Allocation-free mass/momentum: the same k_mass / k_sum_partials kernels with
// their partials and result in a fixed file-scope device array instead of
// the context's cudaMalloc'd scratch.  Every partial slot the final sum reads
// is written by k_mass in the same call, and k_sum_partials overwrites the
// result, so nothing has to start at zero.  All contexts on one device share
// the array: calls that overlap in time (other host threads or streams on the
// same device) race on it and must be serialised by the caller.
__device__ __align__(256) static double g_mass_scratch[4 * AGAL_MASS_NOALLOC_MAX_PARTIALS + 4];

// Device address of g_mass_scratch on the context's device, looked up on
// every call with that device current, so that a device reset (a new primary
// context) between calls is followed.  The lookup allocates nothing; the
// first one on a device may load the module and belongs before any stream
// capture.
static int mass_scratch_on(agal_ctx *c, double **out)
{
    const int dev = c->device;
    int prev = -1;
    AGAL_CUDA(c, cudaGetDevice(&prev));
    if (prev != dev) AGAL_CUDA(c, cudaSetDevice(dev));
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_mass_scratch);
    if (prev != dev) cudaSetDevice(prev);
    if (e != cudaSuccess) return agal_cuda_check(c, e, "cudaGetSymbolAddress(g_mass_scratch)");
    *out = static_cast<double *>(p);
    return AGAL_OK;
}

template <int DIM, int Q, typename T> struct RunMassNoAlloc {
    static int run(agal_ctx *c, double *out)
    {
        long long total = 0;
        std::vector<long long> grids(c->max_levels);
        for (int L = 0; L < c->max_levels; L++) {
            grids[L] = ((long long)c->n_ids[L] * Geo<DIM>::MC + 255) / 256;
            total += grids[L];
        }
        if (total > AGAL_MASS_NOALLOC_MAX_PARTIALS) {
            char m[256];
            std::snprintf(m, sizeof(m),
                          "agal_mass_momentum_noalloc: %lld partial sums exceed the static scratch of %d "
                          "(one per 256 active cells of each level); use agal_mass_momentum",
                          total, AGAL_MASS_NOALLOC_MAX_PARTIALS);
            return agal_set_err(c, AGAL_ERR_PARAM, m);
        }
        double *scratch = nullptr;
        int rc = mass_scratch_on(c, &scratch);
        if (rc) return rc;
        double *res = scratch + 4 * (size_t)AGAL_MASS_NOALLOC_MAX_PARTIALS;
        long long off = 0;
        for (int L = 0; L < c->max_levels; L++) {
            if (grids[L] == 0) continue;
            MassArgs a;
            a.ids = c->id_set + (long long)L * c->nmb;
            a.n = c->n_ids[L];
            a.f = c->F[c->cur[L]];
            a.nbr_child = c->cblock_ID_nbr_child;
            a.cmask = c->cells_ID_mask;
            a.vol = std::ldexp(1.0, -L * DIM);
            a.partial = scratch + 4 * off;
            k_mass<DIM, Q, T><<<(unsigned)grids[L], 256, 0, c->stream>>>(a);
            AGAL_CUDA(c, cudaGetLastError());
            off += grids[L];
        }
        if (total == 0) {
            AGAL_CUDA(c, cudaMemsetAsync(res, 0, 4 * sizeof(double), c->stream));
        } else {
            k_sum_partials<<<4, 256, 0, c->stream>>>(scratch, (int)total, res);
            AGAL_CUDA(c, cudaGetLastError());
        }
        double h[4];
        AGAL_CUDA(c, cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
        AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
        out[0] = h[0];
        out[1] = h[1];
        out[2] = h[2];
        if (DIM == 3) out[3] = h[3];
        return AGAL_OK;
    }
};

}  // namespace agal

extern "C" int agal_mass_momentum_noalloc(agal_ctx *c, double *out)
{
    if (!c || !out) return AGAL_ERR_PARAM;
    return agal::dispatch<agal::RunMassNoAlloc>(c, out);
}

int agal_launch_step(agal_ctx *c, int L) { return agal::dispatch<agal::RunStep>(c, L, 0, true); }
int agal_launch_tune(agal_ctx *c, int L, int reps, float *ms)
{
    int rc = agal::dispatch<agal::RunPrepare>(c);
    return rc ? rc : agal::dispatch<agal::RunTune>(c, L, reps, ms);
}
int agal_prepare_step(agal_ctx *c) { return agal::dispatch<agal::RunPrepare>(c); }

int agal_build_meta(agal_ctx *c)
{
    const long long tot = c->nmb * (c->dim == 2 ? agal::Meta<2>::W : agal::Meta<3>::W);
    const unsigned grid = (unsigned)((tot + 255) / 256);
    // Wall blocks leave the main step kernels only when k_step_wall takes them.
    const int *wall = agal_wall_active(c) ? c->onb_solid : nullptr;
    const int *bs = nullptr;
    if (c->geometry_init) {
        if (!c->blk_solid) AGAL_CUDA(c, cudaMalloc(&c->blk_solid, sizeof(int) * (size_t)c->nmb));
        const unsigned gb = (unsigned)((c->nmb + 255) / 256);
        if (c->dim == 2) agal::k_block_solid<2><<<gb, 256, 0, c->stream>>>(c->nmb, c->cells_ID_mask, c->blk_solid);
        else agal::k_block_solid<3><<<gb, 256, 0, c->stream>>>(c->nmb, c->cells_ID_mask, c->blk_solid);
        bs = c->blk_solid;
    }
    if (c->dim == 2)
        agal::k_build_meta<2><<<grid, 256, 0, c->stream>>>(c->nmb, c->cblock_ID_nbr, c->cblock_ID_nbr_child,
                                                           c->cblock_ID_mask, c->cblock_ID_onb, wall, bs, c->meta);
    else
        agal::k_build_meta<3><<<grid, 256, 0, c->stream>>>(c->nmb, c->cblock_ID_nbr, c->cblock_ID_nbr_child,
                                                           c->cblock_ID_mask, c->cblock_ID_onb, wall, bs, c->meta);
    AGAL_CUDA(c, cudaGetLastError());
    int rc;
    if ((rc = agal_build_tiles(c))) return rc;
    if (c->amr && (rc = agal_build_iface_lists(c))) return rc;
    if (c->onb_solid) return agal_build_wall_lists(c);
    return AGAL_OK;
}
int agal_launch_set_ic(agal_ctx *c, int L)
{
    // Cu_SetInitialConditions also writes the level's macro rows
    // (solver_lbm_kernels.cu:70-74); in LES macro mode they are refreshed from
    // the new populations.
    const int rc = agal::dispatch<agal::RunIc>(c, L);
    return rc ? rc : agal_les_refresh(c, L);
}

int agal_les_refresh(agal_ctx *c, int L) { return agal_les_macros(c) ? agal_launch_refresh(c, L) : AGAL_OK; }
int agal_launch_refresh(agal_ctx *c, int L) { return agal::dispatch<agal::RunRefresh>(c, L); }
int agal_launch_mass_async(agal_ctx *c, double *host_out) { return agal::dispatch<agal::RunMass>(c, host_out); }
int agal_launch_mass(agal_ctx *c, double *out)
{
    double h[4];
    int rc = agal_launch_mass_async(c, h);
    if (rc) return rc;
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < c->dim + 1; k++) out[k] = h[k];
    return AGAL_OK;
}

// Batched step of many cases (batch.cu): `key` is agal_step_batch_key of the
// cases, all of one velocity set and storage; fixup_only launches the
// batched fix-ups instead of the step.
int agal_step_batch_key(const agal_ctx *c) { return (c->Q * 8 + c->storage) * 2 + (c->geometry_init ? 1 : 0); }

int agal_launch_step_batch(int key, cudaStream_t s, const void *dev_args, const int *dev_start, int n, int total,
                           int fixup_only)
{
    const bool solid = key & 1;
    const int storage = (key >> 1) % 8, Q = (key >> 1) / 8;
    const auto *A = static_cast<const agal::StepArgs *>(dev_args);
    auto go = [&](auto tag) -> int {
        using T = decltype(tag);
        switch (Q) {
        case 9: return agal::StepBatch<2, 9, T>::run(s, A, dev_start, n, fixup_only ? 0 : total, solid, fixup_only);
        case 19: return agal::StepBatch<3, 19, T>::run(s, A, dev_start, n, fixup_only ? 0 : total, solid, fixup_only);
        case 27: return agal::StepBatch<3, 27, T>::run(s, A, dev_start, n, fixup_only ? 0 : total, solid, fixup_only);
        default: return AGAL_ERR_PARAM;
        }
    };
    switch (storage) {
    case AGAL_STORE_FP32: return go(float{});
    case AGAL_STORE_FP64: return go(double{});
    case AGAL_STORE_FP16: return go(__half{});
    case AGAL_STORE_BF16: return go(__nv_bfloat16{});
    default: return AGAL_ERR_PARAM;
    }
}
