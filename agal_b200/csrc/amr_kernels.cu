// Level-interface transfers and the solution-based refinement criterion.
//
//   k_interp     coarse-to-fine: the parent's cells (populations rescaled by
//                tau_{L+1}/tau_L around their equilibrium) interpolated
//                bilinearly/trilinearly or by tensor-product cubic Lagrange
//                into the ghost cells of its children (INTERP_INTERFACE) or
//                into every cell of newly added children (INTERP_ADDED).
//                Cu_Interpolate_Linear / Cu_Interpolate_Cubic,
//                solver_lbm_kernels_comm.cu:15-138, 406-640.
//   k_average    fine-to-coarse: each parent cell the mean of the 2^d child
//                cells under it, rescaled by tau_L/tau_{L+1}, where the child
//                group's corner cell qualifies (Cu_Average, :174-347).
//   k_criterion  velocity-gradient criterion per block (vorticity magnitude or
//                Q, floor(log2)), block maximum, refine/coarsen marks
//                (Cu_ComputeRefCriteria, solver_lbm_criterion.cu:440-592).
//
// The transfers compute each cell's macros from its populations with the
// arithmetic of k_refresh, so they equal what the reference reads from the
// macro rows its S_Interpolate / S_Average refresh just wrote.  One CTA per
// parent block; NCH x M_CBLOCK threads (one per child cell).
// Half-precision storage keeps weight offsets g = f - w: both transfers are
// affine with weights summing to one, so they run on g directly, with the
// equilibrium difference formed as a small quantity.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "ctx.h"
#include "lattice.cuh"
#include "storage.cuh"
#include "step_common.cuh"
#include "dispatch.cuh"

namespace agal {

// Macros of one cell with k_refresh's operation order; drho = rho - 1 in the
// offset form (exact sum of the stored offsets), else rho.
template <int DIM, int Q, typename T>
__device__ __forceinline__ void cell_macros(const T *__restrict__ f, typename ST<T>::C &rho, typename ST<T>::C &drho,
                                            typename ST<T>::C &u, typename ST<T>::C &v, typename ST<T>::C &w)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC;
    C r = 0, d = 0, x = 0, y = 0, z = 0;
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const C g = ST<T>::dec(f[lat_pb(DIM, p) * MC]);
        const C fp = g + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        r += fp;
        d += g;
        x += C(lat_c(DIM, 0, p)) * fp;
        y += C(lat_c(DIM, 1, p)) * fp;
        if (DIM == 3) z += C(lat_c(DIM, 2, p)) * fp;
    }
    rho = r;
    drho = ST<T>::OFF ? d : r;
    u = x / r;
    v = y / r;
    w = (DIM == 3) ? z / r : C(0);
}

// (feq_p - w_p) in the offset form, feq_p otherwise.
template <int DIM, int Q, typename C, bool OFF>
__device__ __forceinline__ C feq_stored(int p, C rho, C drho, C u, C v, C w)
{
    const C wp = C(lat_w(Q, p));
    const C cu = C(lat_c(DIM, 0, p)) * u + C(lat_c(DIM, 1, p)) * v + C(lat_c(DIM, 2, p)) * w;
    const C usq = u * u + v * v + w * w;
    const C poly = C(3) * cu + C(4.5) * cu * cu - C(1.5) * usq;
    if (OFF) return wp * (drho + rho * poly);
    return wp * rho * (C(1) + poly);
}

// Lagrange weight of node a (nodes at 0, 1/3, 2/3, 1 of the parent block) at
// child position m (centres at -1/12 + m/6).
__host__ __device__ constexpr double lag_w(int a, int m)
{
    double x = -1.0 / 12.0 + m / 6.0, r = 1.0;
    for (int k = 0; k < 4; k++)
        if (k != a) r *= (x - k / 3.0) / (a / 3.0 - k / 3.0);
    return r;
}

// Seed of a transfer launch: the coarse-step counter and the launch's salt.
__device__ __forceinline__ unsigned transfer_seed(int sr, const unsigned *ctr, unsigned salt)
{
    return sr ? (*ctr) * 0x9E3779B9u + salt * 0x85EBCA77u + 0x27D4EB2Fu : 0u;
}

struct InterpArgs {
    const int *ids;
    int n;
    const void *fpar;      // level L current buffer
    void *fch;             // level L+1 current buffer
    const int *nbr_child;  // row 0: first child
    const int *bmask, *ref, *cmask;
    double ratio;          // tau_{L+1} / tau_L in the compute type
    int var;               // AGAL_INTERP_INTERFACE / AGAL_INTERP_ADDED
    // stochastic rounding of half-precision offsets (step_common.cuh)
    int sr;
    const unsigned *sr_ctr;
    unsigned sr_salt;
};

// Interpolation into the children of block a.ids[blk].
template <int DIM, int Q, typename T, bool CUBIC>
__device__ __forceinline__ void interp_body(const InterpArgs &a, int blk)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC, NT = Geo<DIM>::NCH * Geo<DIM>::MC;
    constexpr bool OFF = ST<T>::OFF;
    // The parent's populations as stored, its cells' macros, and the rescaled
    // values of every direction: staged once, so that the per-direction
    // interpolation below needs no barrier.
    __shared__ T sRaw[BLK];
    __shared__ C sMac[5][MC];
    __shared__ C sF[Q][MC];
    __shared__ C sW[4][8];
    // Uniform per CTA: every early return below depends on blockIdx only.
    // The mesh arrays are read before the wait for the predecessor (no kernel
    // that launches this one early writes them), the populations after it.
    const int b = a.ids[blk];
    if (b < 0) return;
    const bool b1 = a.var == AGAL_INTERP_INTERFACE && a.bmask[b] == BLOCK_INTERFACE;
    const bool b2 = a.var == AGAL_INTERP_ADDED && a.ref[b] == REF_MARK_REFINE;
    if (!(b1 || b2)) return;
    const int bc = a.nbr_child[b];
    if (bc < 0) return;
    const int tid = threadIdx.x;
    if (CUBIC && tid < 32) sW[tid / 8][tid % 8] = C(lag_w(tid / 8, tid % 8));
    const bool ghost = a.cmask[(long long)(bc + tid / MC) * MC + tid % MC] == CELL_GHOST;
    pdl_wait();
    const T *fp = static_cast<const T *>(a.fpar) + (long long)b * BLK;
    for (int i = tid; i < BLK; i += NT) sRaw[i] = fp[i];
    __syncthreads();
    if (tid < MC) {
        C rho, drho, u, v, w;
        cell_macros<DIM, Q, T>(sRaw + tid, rho, drho, u, v, w);
        sMac[0][tid] = rho;
        sMac[1][tid] = drho;
        sMac[2][tid] = u;
        sMac[3][tid] = v;
        sMac[4][tid] = w;
    }
    __syncthreads();
    const C ratio = C(a.ratio);
    for (int i = tid; i < BLK; i += NT) {
        const int p = i / MC, cl = i % MC;
        const C g = ST<T>::dec(sRaw[lat_pb(DIM, p) * MC + cl]);
        const C e = feq_stored<DIM, Q, C, OFF>(p, sMac[0][cl], sMac[1][cl], sMac[2][cl], sMac[3][cl], sMac[4][cl]);
        sF[p][cl] = e + (g - e) * ratio;
    }
    __syncthreads();
    if (!(a.var == AGAL_INTERP_ADDED || ghost)) return;
    // Child cell of this thread.
    T *fc = static_cast<T *>(a.fch);
    const int ch = tid / MC, t = tid % MC;
    const int ci = ch & 1, cj = (ch >> 1) & 1, ck = (ch >> 2) & 1;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    const long long cell = (long long)(bc + ch) * BLK + t;
    const unsigned rnd = a.sr ? sr_cell((long long)(bc + ch) * MC + t, transfer_seed(a.sr, a.sr_ctr, a.sr_salt)) : 0u;
#pragma unroll 1
    for (int p = 0; p < Q; p++) {
        const C *F = sF[p];
        C val;
        if (!CUBIC) {
            const int s = 2 * ci + 8 * cj + 32 * ck;
            const C x = C(-0.25) + C(0.5) * C(I), y = C(-0.25) + C(0.5) * C(J);
            if (DIM == 2) {
                val = F[s] + (F[1 + s] - F[s]) * x + (F[4 + s] - F[s]) * y + (F[5 + s] - F[4 + s] - F[1 + s] + F[s]) * x * y;
            } else {
                const C z = C(-0.25) + C(0.5) * C(K);
                val = F[s] + (F[1 + s] - F[s]) * x + (F[4 + s] - F[s]) * y + (F[16 + s] - F[s]) * z +
                      (F[5 + s] - F[1 + s] - F[4 + s] + F[s]) * x * y +
                      (F[17 + s] - F[1 + s] - F[16 + s] + F[s]) * x * z +
                      (F[20 + s] - F[4 + s] - F[16 + s] + F[s]) * y * z +
                      (F[21 + s] + F[1 + s] + F[4 + s] + F[16 + s] - F[5 + s] - F[17 + s] - F[20 + s] - F[s]) * x * y * z;
            }
        } else {
            const int mx = I + 4 * ci, my = J + 4 * cj, mz = K + 4 * ck;
            val = C(0);
            if (DIM == 2) {
#pragma unroll
                for (int bj = 0; bj < 4; bj++) {
                    C row = C(0);
#pragma unroll
                    for (int ai = 0; ai < 4; ai++) row += sW[ai][mx] * F[ai + 4 * bj];
                    val += sW[bj][my] * row;
                }
            } else {
#pragma unroll
                for (int ck2 = 0; ck2 < 4; ck2++) {
                    C pl = C(0);
#pragma unroll
                    for (int bj = 0; bj < 4; bj++) {
                        C row = C(0);
#pragma unroll
                        for (int ai = 0; ai < 4; ai++) row += sW[ai][mx] * F[ai + 4 * bj + 16 * ck2];
                        pl += sW[bj][my] * row;
                    }
                    val += sW[ck2][mz] * pl;
                }
            }
        }
        fc[cell + lat_pb(DIM, p) * MC] = enc_r<T>(val, rnd * sr_dir(p), a.sr);
    }
}

template <int DIM, int Q, typename T, bool CUBIC>
__global__ void __launch_bounds__(Geo<DIM>::NCH * Geo<DIM>::MC) k_interp(const InterpArgs a)
{
    interp_body<DIM, Q, T, CUBIC>(a, blockIdx.x);
}

// Batched forms (the batch's work list): item w is block w - start[i] of case
// i's list, transferred with that case's arguments A[i].
template <int DIM, int Q, typename T, bool CUBIC>
__global__ void __launch_bounds__(Geo<DIM>::NCH * Geo<DIM>::MC)
k_interp_batch(const InterpArgs *__restrict__ A, const int *__restrict__ start, int n_cases)
{
    const int total = start[n_cases];
    int i = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        while (start[i + 1] <= w) i++;
        const InterpArgs a = A[i];
        interp_body<DIM, Q, T, CUBIC>(a, w - start[i]);
        __syncthreads();   // the shared staging is refilled for the next item
    }
}

struct AverageArgs {
    const int *ids;
    int n;
    void *fpar;            // level L current buffer
    const void *fch;       // level L+1 current buffer
    const int *nbr_child, *bmask, *cmask;
    double ratio;          // tau_L / tau_{L+1} in the compute type
    int var;               // AGAL_AVERAGE_INTERFACE / _BLOCK / _GRID
    int sr;
    const unsigned *sr_ctr;
    unsigned sr_salt;
    // Non-null: the launch's last CTA advances the rounding counter once all
    // CTAs have read it (the coarse step's tick), ticket counting the CTAs.
    unsigned *tick;
    int *ticket;
};


// Averaging of the children of block a.ids[blk] into it.
template <int DIM, int Q, typename T>
__device__ __forceinline__ void average_body(const AverageArgs &a, int blk)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, NCH = Geo<DIM>::NCH, BLK = Q * MC;
    constexpr bool OFF = ST<T>::OFF;
    __shared__ C sg[2][NCH * MC];   // double-buffered: one barrier per direction
    __shared__ int smask[NCH * MC];
    // Mesh arrays before the wait for the predecessor, populations after it.
    const int b = a.ids[blk];
    if (b < 0) return;
    const int bc = a.nbr_child[b];
    if (!(bc > -1 && (a.var == AGAL_AVERAGE_GRID || a.bmask[b] == BLOCK_INTERFACE))) return;
    const int tid = threadIdx.x;
    const T *fc = static_cast<const T *>(a.fch) + (long long)bc * BLK;   // children are consecutive IDs
    const int ch = tid / MC, t = tid % MC;
    const T *own = fc + (long long)ch * BLK + t;
    int m = a.cmask[(long long)(bc + ch) * MC + t];
    pdl_wait();
    C rho, drho, u, v, w;
    cell_macros<DIM, Q, T>(own, rho, drho, u, v, w);
    if (a.var > 0 && m < 2) m = 1;
    smask[tid] = m;
    const C ratio = C(a.ratio);
    // Parent cell of this thread (tid < MC): its quadrant and the corner cell
    // of the 2^d child cells under it.
    const int I = tid & 3, J = (tid >> 2) & 3, K = (DIM == 3) ? ((tid >> 4) & 3) : 0;
    const int qd = (I >= 2 ? 1 : 0) + (J >= 2 ? 2 : 0) + ((DIM == 3 && K >= 2) ? 4 : 0);
    const int c0 = 2 * (I & 1) + 8 * (J & 1) + (DIM == 3 ? 32 * (K & 1) : 0);
    T *fp = static_cast<T *>(a.fpar) + (long long)b * BLK + tid;
    const unsigned rnd = (a.sr && tid < MC) ? sr_cell((long long)b * MC + tid, transfer_seed(a.sr, a.sr_ctr, a.sr_salt)) : 0u;
    for (int p = 0; p < Q; p++) {
        const int slot = lat_pb(DIM, p);
        C *buf = sg[p & 1];
        {
            const C g = ST<T>::dec(own[slot * MC]);
            const C e = feq_stored<DIM, Q, C, OFF>(p, rho, drho, u, v, w);
            buf[tid] = e + (g - e) * ratio;
        }
        // the buffer written here was last read two directions ago, before
        // the previous barrier
        __syncthreads();
        if (tid < MC && smask[qd * MC + c0] == 1) {
            const C *s = buf + qd * MC + c0;
            C val;
            if (DIM == 2) val = C(0.25) * (s[0] + s[1] + s[4] + s[5]);
            else val = C(0.125) * (s[0] + s[1] + s[4] + s[5] + s[16] + s[17] + s[20] + s[21]);
            fp[slot * MC] = enc_r<T>(val, rnd * sr_dir(p), a.sr);
        }
    }
}

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(Geo<DIM>::NCH * Geo<DIM>::MC) k_average(const AverageArgs a)
{
    average_body<DIM, Q, T>(a, blockIdx.x);
    if (a.tick) {
        __syncthreads();   // every thread of this CTA is past its read of the counter
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(a.ticket, 1) == (int)gridDim.x - 1) {
                *a.ticket = 0;
                atomicAdd(a.tick, 1u);
            }
        }
    }
}

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(Geo<DIM>::NCH * Geo<DIM>::MC)
k_average_batch(const AverageArgs *__restrict__ A, const int *__restrict__ start, int n_cases)
{
    const int total = start[n_cases];
    int i = 0;
    for (int w = blockIdx.x; w < total; w += gridDim.x) {
        while (start[i + 1] <= w) i++;
        const AverageArgs a = A[i];
        average_body<DIM, Q, T>(a, w - start[i]);
        __syncthreads();   // the shared buffers are refilled for the next item
    }
}

struct CriterionArgs {
    int idm;
    long long nmb, nmc;
    const void *macro;     // [dim+1][n_maxcells] of the compute type
    const int *cmask, *level, *nbr;
    int *ref;
    double dx;             // level-0 spacing (the reference passes dxf_vec[0])
    int criterion;         // S_CRITERION: 0 vorticity magnitude, 1 Q
    double nrs, nri, nrm;  // N_REFINE_START / _INC / _MAX
    int mli;               // MAX_LEVELS_INTERIOR
};

// Fourth-order extrapolation to the one-cell halo (util_math.h:26-116).
template <typename C>
__device__ __forceinline__ C extrap4(C a, C b, C c, C d)
{
    return C(4) * a + C(-6) * b + C(4) * c + C(-1) * d;
}

template <int DIM>
__device__ __forceinline__ int halo_ix(int i, int j, int k)
{
    return (i + 1) + 6 * (j + 1) + (DIM == 3 ? 36 * (k + 1) : 0);
}

template <int DIM, typename C>
__global__ void __launch_bounds__(Geo<DIM>::MC) k_criterion(const CriterionArgs a)
{
    constexpr int MC = Geo<DIM>::MC, QMAX = Geo<DIM>::QMAX, H = (DIM == 2) ? 36 : 216;
    __shared__ C s[DIM][H];
    __shared__ C sW[MC];
    const int b = blockIdx.x;
    if (a.ref[b] == REF_INACTIVE) return;   // uniform per CTA
    const int t = threadIdx.x;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    const C *m = static_cast<const C *>(a.macro);
    const long long cell = (long long)b * MC + t;
#pragma unroll
    for (int d = 0; d < DIM; d++) s[d][halo_ix<DIM>(I, J, K)] = m[(long long)(1 + d) * a.nmc + cell];
    __syncthreads();
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        C *q = s[d];
        if (I == 0) {
            q[halo_ix<DIM>(-1, J, K)] = extrap4(q[halo_ix<DIM>(0, J, K)], q[halo_ix<DIM>(1, J, K)],
                                                q[halo_ix<DIM>(2, J, K)], q[halo_ix<DIM>(3, J, K)]);
            q[halo_ix<DIM>(4, J, K)] = extrap4(q[halo_ix<DIM>(3, J, K)], q[halo_ix<DIM>(2, J, K)],
                                               q[halo_ix<DIM>(1, J, K)], q[halo_ix<DIM>(0, J, K)]);
        }
        if (J == 0) {
            q[halo_ix<DIM>(I, -1, K)] = extrap4(q[halo_ix<DIM>(I, 0, K)], q[halo_ix<DIM>(I, 1, K)],
                                                q[halo_ix<DIM>(I, 2, K)], q[halo_ix<DIM>(I, 3, K)]);
            q[halo_ix<DIM>(I, 4, K)] = extrap4(q[halo_ix<DIM>(I, 3, K)], q[halo_ix<DIM>(I, 2, K)],
                                               q[halo_ix<DIM>(I, 1, K)], q[halo_ix<DIM>(I, 0, K)]);
        }
        if (DIM == 3 && K == 0) {
            q[halo_ix<DIM>(I, J, -1)] = extrap4(q[halo_ix<DIM>(I, J, 0)], q[halo_ix<DIM>(I, J, 1)],
                                                q[halo_ix<DIM>(I, J, 2)], q[halo_ix<DIM>(I, J, 3)]);
            q[halo_ix<DIM>(I, J, 4)] = extrap4(q[halo_ix<DIM>(I, J, 3)], q[halo_ix<DIM>(I, J, 2)],
                                               q[halo_ix<DIM>(I, J, 1)], q[halo_ix<DIM>(I, J, 0)]);
        }
    }
    __syncthreads();
    C g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // g[component][axis]
    const C dxL = C(a.dx);
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const C *q = s[d];
        const C ex = q[halo_ix<DIM>(I + 1, J, K)] - q[halo_ix<DIM>(I - 1, J, K)];
        const C ey = q[halo_ix<DIM>(I, J + 1, K)] - q[halo_ix<DIM>(I, J - 1, K)];
        if (DIM == 2) {
            // the 2D kernel divides by the double 2.0*dx_L (criterion.cu:502-505)
            g[d][0] = C((double)ex / (2.0 * (double)dxL));
            g[d][1] = C((double)ey / (2.0 * (double)dxL));
        } else {
            const C ez = q[halo_ix<DIM>(I, J, K + 1)] - q[halo_ix<DIM>(I, J, K - 1)];
            g[d][0] = ex / (C(2) * dxL);
            g[d][1] = ey / (C(2) * dxL);
            g[d][2] = ez / (C(2) * dxL);
        }
    }
    const C uX = g[0][0], uY = g[0][1], uZ = g[0][2], vX = g[1][0], vY = g[1][1], vZ = g[1][2];
    const C wX = g[2][0], wY = g[2][1], wZ = g[2][2];
    C W = C(0);
    if (a.criterion == 0) W = floor(log2(sqrt((wY - vZ) * (wY - vZ) + (uZ - wX) * (uZ - wX) + (vX - uY) * (vX - uY))));
    if (a.criterion == 1)
        W = floor(log2(fabs(C(0.5) * (uX * uX + vY * vY + wZ * wZ + C(2) * (uY * vX + uZ * wX + wY * vZ)))));
    if (a.cmask[cell] == CELL_GHOST) W = C(0);
    sW[t] = W;
    __syncthreads();
    for (int st = MC / 2; st > 0; st >>= 1) {
        if (t < st) sW[t] = fmax(sW[t], sW[t + st]);
        __syncthreads();
    }
    if (t == 0) {
        C Wm = sW[0];
        if (Wm > C(a.nrm)) Wm = C(a.nrm);
        const int rk = a.ref[b], lk = a.level[b];
        int Ld = a.mli - 1;
        for (int p = 1; p <= a.mli - 1; p++)
            if (Wm < C(a.nrs) - C(a.nri) * C(p)) Ld = (a.mli - 1) - p;
        bool eligible = true;
        for (int p = 0; p < QMAX; p++)
            if (a.nbr[b + (long long)p * a.nmb] == N_SKIPID) eligible = false;
        if (eligible && lk != a.mli - 1 && rk == REF_UNREFINED && Ld > lk) a.ref[b] = REF_MARK_REFINE;
        if (rk == REF_REFINED && Ld < lk + 1) a.ref[b] = REF_MARK_COARSEN;
    }
}

// ---------------------------------------------------------------------------
// Percentile criterion (S_CRITERION = AGAL_CRITERION_PERCENTILE; no reference
// counterpart).  k_wmax: maximum vorticity magnitude of each block over its
// non-ghost cells at the block's own spacing, every operation explicitly
// rounded in the order the oracle writes it.  The ref_pct_hi / ref_pct_lo
// quantiles of the leaf blocks' values are then selected exactly on the
// device by a radix select over the bits of the (non-negative, so
// order-preserving) FP64 keys (one CTA, 8 bits per pass, on pools of up to
// 65,536 blocks; 16 bits per pass over the whole grid beyond), and
// k_pct_mark marks.
__device__ __forceinline__ float r_sqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ double r_sqrt(double a) { return __dsqrt_rn(a); }

struct PctState {
    unsigned long long prefix[2];   // key bits selected so far, per quantile
    int k[2];                       // rank still sought within the prefix
    int n;                          // leaf blocks in the population
};

struct WmaxArgs {
    int idm;
    long long nmc;
    const void *macro;
    const int *cmask, *level, *ref, *nbr_child;
    double dx[16];                  // dx_L per level, in the compute type's value
    double *wval;                   // [idm]: block maximum (-1 for inactive)
    int *pop;                       // [idm]: 1 for a leaf block
    PctState *st;
};

template <typename C>
__device__ __forceinline__ C xpol4_rn(C a, C b, C c, C d)
{
    return r_add(r_add(r_add(r_mul(C(4), a), r_mul(C(-6), b)), r_mul(C(4), c)), r_mul(C(-1), d));
}

template <int DIM, typename C>
__global__ void __launch_bounds__(Geo<DIM>::MC) k_wmax(const WmaxArgs a)
{
    constexpr int MC = Geo<DIM>::MC, H = (DIM == 2) ? 36 : 216;
    __shared__ C s[DIM][H];
    __shared__ C sW[MC];
    const int b = blockIdx.x;
    const int t = threadIdx.x;
    if (a.ref[b] == REF_INACTIVE) {   // uniform per CTA
        if (t == 0) {
            a.wval[b] = -1.0;
            a.pop[b] = 0;
        }
        return;
    }
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    const C *m = static_cast<const C *>(a.macro);
    const long long cell = (long long)b * MC + t;
#pragma unroll
    for (int d = 0; d < DIM; d++) s[d][halo_ix<DIM>(I, J, K)] = m[(long long)(1 + d) * a.nmc + cell];
    __syncthreads();
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        C *q = s[d];
        if (I == 0) {
            q[halo_ix<DIM>(-1, J, K)] = xpol4_rn(q[halo_ix<DIM>(0, J, K)], q[halo_ix<DIM>(1, J, K)],
                                                 q[halo_ix<DIM>(2, J, K)], q[halo_ix<DIM>(3, J, K)]);
            q[halo_ix<DIM>(4, J, K)] = xpol4_rn(q[halo_ix<DIM>(3, J, K)], q[halo_ix<DIM>(2, J, K)],
                                                q[halo_ix<DIM>(1, J, K)], q[halo_ix<DIM>(0, J, K)]);
        }
        if (J == 0) {
            q[halo_ix<DIM>(I, -1, K)] = xpol4_rn(q[halo_ix<DIM>(I, 0, K)], q[halo_ix<DIM>(I, 1, K)],
                                                 q[halo_ix<DIM>(I, 2, K)], q[halo_ix<DIM>(I, 3, K)]);
            q[halo_ix<DIM>(I, 4, K)] = xpol4_rn(q[halo_ix<DIM>(I, 3, K)], q[halo_ix<DIM>(I, 2, K)],
                                                q[halo_ix<DIM>(I, 1, K)], q[halo_ix<DIM>(I, 0, K)]);
        }
        if (DIM == 3 && K == 0) {
            q[halo_ix<DIM>(I, J, -1)] = xpol4_rn(q[halo_ix<DIM>(I, J, 0)], q[halo_ix<DIM>(I, J, 1)],
                                                 q[halo_ix<DIM>(I, J, 2)], q[halo_ix<DIM>(I, J, 3)]);
            q[halo_ix<DIM>(I, J, 4)] = xpol4_rn(q[halo_ix<DIM>(I, J, 3)], q[halo_ix<DIM>(I, J, 2)],
                                                q[halo_ix<DIM>(I, J, 1)], q[halo_ix<DIM>(I, J, 0)]);
        }
    }
    __syncthreads();
    const C h2 = r_mul(C(2), C(a.dx[a.level[b]]));
    C g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        const C *q = s[d];
        g[d][0] = r_div(r_add(q[halo_ix<DIM>(I + 1, J, K)], -q[halo_ix<DIM>(I - 1, J, K)]), h2);
        g[d][1] = r_div(r_add(q[halo_ix<DIM>(I, J + 1, K)], -q[halo_ix<DIM>(I, J - 1, K)]), h2);
        if (DIM == 3) g[d][2] = r_div(r_add(q[halo_ix<DIM>(I, J, K + 1)], -q[halo_ix<DIM>(I, J, K - 1)]), h2);
    }
    C w;
    if (DIM == 2) {
        w = fabs(r_add(g[1][0], -g[0][1]));
    } else {
        const C wx = r_add(g[2][1], -g[1][2]), wy = r_add(g[0][2], -g[2][0]), wz = r_add(g[1][0], -g[0][1]);
        w = r_sqrt(r_add(r_add(r_mul(wx, wx), r_mul(wy, wy)), r_mul(wz, wz)));
    }
    if (a.cmask[cell] == CELL_GHOST) w = C(0);
    sW[t] = w;
    __syncthreads();
    for (int st = MC / 2; st > 0; st >>= 1) {
        if (t < st) sW[t] = fmax(sW[t], sW[t + st]);
        __syncthreads();
    }
    if (t == 0) {
        const int leaf = a.nbr_child[b] < 0;
        a.wval[b] = (double)sW[0];
        a.pop[b] = leaf;
        if (leaf) atomicAdd(&a.st->n, 1);
    }
}

// One radix pass: histogram of the next 16 key bits of the population
// elements that match each quantile's prefix.
__global__ void k_pct_hist(const double *wval, const int *pop, int idm, const PctState *st, int pass, int *hist)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= idm || !pop[b]) return;
    const unsigned long long key = (unsigned long long)__double_as_longlong(wval[b]);
    const int sh = 48 - 16 * pass;
    for (int r = 0; r < 2; r++) {
        if (pass > 0 && (key >> (sh + 16)) != st->prefix[r]) continue;
        atomicAdd(&hist[r * 65536 + (int)((key >> sh) & 0xFFFFull)], 1);
    }
}

// Select the bin holding each quantile's rank (one CTA per quantile, 1024
// threads x 64 bins), extend its prefix, and clear the histogram.
__global__ void __launch_bounds__(1024) k_pct_pick(int *hist, PctState *st, int pass, double pct_hi, double pct_lo)
{
    __shared__ int s_warp[32];
    const int r = blockIdx.x, t = threadIdx.x;
    const int n = st->n;
    if (n <= 0) return;   // uniform
    int *h = hist + r * 65536;
    const int k = (pass == 0) ? (int)floor((r == 0 ? pct_hi : pct_lo) * (double)(n - 1)) : st->k[r];
    int sum = 0;
    for (int i = 0; i < 64; i++) sum += h[t * 64 + i];
    // exclusive scan of the per-thread sums
    const int lane = t & 31, wid = t >> 5;
    int x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int v = s_warp[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        s_warp[lane] = v;
    }
    __syncthreads();
    int start = (wid ? s_warp[wid - 1] : 0) + x - sum;
    if (start <= k && k < start + sum) {
        for (int i = 0; i < 64; i++) {
            const int c = h[t * 64 + i];
            if (k < start + c) {
                st->prefix[r] = (st->prefix[r] << 16) | (unsigned long long)(t * 64 + i);
                st->k[r] = k - start;
                break;
            }
            start += c;
        }
    }
    __syncthreads();
    for (int i = 0; i < 64; i++) h[t * 64 + i] = 0;
}

// The whole selection in one CTA, for pools of up to kPctOneCta blocks: eight
// passes of 8 key bits, histograms in shared memory, warp r picking the bin
// of quantile r.  Selects the same keys as the 16-bit passes above.
constexpr int kPctOneCta = 1 << 16;

__global__ void __launch_bounds__(1024) k_pct_select(const double *wval, const int *pop, int idm, PctState *st,
                                                     double pct_hi, double pct_lo)
{
    __shared__ int s_hist[2][256];
    __shared__ unsigned long long s_prefix[2];
    __shared__ int s_k[2];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int n = st->n;
    if (n <= 0) return;   // uniform
    if (t < 2) {
        s_prefix[t] = 0ull;
        s_k[t] = (int)floor((t == 0 ? pct_hi : pct_lo) * (double)(n - 1));
    }
    for (int pass = 0; pass < 8; pass++) {
        const int sh = 56 - 8 * pass;
        for (int i = t; i < 512; i += blockDim.x) s_hist[i >> 8][i & 255] = 0;
        __syncthreads();
        const unsigned long long p0 = s_prefix[0], p1 = s_prefix[1];
        for (int b = t; b < idm; b += blockDim.x) {
            if (!pop[b]) continue;
            const unsigned long long key = (unsigned long long)__double_as_longlong(wval[b]);
            const int bin = (int)((key >> sh) & 0xFFull);
            const unsigned long long hi = pass ? (key >> (sh + 8)) : 0ull;
            if (hi == p0) atomicAdd(&s_hist[0][bin], 1);
            if (hi == p1) atomicAdd(&s_hist[1][bin], 1);
        }
        __syncthreads();
        if (wid < 2) {
            const int r = wid, k = s_k[r];
            int c[8], sum = 0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                c[i] = s_hist[r][lane * 8 + i];
                sum += c[i];
            }
            int x = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            int start = x - sum;
            if (start <= k && k < start + sum) {
                for (int i = 0; i < 8; i++) {
                    if (k < start + c[i]) {
                        s_prefix[r] = (s_prefix[r] << 8) | (unsigned long long)(lane * 8 + i);
                        s_k[r] = k - start;
                        break;
                    }
                    start += c[i];
                }
            }
        }
        __syncthreads();
    }
    if (t < 2) {
        st->prefix[t] = s_prefix[t];
        st->k[t] = s_k[t];
    }
}

__global__ void k_pct_mark(const double *wval, const PctState *st, const int *nbr, long long nmb, int qmax,
                           const int *level, int mli, int idm, int *ref)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= idm || st->n <= 0) return;
    const int r = ref[b];
    if (r == REF_INACTIVE) return;
    const double thr_hi = __longlong_as_double((long long)st->prefix[0]);
    const double thr_lo = __longlong_as_double((long long)st->prefix[1]);
    bool eligible = true;
    for (int p = 0; p < qmax; p++)
        if (nbr[b + (long long)p * nmb] == N_SKIPID) eligible = false;
    const double w = wval[b];
    if (r == REF_UNREFINED && eligible && level[b] < mli - 1 && w > thr_hi) ref[b] = REF_MARK_REFINE;
    if (r == REF_REFINED && w < thr_lo) ref[b] = REF_MARK_COARSEN;
}

// The percentile rule's decisions for listed blocks (learned-predictor
// labels): Y[j] = {leaf block value above the upper quantile, value below the
// lower quantile}.  With lvl0, Wt[j] = 1 if block ids[j] is still active on
// level lvl0[j], else 0 (and Y = 0).
__global__ void k_pct_decide(const double *wval, const int *pop, const PctState *st, const int *ids,
                             const int *lvl0, int n, const int *ref, const int *level, float *Y, float *Wt)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int b = ids[j];
    const bool valid = ref[b] != REF_INACTIVE && (!lvl0 || level[b] == lvl0[j]) && st->n > 0;
    const double thr_hi = __longlong_as_double((long long)st->prefix[0]);
    const double thr_lo = __longlong_as_double((long long)st->prefix[1]);
    const double w = wval[b];
    Y[2 * j + 0] = (valid && pop[b] && w > thr_hi) ? 1.f : 0.f;
    Y[2 * j + 1] = (valid && w < thr_lo) ? 1.f : 0.f;
    if (Wt) Wt[j] = valid ? 1.f : 0.f;
}

template <int DIM, int Q, typename T> struct RunInterp {
    static int run(agal_ctx *c, int L, int var)
    {
        const int n = c->n_ids[L];
        if (n <= 0) return AGAL_OK;
        InterpArgs a;
        a.ids = c->id_set + (long long)L * c->nmb;
        a.n = n;
        a.sr = (c->storage == AGAL_STORE_FP16 || c->storage == AGAL_STORE_BF16) &&
               c->P.half_rounding == AGAL_ROUND_STOCHASTIC;
        a.sr_ctr = c->d_sr;
        a.sr_salt = (unsigned)c->sr_salt | 0x40000000u;
        // Interface interpolation touches the interface parents only.
        if (var == AGAL_INTERP_INTERFACE && (int)c->iface_n.size() > L) {
            a.ids = c->iface_ids + c->iface_off[L];
            a.n = c->iface_n[L];
            if (a.n <= 0) return AGAL_OK;
        }
        a.fpar = c->F[c->cur[L]];
        a.fch = c->F[c->cur[L + 1]];
        a.nbr_child = c->cblock_ID_nbr_child;
        a.bmask = c->cblock_ID_mask;
        a.ref = c->cblock_ID_ref;
        a.cmask = c->cells_ID_mask;
        a.ratio = c->tau[L + 1] / c->tau[L];
        if (sizeof(typename ST<T>::C) == 4) a.ratio = (double)((float)c->tau[L + 1] / (float)c->tau[L]);
        a.var = var;
        if (c->rec)   // batch recording: one batched launch per phase (batch.cu)
            return agal_record_args(c, AGAL_OP_INTERP, L, &a, sizeof(a),
                                    agal_transfer_batch_key(c, c->P.interp_order == AGAL_INTERP_CUBIC), a.n);
        constexpr int NT = Geo<DIM>::NCH * Geo<DIM>::MC;
        if (c->P.interp_order == AGAL_INTERP_CUBIC)
            AGAL_CUDA(c, launch_pdl(k_interp<DIM, Q, T, true>, dim3((unsigned)a.n), dim3(NT), 0, c->stream, a));
        else
            AGAL_CUDA(c, launch_pdl(k_interp<DIM, Q, T, false>, dim3((unsigned)a.n), dim3(NT), 0, c->stream, a));
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
};

template <int DIM, int Q, typename T> struct RunAverage {
    static int run(agal_ctx *c, int L, int var)
    {
        const int n = c->n_ids[L];
        if (n <= 0) return AGAL_OK;
        AverageArgs a;
        a.ids = c->id_set + (long long)L * c->nmb;
        a.n = n;
        a.sr = (c->storage == AGAL_STORE_FP16 || c->storage == AGAL_STORE_BF16) &&
               c->P.half_rounding == AGAL_ROUND_STOCHASTIC;
        a.sr_ctr = c->d_sr;
        a.sr_salt = (unsigned)c->sr_salt | 0x80000000u;
        // Interface and block averaging touch the interface parents only.
        if (var != AGAL_AVERAGE_GRID && (int)c->iface_n.size() > L) {
            a.ids = c->iface_ids + c->iface_off[L];
            a.n = c->iface_n[L];
            if (a.n <= 0) return AGAL_OK;
        }
        a.fpar = c->F[c->cur[L]];
        a.fch = c->F[c->cur[L + 1]];
        a.nbr_child = c->cblock_ID_nbr_child;
        a.bmask = c->cblock_ID_mask;
        a.cmask = c->cells_ID_mask;
        a.ratio = c->tau[L] / c->tau[L + 1];
        if (sizeof(typename ST<T>::C) == 4) a.ratio = (double)((float)c->tau[L] / (float)c->tau[L + 1]);
        a.var = var;
        a.tick = nullptr;
        a.ticket = nullptr;
        if (c->rec)   // batch recording: one batched launch per phase (batch.cu)
            return agal_record_args(c, AGAL_OP_AVERAGE, L, &a, sizeof(a), agal_transfer_batch_key(c, false), a.n);
        if (c->tick_pending && L == c->L0) {   // the coarse step's last launch
            a.tick = c->d_sr;
            a.ticket = c->d_status + 3;
            c->tick_pending = false;
            c->tick_done = true;
        }
        constexpr int NT = Geo<DIM>::NCH * Geo<DIM>::MC;
        AGAL_CUDA(c, launch_pdl(k_average<DIM, Q, T>, dim3((unsigned)a.n), dim3(NT), 0, c->stream, a));
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
};

}  // namespace agal

int agal_launch_interp(agal_ctx *c, int L, int var) { return agal::dispatch<agal::RunInterp>(c, L, var); }
int agal_launch_average(agal_ctx *c, int L, int var) { return agal::dispatch<agal::RunAverage>(c, L, var); }

// Batched transfers of many cases (batch.cu).  key: velocity set, storage and
// (interpolation) the cubic flag.
int agal_transfer_batch_key(const agal_ctx *c, bool cubic) { return (c->Q * 8 + c->storage) * 2 + (cubic ? 1 : 0); }

namespace {
template <int DIM, int Q, typename T>
int transfer_batch(int kind, bool cubic, cudaStream_t s, const void *args, const int *start, int n, int total)
{
    constexpr int NT = agal::Geo<DIM>::NCH * agal::Geo<DIM>::MC;
    if (total <= 0) return AGAL_OK;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (kind == AGAL_OP_INTERP) {
        const auto *A = static_cast<const agal::InterpArgs *>(args);
        auto k = cubic ? agal::k_interp_batch<DIM, Q, T, true> : agal::k_interp_batch<DIM, Q, T, false>;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, 0);
        if (e != cudaSuccess) return AGAL_ERR_CUDA;
        k<<<std::min(total, std::max(per_sm, 1) * sms), NT, 0, s>>>(A, start, n);
    } else {
        const auto *A = static_cast<const agal::AverageArgs *>(args);
        auto k = agal::k_average_batch<DIM, Q, T>;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, 0);
        if (e != cudaSuccess) return AGAL_ERR_CUDA;
        k<<<std::min(total, std::max(per_sm, 1) * sms), NT, 0, s>>>(A, start, n);
    }
    return cudaGetLastError() == cudaSuccess ? AGAL_OK : AGAL_ERR_CUDA;
}
}  // namespace

int agal_launch_transfer_batch(int kind, int key, cudaStream_t s, const void *args, const int *start, int n, int total)
{
    const bool cubic = key & 1;
    const int storage = (key >> 1) % 8, Q = (key >> 1) / 8;
    auto go = [&](auto tag) -> int {
        using T = decltype(tag);
        switch (Q) {
        case 9: return transfer_batch<2, 9, T>(kind, cubic, s, args, start, n, total);
        case 19: return transfer_batch<3, 19, T>(kind, cubic, s, args, start, n, total);
        case 27: return transfer_batch<3, 27, T>(kind, cubic, s, args, start, n, total);
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

// Argument-structure sizes the batch checks recorded launches against.
size_t agal_transfer_args_size(int kind)
{
    return kind == AGAL_OP_INTERP ? sizeof(agal::InterpArgs) : sizeof(agal::AverageArgs);
}

// Block values and the two quantiles of the percentile rule (no marks).
static int percentile_select(agal_ctx *c, int idm)
{
    if (!c->crit) return agal_set_err(c, AGAL_ERR_STATE, "percentile criterion needs MAX_LEVELS > 1");
    double *wval = static_cast<double *>(c->crit);
    int *hist = reinterpret_cast<int *>(wval + c->nmb);
    agal::PctState *st = reinterpret_cast<agal::PctState *>(hist + 2 * 65536);
    const bool one_cta = idm <= agal::kPctOneCta;
    AGAL_CUDA(c, cudaMemsetAsync(st, 0, sizeof(agal::PctState), c->stream));
    if (!one_cta) AGAL_CUDA(c, cudaMemsetAsync(hist, 0, sizeof(int) * 2 * 65536, c->stream));
    agal::WmaxArgs a;
    a.idm = idm;
    a.nmc = c->nmc;
    a.macro = c->macro;
    a.cmask = c->cells_ID_mask;
    a.level = c->cblock_level;
    a.ref = c->cblock_ID_ref;
    a.nbr_child = c->cblock_ID_nbr_child;
    for (int L = 0; L < 16; L++) a.dx[L] = (L < c->max_levels) ? c->dxf[L] : 0.0;
    a.wval = wval;
    a.pop = c->amr_a;
    a.st = st;
    const bool f64 = c->storage == AGAL_STORE_FP64;
    if (c->dim == 2) {
        if (f64) agal::k_wmax<2, double><<<(unsigned)idm, 16, 0, c->stream>>>(a);
        else agal::k_wmax<2, float><<<(unsigned)idm, 16, 0, c->stream>>>(a);
    } else {
        if (f64) agal::k_wmax<3, double><<<(unsigned)idm, 64, 0, c->stream>>>(a);
        else agal::k_wmax<3, float><<<(unsigned)idm, 64, 0, c->stream>>>(a);
    }
    const unsigned g = (unsigned)((idm + 255) / 256);
    if (one_cta) {
        agal::k_pct_select<<<1, 1024, 0, c->stream>>>(wval, c->amr_a, idm, st, c->P.ref_pct_hi, c->P.ref_pct_lo);
    } else {
        for (int pass = 0; pass < 4; pass++) {
            agal::k_pct_hist<<<g, 256, 0, c->stream>>>(wval, c->amr_a, idm, st, pass, hist);
            agal::k_pct_pick<<<2, 1024, 0, c->stream>>>(hist, st, pass, c->P.ref_pct_hi, c->P.ref_pct_lo);
        }
    }
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

static int launch_percentile(agal_ctx *c, int idm)
{
    const int rc = percentile_select(c, idm);
    if (rc) return rc;
    double *wval = static_cast<double *>(c->crit);
    agal::PctState *st = reinterpret_cast<agal::PctState *>(reinterpret_cast<int *>(wval + c->nmb) + 2 * 65536);
    const unsigned g = (unsigned)((idm + 255) / 256);
    agal::k_pct_mark<<<g, 256, 0, c->stream>>>(wval, st, c->cblock_ID_nbr, c->nmb, c->Qmax, c->cblock_level,
                                               c->P.MAX_LEVELS_INTERIOR, idm, c->cblock_ID_ref);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

int agal_percentile_decisions(agal_ctx *c, int select, const int *ids, const int *lvl0, int n, float *Y, float *Wt)
{
    if (!c->crit) return agal_set_err(c, AGAL_ERR_STATE, "percentile criterion needs MAX_LEVELS > 1");
    const int idm = c->id_max[c->max_levels];
    if (select && idm > 0) {
        const int rc = percentile_select(c, idm);
        if (rc) return rc;
    }
    if (n <= 0) return AGAL_OK;
    double *wval = static_cast<double *>(c->crit);
    agal::PctState *st = reinterpret_cast<agal::PctState *>(reinterpret_cast<int *>(wval + c->nmb) + 2 * 65536);
    agal::k_pct_decide<<<(unsigned)((n + 127) / 128), 128, 0, c->stream>>>(wval, c->amr_a, st, ids, lvl0, n,
                                                                           c->cblock_ID_ref, c->cblock_level, Y, Wt);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

int agal_launch_criterion(agal_ctx *c)
{
    const int idm = c->id_max[c->max_levels];
    if (idm <= 0) return AGAL_OK;
    // The learned mode's judge (and its stand-in without a network) is the percentile rule.
    if (c->P.S_CRITERION == AGAL_CRITERION_PERCENTILE || c->P.S_CRITERION == AGAL_CRITERION_LEARNED)
        return launch_percentile(c, idm);
    agal::CriterionArgs a;
    a.idm = idm;
    a.nmb = c->nmb;
    a.nmc = c->nmc;
    a.macro = c->macro;
    a.cmask = c->cells_ID_mask;
    a.level = c->cblock_level;
    a.nbr = c->cblock_ID_nbr;
    a.ref = c->cblock_ID_ref;
    a.dx = c->dxf[0];
    a.criterion = c->P.S_CRITERION;
    a.nrs = c->P.N_REFINE_START;
    a.nri = c->P.N_REFINE_INC;
    a.nrm = c->P.N_REFINE_MAX;
    a.mli = c->P.MAX_LEVELS_INTERIOR;
    const bool f64 = c->storage == AGAL_STORE_FP64;
    if (c->dim == 2) {
        if (f64) agal::k_criterion<2, double><<<(unsigned)idm, 16, 0, c->stream>>>(a);
        else agal::k_criterion<2, float><<<(unsigned)idm, 16, 0, c->stream>>>(a);
    } else {
        if (f64) agal::k_criterion<3, double><<<(unsigned)idm, 64, 0, c->stream>>>(a);
        else agal::k_criterion<3, float><<<(unsigned)idm, 64, 0, c->stream>>>(a);
    }
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}
