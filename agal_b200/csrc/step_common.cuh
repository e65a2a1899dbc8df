// Shared pieces of the fused step kernels: kernel arguments, the neighbour
// slot map, the boundary-condition hook presets and the BGK collision.
#pragma once

#include <cuda_runtime.h>

#include "lattice.cuh"
#include "storage.cuh"
#include "../../include/agal_b200.h"

namespace agal {

// Neighbour-slot -> neighbour-array index (inc/util.h:100-101).  Read with a
// different index by every thread, so it lives in global memory (L1-cached)
// rather than in the constant bank, which serialises divergent reads.
static __device__ const int g_map2[9] = {7, 4, 8, 3, 0, 1, 6, 2, 5};
static __device__ const int g_map3[27] = {20, 12, 26, 10, 6, 15, 24, 17, 21, 8, 4, 13, 2, 0,
                                   1, 14, 3, 7, 22, 18, 23, 16, 5, 9, 25, 11, 19};

// Programmatic dependent launch.  A kernel launched with launch_pdl may start
// while its predecessor on the stream is still draining; griddepcontrol.wait
// blocks until that predecessor has completed and its writes are visible
// (returns at once when there is none).  Every kernel launched this way calls
// pdl_wait() before it touches memory, then lets its own successor launch.
__device__ __forceinline__ void pdl_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...);
}

// Per-block step metadata row, rebuilt whenever the mesh changes
// (agal_build_meta): the neighbour block in each lexicographic neighbour slot
// S (the centre slot holds the block itself) and the step flags.  One
// contiguous 16-byte-multiple row per block, so the step kernels fetch it
// with one coalesced load or one bulk copy instead of Q_max strided loads
// from the structure-of-arrays neighbour table.
template <int DIM> struct Meta {
    static constexpr int W = (DIM == 2) ? 12 : 28;        // ints per row (48 / 112 bytes)
    static constexpr int FLAGS = (DIM == 2) ? 9 : 27;     // index of the flag word
};
constexpr int META_ACTIVE = 1;   // collide/stream this block (kernels.cu:236)
constexpr int META_ONB = 2;      // block touches a domain boundary (kernels.cu:736)
constexpr int META_WALL = 4;     // wall block stepped by k_step_wall (interpolated bounce-back)
constexpr int META_NEARSOLID = 8;   // a solid cell in this block or a neighbour (geometry cases)
constexpr int META_CLOSED = 16;     // some neighbour slot holds no block (closed links possible)

struct StepArgs {
    const int *ids;
    int n;
    const void *fin;
    void *fout;
    const int *meta;
    const int *cmask;
    double omega;
    double u_ref;
    int bc_preset;
    int mrt;               // D3Q19 multiple-relaxation-time collision instead of BGK
    double s[5];           // MRT rates s1, s2, s3, s5, s6
    // Links whose in-place swap the reference's guard would refuse (see
    // push_cell): appended here, swapped back by k_stream_fixup.
    int *fix_count;
    long long *fix_list;   // [fix_cap][2] element offsets into fout
    int fix_cap;
    // Non-null: the step kernel's last CTA applies the list itself (small
    // grids, where the fence costs less than a separate launch).
    int *fix_ticket;
    int *status;
    // LES (S_LES > 0): eddy viscosity per cell of the pool (compute type);
    // the cell relaxes with omega = dx / (3 (nu + nu_SGS) + dx / 2)
    // (Cu_CollideLES, solver_lbm_kernels.cu:352-355).  Null otherwise.
    const void *nu_sgs;
    double nu, dxL;
    // Multi-level LES: the macro rows rho, u, v(, w) [dim+1][nmc] that the
    // collide rewrites from the pre-collision populations of every cell of
    // the blocks it steps, solid cells included (Cu_CollideLES,
    // solver_lbm_kernels.cu:337-350); the level's next eddy viscosity reads
    // them.  Null otherwise.
    void *macro;
    long long nmc;
    // Stochastic rounding of half-precision offsets (agal_params
    // half_rounding): on when sr is set.  The launch seed mixes the coarse-step
    // counter in device memory (advanced once per coarse step, so replayed
    // graphs see a new value) with this launch's ordinal in the coarse step.
    int sr;
    const unsigned *sr_ctr;
    unsigned sr_salt;
};

// Seed of a step launch (read after the wait on the predecessor).
__device__ __forceinline__ unsigned step_seed(const StepArgs &a)
{
    return a.sr ? (*a.sr_ctr) * 0x9E3779B9u + a.sr_salt * 0x85EBCA77u + 0x165667B1u : 0u;
}

// Random bits of the stochastic rounding of the values of cell t of block b:
// one hash per cell (its index in the pool), sr_dir(p) per direction.  Keyed
// by the cell and direction a value was collided for, so every variant
// rounds it alike wherever it is stored.
template <int DIM>
__device__ __forceinline__ unsigned sr_cell_of(long long b, int t, unsigned seed)
{
    return sr_cell(b * Geo<DIM>::MC + t, seed);
}

// The stream-guard fix-ups applied by the last CTA of the step kernel: every
// thread fences its stores, the CTA takes a ticket, and the CTA holding the
// last ticket swaps back the recorded pairs (the refused in-place swaps), then
// resets the list and the ticket for the next launch.  Called by every thread
// of every CTA.
template <typename T>
__device__ __forceinline__ void fused_fixup(const StepArgs &a)
{
    __shared__ int s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(a.fix_ticket, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int n = atomicAdd(a.fix_count, 0);
    const int m = n < a.fix_cap ? n : a.fix_cap;
    T *fo = static_cast<T *>(a.fout);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const long long x = __ldcg(&a.fix_list[2 * i]), y = __ldcg(&a.fix_list[2 * i + 1]);
        const T vx = __ldcg(&fo[x]), vy = __ldcg(&fo[y]);
        fo[x] = vy;
        fo[y] = vx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (n > a.fix_cap) atomicCAS(a.status, 0, AGAL_ERR_STATE);
        *a.fix_count = 0;
        *a.fix_ticket = 0;
    }
}

// Explicitly rounded arithmetic (never contracted or reordered by the
// compiler), so that every kernel variant that inlines the collision performs
// the same operation sequence and produces bit-identical populations.
__device__ __forceinline__ float r_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float r_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float r_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float r_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double r_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double r_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double r_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ double r_div(double a, double b) { return __ddiv_rn(a, b); }

// Boundary hook presets (inc/custom.h:79-122); f is the full population.
// Every operation is rounded as written (the order of the C++ expressions
// of the presets, no fused multiply-add), so the bounced value is the same in
// every kernel that inlines the hook.
template <typename C>
__device__ __forceinline__ C bc_hook(int preset, int nb, C f, C u, C v, C w, C wp, int cx, int cy, int cz, C U)
{
    bool inflow = false, outflow = false;
    switch (preset) {
    case AGAL_BC_LDC2D: inflow = (nb == -4); break;
    case AGAL_BC_LDC3D: inflow = (nb == -6); break;
    case AGAL_BC_FPSC2D: inflow = (nb == -1 || nb == -3 || nb == -4); outflow = (nb == -2); break;
    case AGAL_BC_FPSC3D:
        inflow = (nb == -1 || nb == -3 || nb == -4 || nb == -5 || nb == -6);
        outflow = (nb == -2);
        break;
    default: break;
    }
    if (inflow) return r_add(f, -r_mul(r_mul(C(2), wp), r_mul(C(3), r_mul(C(cx), U))));
    if (outflow) {
        const C cu = r_add(r_add(r_mul(C(cx), u), r_mul(C(cy), v)), r_mul(C(cz), w));
        const C uu = r_add(r_add(r_mul(u, u), r_mul(v, v)), r_mul(w, w));
        const C e = r_add(r_add(C(1), r_mul(r_mul(C(4.5), cu), cu)), -r_mul(C(1.5), uu));
        return r_add(-f, r_mul(r_mul(C(2), wp), e));
    }
    return f;
}

// Minimum resident 256-thread CTAs per SM requested from the register
// allocator: as many as fit without spilling the Q populations held per thread.
template <int DIM, int Q, typename T, int CPT> struct StepOcc {
    static constexpr int words = CPT * Q * (sizeof(typename ST<T>::C) == 8 ? 2 : 1);   // registers for g[][]
    static constexpr int value = words <= 9 ? 6 : words <= 19 ? 4 : words <= 27 ? 3 : words <= 38 ? 2 : 1;
};

// sum_p c_p g_p along one axis for lattice directions with c in {-1, 0, 1}.
template <int DIM, int Q, int AXIS, typename C>
__device__ __forceinline__ C moment1(const C (&g)[Q])
{
    C s = C(0);
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const int c = lat_c(DIM, AXIS, p);
        if (c > 0) s = r_add(s, g[p]);
        if (c < 0) s = r_add(s, -g[p]);
    }
    return s;
}

// c_p . u for c in {-1, 0, 1}^3.
template <int DIM, typename C>
__device__ __forceinline__ C cdot(int p, C ux, C uy, C uz)
{
    C s = C(0);
    const int cx = lat_c(DIM, 0, p), cy = lat_c(DIM, 1, p), cz = lat_c(DIM, 2, p);
    s = cx > 0 ? ux : (cx < 0 ? -ux : s);
    if (cy != 0) s = r_add(s, cy > 0 ? uy : -uy);
    if (cz != 0) s = r_add(s, cz > 0 ? uz : -uz);
    return s;
}

// BGK collision of one cell in place on g[] (full populations, or weight
// offsets g = f - w for the half-precision forms).  Opposite directions share
// the even part of the equilibrium, feq_{p,pb} = w rho (1 + 4.5 cu^2 -
// 1.5 u^2) +- 3 w rho cu, so each pair is evaluated once
// (Cu_Collide, kernels.cu:249-286).  Returns the macros for the boundary hook.
// Macro rows of one cell from its populations (offset form when OFF), as
// Cu_CollideLES stores them before relaxing: rho, then u = j / rho.
template <int DIM, int Q, typename C, bool OFF>
__device__ __forceinline__ void store_macros(const C (&g)[Q], void *macro, long long nmc, long long cell)
{
    C drho = C(0);
#pragma unroll
    for (int p = 0; p < Q; p++) drho = r_add(drho, g[p]);
    const C rho = OFF ? r_add(C(1), drho) : drho;
    C *m = static_cast<C *>(macro);
    m[cell] = rho;
    m[nmc + cell] = r_div(moment1<DIM, Q, 0>(g), rho);
    m[2 * nmc + cell] = r_div(moment1<DIM, Q, 1>(g), rho);
    if (DIM == 3) m[3 * nmc + cell] = r_div(moment1<DIM, Q, 2>(g), rho);
}

template <int DIM, int Q, typename C, bool OFF>
__device__ __forceinline__ void bgk_collide(C (&g)[Q], C omeg, C &ux, C &uy, C &uz)
{
    C drho = C(0);
#pragma unroll
    for (int p = 0; p < Q; p++) drho = r_add(drho, g[p]);
    const C jx = moment1<DIM, Q, 0>(g), jy = moment1<DIM, Q, 1>(g);
    const C jz = (DIM == 3) ? moment1<DIM, Q, 2>(g) : C(0);
    // Offset form: sum_p w_p = 1 and sum_p w_p c_p = 0.
    const C rho = OFF ? r_add(C(1), drho) : drho;
    const C inv = r_div(C(1), rho);
    ux = r_mul(jx, inv);
    uy = r_mul(jy, inv);
    uz = (DIM == 3) ? r_mul(jz, inv) : C(0);
    const C omegp = r_add(C(1), -omeg);
    const C usq = r_fma(uz, uz, r_fma(uy, uy, r_mul(ux, ux)));
    const C h = r_mul(C(1.5), usq);   // 1.5 u^2
    const C one_h = r_add(C(1), -h);
    const C orho = r_mul(omeg, rho);
    // Rest population.  The offset form keeps omega (feq - w) as the small
    // quantity w omega (drho + rho (...)) instead of a difference of O(w) terms.
    {
        const C w0 = C(lat_w(Q, 0));
        const C e0 = OFF ? r_mul(r_mul(omeg, w0), r_fma(-rho, h, drho)) : r_mul(r_mul(w0, orho), one_h);
        g[0] = r_fma(g[0], omegp, e0);
    }
#pragma unroll
    for (int p = 1; p < Q; p++) {
        const int q = lat_pb(DIM, p);
        if (q < p) continue;   // each pair once, from its lower index
        const C cu = cdot<DIM>(p, ux, uy, uz);
        const C wp = C(lat_w(Q, p));
        const C wo = r_mul(wp, orho);
        const C cu2 = r_mul(cu, cu);
        const C even = OFF ? r_mul(r_mul(wp, omeg), r_fma(rho, r_fma(C(4.5), cu2, -h), drho))
                           : r_mul(wo, r_fma(C(4.5), cu2, one_h));
        const C odd = r_mul(r_mul(C(3), wo), cu);
        g[p] = r_fma(g[p], omegp, r_add(even, odd));
        g[q] = r_fma(g[q], omegp, r_add(even, -odd));
    }
}

// D3Q19 multiple-relaxation-time collision (d'Humieres moment basis: rho, e,
// eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww, pxy, pyz, pxz, mx, my,
// mz), with the equilibria of the reference's legacy MRT kernel
// (solver_old/solver_lbm_collide_mrt_d3q19.cu:131-148; its e equilibrium is read
// as 19 rho |u|^2).  Rates: s1 (e), s2 (eps), s3 (q), omega_L (3pxx, pww, pxy,
// pyz, pxz), s5 (3pixx, piww), s6 (mx, my, mz); rho and j are conserved.
// Entries of the basis, a polynomial in the direction vector:
__host__ __device__ constexpr int mrt_m(int i, int p)
{
    const int x = lat_c(3, 0, p), y = lat_c(3, 1, p), z = lat_c(3, 2, p), c2 = x * x + y * y + z * z;
    switch (i) {
    case 0: return 1;
    case 1: return 19 * c2 - 30;
    case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
    case 3: return x;
    case 4: return (5 * c2 - 9) * x;
    case 5: return y;
    case 6: return (5 * c2 - 9) * y;
    case 7: return z;
    case 8: return (5 * c2 - 9) * z;
    case 9: return 3 * x * x - c2;
    case 10: return (3 * c2 - 5) * (3 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (3 * c2 - 5) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    default: return (x * x - y * y) * z;
    }
}
// Squared norm of basis row i (the rows are orthogonal: M^-1 = M^T diag(1/n)).
__host__ __device__ constexpr int mrt_n(int i)
{
    int s = 0;
    for (int p = 0; p < 19; p++) s += mrt_m(i, p) * mrt_m(i, p);
    return s;
}

// OFF: g holds weight offsets (rest moments of the weights, rho = 1, e = -11,
// eps = 3, are carried implicitly).  The rates s = {s1, s2, s3, s5, s6}.
template <typename C, bool OFF>
__device__ __forceinline__ void mrt_collide(C (&g)[19], C omeg, const C (&s)[5], C &ux, C &uy, C &uz)
{
    C m[19];
#pragma unroll
    for (int i = 0; i < 19; i++) {
        C acc = C(0);
#pragma unroll
        for (int p = 0; p < 19; p++) {
            const int k = mrt_m(i, p);
            if (k == 1) acc = r_add(acc, g[p]);
            else if (k == -1) acc = r_add(acc, -g[p]);
            else if (k != 0) acc = r_fma(C(k), g[p], acc);
        }
        m[i] = acc;
    }
    const C drho = m[0];
    const C rho = OFF ? r_add(C(1), drho) : drho;
    const C inv = r_div(C(1), rho);
    ux = r_mul(m[3], inv);
    uy = r_mul(m[5], inv);
    uz = r_mul(m[7], inv);
    const C uu = r_mul(ux, ux), vv = r_mul(uy, uy), ww = r_mul(uz, uz);
    const C usq = r_add(r_add(uu, vv), ww);
    const C rusq = r_mul(rho, usq);
    // deviations of the equilibria from the stored reference (rest moments in
    // the offset form, zero otherwise)
    const C dr = OFF ? drho : rho;
    C eq[19];
    eq[1] = r_fma(C(19), rusq, r_mul(C(-11), dr));
    eq[2] = r_fma(C(-5.5), rusq, r_mul(C(3), dr));
    eq[4] = r_mul(C(-2.0 / 3.0), m[3]);
    eq[6] = r_mul(C(-2.0 / 3.0), m[5]);
    eq[8] = r_mul(C(-2.0 / 3.0), m[7]);
    const C pxx = r_mul(rho, r_add(r_mul(C(2), uu), -r_add(vv, ww)));
    const C pww = r_mul(rho, r_add(vv, -ww));
    eq[9] = pxx;
    eq[10] = r_mul(C(-0.5), pxx);
    eq[11] = pww;
    eq[12] = r_mul(C(-0.5), pww);
    eq[13] = r_mul(rho, r_mul(ux, uy));
    eq[14] = r_mul(rho, r_mul(uy, uz));
    eq[15] = r_mul(rho, r_mul(ux, uz));
    auto relax = [&](int i, C rate, C e) { m[i] = r_add(m[i], -r_mul(rate, r_add(m[i], -e))); };
    relax(1, s[0], eq[1]);
    relax(2, s[1], eq[2]);
    relax(4, s[2], eq[4]);
    relax(6, s[2], eq[6]);
    relax(8, s[2], eq[8]);
    relax(9, omeg, eq[9]);
    relax(10, s[3], eq[10]);
    relax(11, omeg, eq[11]);
    relax(12, s[3], eq[12]);
    relax(13, omeg, eq[13]);
    relax(14, omeg, eq[14]);
    relax(15, omeg, eq[15]);
    relax(16, s[4], C(0));
    relax(17, s[4], C(0));
    relax(18, s[4], C(0));
#pragma unroll
    for (int p = 0; p < 19; p++) {
        C acc = C(0);
#pragma unroll
        for (int i = 0; i < 19; i++) {
            const int k = mrt_m(i, p);
            if (k != 0) acc = r_fma(C((double)k / (double)mrt_n(i)), m[i], acc);
        }
        g[p] = acc;
    }
}

// BGK, or for D3Q19 with a.mrt the MRT collision (uniform per launch).
template <int DIM, int Q, typename T>
__device__ __forceinline__ void collide_cell(typename ST<T>::C (&g)[Q], const StepArgs &a, typename ST<T>::C &ux,
                                             typename ST<T>::C &uy, typename ST<T>::C &uz)
{
    using C = typename ST<T>::C;
    if constexpr (Q == 19) {
        if (a.mrt) {
            const C s[5] = {C(a.s[0]), C(a.s[1]), C(a.s[2]), C(a.s[3]), C(a.s[4])};
            mrt_collide<C, ST<T>::OFF>(g, C(a.omega), s, ux, uy, uz);
            return;
        }
    }
    bgk_collide<DIM, Q, C, ST<T>::OFF>(g, C(a.omega), ux, uy, uz);
}

// The collision of one cell of the pool (index cell = b * MC + t): with LES,
// BGK at omega = dx / (3 (nu + nu_SGS) + dx / 2) from the cell's eddy
// viscosity (Cu_CollideLES, solver_lbm_kernels.cu:352-355); else collide_cell.
template <int DIM, int Q, typename T>
__device__ __forceinline__ void collide_at(typename ST<T>::C (&g)[Q], const StepArgs &a, long long cell,
                                           typename ST<T>::C &ux, typename ST<T>::C &uy, typename ST<T>::C &uz)
{
    using C = typename ST<T>::C;
    if (a.nu_sgs) {
        const C nus = static_cast<const C *>(a.nu_sgs)[cell];
        const C dx = C(a.dxL);
        const C tau = r_fma(C(3), r_add(C(a.nu), nus), r_mul(C(0.5), dx));
        bgk_collide<DIM, Q, C, ST<T>::OFF>(g, r_div(dx, tau), ux, uy, uz);
    } else {
        collide_cell<DIM, Q, T>(g, a, ux, uy, uz);
    }
}

// Stream one collided cell (cell t of block b, populations g) into the
// output buffer: push along open links, bounce back along closed ones with
// the boundary hook on domain boundaries (kernels.cu:534-633, 693-887).
// nrow[S] = neighbour block in lexicographic neighbour slot S (centre = b).
template <int DIM, int Q, typename T, bool SOLID>
__device__ __forceinline__ void push_cell(const typename ST<T>::C (&g)[Q], typename ST<T>::C ux,
                                          typename ST<T>::C uy, typename ST<T>::C uz, int b, int t,
                                          const int *nrow, bool hook, T *__restrict__ fo, const StepArgs &a,
                                          unsigned seed)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    // Neighbour-slot and wrapped-cell components per axis offset -1, 0, +1
    // (util_index.h:45-98): slot S = sx + sy + sz, cell = nx + ny + nz.
    const int sx[3] = {I > 0 ? 1 : 0, 1, I < 3 ? 1 : 2};
    const int nx[3] = {(I + 3) & 3, I, (I + 1) & 3};
    const int sy[3] = {J > 0 ? 3 : 0, 3, J < 3 ? 3 : 6};
    const int ny[3] = {4 * ((J + 3) & 3), 4 * J, 4 * ((J + 1) & 3)};
    const int sz[3] = {DIM == 3 ? (K > 0 ? 9 : 0) : 0, DIM == 3 ? 9 : 0, DIM == 3 ? (K < 3 ? 9 : 18) : 0};
    const int nz[3] = {16 * ((K + 3) & 3), 16 * K, 16 * ((K + 1) & 3)};
    T *__restrict__ own = fo + (long long)b * BLK + t;
    const unsigned rc = a.sr ? sr_cell_of<DIM>(b, t, seed) : 0u;
    // The reference streams in place: the owner x of a pair (p in the half
    // set) swaps its f*_p with the neighbour y's f*_pb only if that value is
    // positive (kernels.cu:620-628, the solid-cell guard f_pb > 0).  Here each
    // cell pushes unconditionally; the cell on the non-owning side of an open
    // link, which holds that value, records the link when it is not positive,
    // and k_stream_fixup swaps the two pushed entries back, which is exactly
    // the refused swap.  Non-positive populations are rare (strong
    // over-relaxation near singular corners), so the list stays short.
    auto guard = [&](int p, bool open, long long dst) {
        if (p == 0 || lat_half(DIM, p) || !open) return;
        const C full = g[p] + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        if (full > C(0)) return;
        const int k = atomicAdd(a.fix_count, 1);
        if (k < a.fix_cap) {
            a.fix_list[2 * k] = dst;
            a.fix_list[2 * k + 1] = (long long)b * BLK + p * MC + t;
        }
    };
    if (!hook) {
        // No boundary hook on this block: closed links are plain bounce-back.
#pragma unroll
        for (int p = 0; p < Q; p++) {
            const int cx = lat_c(DIM, 0, p) + 1, cy = lat_c(DIM, 1, p) + 1, cz = lat_c(DIM, 2, p) + 1;
            const int nb = nrow[sx[cx] + sy[cy] + sz[cz]];
            const int nc = nx[cx] + ny[cy] + (DIM == 3 ? nz[cz] : 0);
            bool open = nb >= 0;
            if (SOLID && open) open = __ldg(&a.cmask[(long long)nb * MC + nc]) != CELL_SOLID;
            const long long to = (long long)nb * BLK + lat_pb(DIM, p) * MC + nc;
            T *dst = open ? fo + to : own + p * MC;
            *dst = enc_r<T>(g[p], rc * sr_dir(p), a.sr);
            guard(p, open, to);
        }
    } else {
#pragma unroll
        for (int p = 0; p < Q; p++) {
            const int cx = lat_c(DIM, 0, p) + 1, cy = lat_c(DIM, 1, p) + 1, cz = lat_c(DIM, 2, p) + 1;
            const int nb = nrow[sx[cx] + sy[cy] + sz[cz]];
            const int nc = nx[cx] + ny[cy] + (DIM == 3 ? nz[cz] : 0);
            bool open = nb >= 0;
            if (SOLID && open) open = __ldg(&a.cmask[(long long)nb * MC + nc]) != CELL_SOLID;
            if (open) {
                const long long to = (long long)nb * BLK + lat_pb(DIM, p) * MC + nc;
                fo[to] = enc_r<T>(g[p], rc * sr_dir(p), a.sr);
                guard(p, true, to);
            } else {
                C v = g[p];
                if (nb != N_SKIPID) {   // domain boundary: Cu_ImposeBC hook (kernels.cu:791-792)
                    const C wp = C(lat_w(Q, p));
                    const C off = ST<T>::OFF ? wp : C(0);
                    v = bc_hook<C>(a.bc_preset, nb, v + off, ux, uy, uz, wp, cx - 1, cy - 1, cz - 1, C(a.u_ref)) -
                        off;
                }
                own[p * MC] = enc_r<T>(v, rc * sr_dir(p), a.sr);
            }
        }
    }
}

}  // namespace agal
