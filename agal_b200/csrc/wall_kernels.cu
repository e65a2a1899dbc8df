// Wall blocks of a geometry: the step with the interpolated bounce-back and
// the momentum-exchange (MEA) forces.
//
// A wall block is a block on a boundary (cblock_ID_onb == 1) with a wall slot
// (cblock_ID_onb_solid >= 0).  When S_BC_TYPE > 0 the main step kernels skip
// them (META_WALL) and k_step_wall steps them instead: collide, then for each
// direction pair (p, pb) the reference's order of Cu_ImposeBC
// (solver_lbm_kernels.cu:769-876): boundary hook of p, interpolated
// bounce-back of p, hook of pb, bounce-back of pb; then the push with the
// stream guard.  The bounce-back needs the post-collision population of the
// cell behind the boundary cell; the step reads the previous buffer only, so
// that value is recomputed from it (one collision per link with 0 < q < 1/2).
// The reference reads it while other blocks rewrite their own pairs; here
// every block sees the values before the boundary phase.
//
// k_forces (Cu_ComputeForcesMEA, solver_lbm_kernels_forces.cu:324-537) sums
// per wall block of the finest level the momentum carried along the wall
// links of boundary cells, before the stream (post = 0, from the recomputed
// post-collision populations) and after it (post = 1, from the new buffer),
// into cblock_f_Ff; agal_forces reduces the partials in FP64.
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "ctx.h"
#include "dispatch.cuh"
#include "step_common.cuh"

namespace agal {
namespace {

struct WallArgs {
    StepArgs s;
    const int *wall;          // wall blocks of the level
    const int *onb_solid;
    const float *Xb;          // [27][ncb]
    long long ncb;
    int bc_type;
    int *status;
};

template <int DIM, int Q, typename T>
__device__ __forceinline__ typename ST<T>::C full_of(T v, int slot)
{
    using C = typename ST<T>::C;
    return ST<T>::dec(v) + (ST<T>::OFF ? C(lat_w(Q, slot)) : C(0));
}

// Post-collision value of direction k at cell nc of block nb, as the
// reference's collide kernel leaves it in slot k: collided for an active
// block's fluid cell, the stored value otherwise (solid guard, inactive block).
template <int DIM, int Q, typename T>
__device__ typename ST<T>::C post_collision(const StepArgs &a, int nb, int nc, int k)
{
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC, W = Meta<DIM>::W;
    const T *fin = static_cast<const T *>(a.fin) + (long long)nb * BLK + nc;
    const bool active = (__ldg(&a.meta[(long long)nb * W + Meta<DIM>::FLAGS]) & META_ACTIVE) != 0;
    if (!active || __ldg(&a.cmask[(long long)nb * MC + nc]) == CELL_SOLID) return full_of<DIM, Q, T>(fin[k * MC], k);
    C g[Q];
#pragma unroll
    for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(fin[lat_pb(DIM, p) * MC]);
    C ux, uy, uz;
    collide_at<DIM, Q, T>(g, a, (long long)nb * MC + nc, ux, uy, uz);
    return g[k] + (ST<T>::OFF ? C(lat_w(Q, k)) : C(0));
}

// Interpolated bounce-back of one link (solver_lbm_kernels.cu:816-824).
template <typename C>
__device__ __forceinline__ C bouzidi(C f, C f_m, C f_o, float dQf)
{
    const C dQ = C(dQf);
    const C two_q = r_mul(C(2), dQ);
    if (dQf > 0.f && dQf < 0.5f) return r_add(r_mul(two_q, f), r_mul(r_add(C(1), -two_q), f_m));
    return r_add(r_mul(r_div(C(1), two_q), f), r_mul(r_div(r_add(two_q, -C(1)), two_q), f_o));
}

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(Geo<DIM>::MC) k_step_wall(const WallArgs w)
{
    pdl_wait();
    const unsigned seed = step_seed(w.s);
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC, W = Meta<DIM>::W;
    const StepArgs &a = w.s;
    __shared__ int s_meta[W];
    const int b = w.wall[blockIdx.x];
    const int t = threadIdx.x;
    for (int i = t; i < W; i += MC) s_meta[i] = a.meta[(long long)b * W + i];
    __syncthreads();
    // Post-collision values of this block's cells (full populations), the
    // f_m the interpolated bounce-back reads from the cell behind a link when
    // that cell is in the same block; other blocks' cells are recomputed.
    __shared__ C sPost[Q][MC];
    const int mask = a.cmask[(long long)b * MC + t];
    const T *fin = static_cast<const T *>(a.fin) + (long long)b * BLK + t;
    if (!(s_meta[Meta<DIM>::FLAGS] & META_ACTIVE)) {   // uniform per CTA
        // untouched by the reference's in-place step: carried over unchanged
        T *fo = static_cast<T *>(a.fout) + (long long)b * BLK + t;
#pragma unroll
        for (int sl = 0; sl < Q; sl++) fo[sl * MC] = fin[sl * MC];
        return;
    }
    const bool solid = mask == CELL_SOLID;
    C g[Q];
#pragma unroll
    for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(fin[lat_pb(DIM, p) * MC]);
    C ux = C(0), uy = C(0), uz = C(0);
    // multi-level LES: the macro rows of every cell of the block, before the
    // collision (Cu_CollideLES, solver_lbm_kernels.cu:337-350)
    if (a.macro) store_macros<DIM, Q, C, ST<T>::OFF>(g, a.macro, a.nmc, (long long)b * MC + t);
    if (!solid) collide_at<DIM, Q, T>(g, a, (long long)b * MC + t, ux, uy, uz);
#pragma unroll
    for (int p = 0; p < Q; p++) sPost[p][t] = g[p] + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
    __syncthreads();
    if (solid) {
        // untouched by the reference's in-place step: carried over unchanged
        T *fo = static_cast<T *>(a.fout) + (long long)b * BLK + t;
#pragma unroll
        for (int sl = 0; sl < Q; sl++) fo[sl * MC] = fin[sl * MC];
        return;
    }
    auto post = [&](int nbh, int nc, int k) {
        return nbh == b ? sPost[k][nc] : post_collision<DIM, Q, T>(a, nbh, nc, k);
    };
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    const int slot = w.onb_solid[b];
    const bool wall = w.bc_type > 0 && mask == CELL_BOUNDARY && slot > -1;
    const bool hook = a.bc_preset != AGAL_BC_NONE;
    const int *nrow = s_meta;
    auto nbr_at = [&](int p, int sgn, int &nc) {
        const int Ip = I + sgn * lat_c(DIM, 0, p), Jp = J + sgn * lat_c(DIM, 1, p);
        const int Kp = (DIM == 3) ? K + sgn * lat_c(DIM, 2, p) : 0;
        nc = nbr_cell(DIM, Ip, Jp, Kp);
        return nrow[nbr_slot(DIM, Ip, Jp, Kp)];
    };
    for (int p = 1; p < Q; p++) {
        if (!lat_half(DIM, p)) continue;
        const int q = lat_pb(DIM, p);
        const C wp = C(lat_w(Q, p)), wq = C(lat_w(Q, q));
        const C offp = ST<T>::OFF ? wp : C(0), offq = ST<T>::OFF ? wq : C(0);
        C fp = g[p] + offp, fq = g[q] + offq;
        int nc;
        int nb = nbr_at(p, 1, nc);
        if (hook && nb < 0 && nb != N_SKIPID)
            fp = bc_hook<C>(a.bc_preset, nb, fp, ux, uy, uz, wp, lat_c(DIM, 0, p), lat_c(DIM, 1, p), lat_c(DIM, 2, p),
                            C(a.u_ref));
        if (wall) {
            const float dQ = w.Xb[(long long)slot * MC + t + (long long)p * w.ncb];
            if (dQ > 0.f) {
                C fm = C(0);
                if (dQ < 0.5f) {
                    const int nbh = nbr_at(q, 1, nc);
                    if (nbh < 0) atomicCAS(w.status, 0, AGAL_ERR_STATE);
                    else fm = post(nbh, nc, p);
                }
                fp = bouzidi<C>(fp, fm, fq, dQ);
            }
        }
        nb = nbr_at(q, 1, nc);
        if (hook && nb < 0 && nb != N_SKIPID)
            fq = bc_hook<C>(a.bc_preset, nb, fq, ux, uy, uz, wq, lat_c(DIM, 0, q), lat_c(DIM, 1, q), lat_c(DIM, 2, q),
                            C(a.u_ref));
        if (wall) {
            const float dQ = w.Xb[(long long)slot * MC + t + (long long)q * w.ncb];
            if (dQ > 0.f) {
                C fm = C(0);
                if (dQ < 0.5f) {
                    const int nbh = nbr_at(p, 1, nc);
                    if (nbh < 0) atomicCAS(w.status, 0, AGAL_ERR_STATE);
                    else fm = post(nbh, nc, q);
                }
                fq = bouzidi<C>(fq, fm, fp, dQ);
            }
        }
        g[p] = fp - offp;
        g[q] = fq - offq;
    }
    T *__restrict__ fo = static_cast<T *>(a.fout);
    push_cell<DIM, Q, T, true>(g, ux, uy, uz, b, t, nrow, false, fo, a, seed);
}

struct ForceArgs {
    StepArgs s;               // fin = the buffer read, meta, cmask, collision
    const int *wall;
    const int *onb_solid;
    const float *Xb;
    long long ncb, nmb;
    double dv;
    int order, post;
    void *Ff;                 // [6][nmb] compute type
    int *status;
};

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(Geo<DIM>::MC) k_forces(const ForceArgs fa)
{
    pdl_wait();
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC, W = Meta<DIM>::W;
    const StepArgs &a = fa.s;
    __shared__ int s_meta[W];
    __shared__ C s_F[3][MC];
    const int b = fa.wall[blockIdx.x];
    const int t = threadIdx.x;
    for (int i = t; i < W; i += MC) s_meta[i] = a.meta[(long long)b * W + i];
    __syncthreads();
    const int slot = fa.onb_solid[b];
    const int mask = a.cmask[(long long)b * MC + t];
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    const T *fin = static_cast<const T *>(a.fin);
    C s[3] = {C(0), C(0), C(0)};
    // Before the stream: every cell's post-collision values (stored values for
    // solid cells and inactive blocks) in shared memory, read for the cells
    // behind the links inside this block; other blocks' cells are recomputed.
    __shared__ C sPost[Q][MC];
    if (!fa.post) {
        const bool collide = (s_meta[Meta<DIM>::FLAGS] & META_ACTIVE) && mask != CELL_SOLID;
        C g[Q];
#pragma unroll
        for (int p = 0; p < Q; p++) g[p] = ST<T>::dec(fin[(long long)b * BLK + lat_pb(DIM, p) * MC + t]);
        C ux, uy, uz;
        if (collide) collide_at<DIM, Q, T>(g, a, (long long)b * MC + t, ux, uy, uz);
#pragma unroll
        for (int p = 0; p < Q; p++) sPost[p][t] = g[p] + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        __syncthreads();
    }
    if (mask == CELL_BOUNDARY && slot > -1) {
        // Populations in slot order: post-collision before the stream (the
        // cell's own collision), stored values after it.
        C f[Q];
        if (!fa.post) {
#pragma unroll
            for (int p = 0; p < Q; p++) f[p] = sPost[p][t];
        } else {
#pragma unroll
            for (int p = 0; p < Q; p++) f[p] = full_of<DIM, Q, T>(fin[(long long)b * BLK + p * MC + t], p);
        }
        for (int p = 1; p < Q; p++) {
            if (!lat_half(DIM, p)) continue;
            const int q = lat_pb(DIM, p);
            for (int side = 0; side < 2; side++) {
                const int ad = side ? q : p;   // link direction
                const int e = side ? p : q;    // towards the cell behind
                const float dist = fa.Xb[(long long)slot * MC + t + (long long)ad * fa.ncb];
                if (!(dist > 0.f)) continue;
                const int Ib = I + lat_c(DIM, 0, e), Jb = J + lat_c(DIM, 1, e);
                const int Kb = (DIM == 3) ? K + lat_c(DIM, 2, e) : 0;
                const int nbh = s_meta[nbr_slot(DIM, Ib, Jb, Kb)];
                const int nc = nbr_cell(DIM, Ib, Jb, Kb);
                if (nbh < 0) {
                    atomicCAS(fa.status, 0, AGAL_ERR_STATE);
                    continue;
                }
                const C fm = fa.post ? full_of<DIM, Q, T>(fin[(long long)nbh * BLK + ad * MC + nc], ad)
                                     : (nbh == b ? sPost[ad][nc] : post_collision<DIM, Q, T>(a, nbh, nc, ad));
                const C fa_ = f[ad];
                for (int d = 0; d < DIM; d++) {
                    const int cd = lat_c(DIM, d, ad);
                    if (fa.order == 1) {
                        s[d] = r_add(s[d], r_mul(fa_, C(cd)));
                    } else {
                        // The reference's 0.5 is a double literal: the term is formed in double.
                        const double qd = (double)(C)dist;
                        const double term = __dmul_rn(__dadd_rn(__dmul_rn(__dadd_rn(0.5, qd), (double)fa_),
                                                                __dmul_rn(__dadd_rn(0.5, -qd), (double)fm)),
                                                      (double)cd);
                        s[d] = (C)__dadd_rn((double)s[d], term);
                    }
                }
            }
        }
    }
    for (int d = 0; d < 3; d++) s_F[d][t] = s[d];
    __syncthreads();
    for (int h = MC / 2; h > 0; h >>= 1) {
        if (t < h)
            for (int d = 0; d < DIM; d++) s_F[d][t] = r_add(s_F[d][t], s_F[d][t + h]);
        __syncthreads();
    }
    if (t == 0) {
        C *Ff = static_cast<C *>(fa.Ff);
        const C dv = C(fa.dv);
        for (int d = 0; d < DIM; d++) {
            const C v = r_mul(s_F[d][0], dv);
            if (!fa.post) {
                Ff[b + (2 * d + 0) * fa.nmb] = v;
                Ff[b + (2 * d + 1) * fa.nmb] = C(0);
            } else {
                Ff[b + (2 * d + 0) * fa.nmb] = r_add(Ff[b + (2 * d + 0) * fa.nmb], v);
            }
        }
    }
}

template <int DIM, int Q, typename T>
StepArgs base_args(agal_ctx *c, int L, const void *fin, void *fout)
{
    StepArgs a{};
    a.ids = c->id_set + (long long)L * c->nmb;
    a.n = c->n_ids[L];
    a.fin = fin;
    a.fout = fout;
    a.meta = c->meta;
    a.cmask = c->cells_ID_mask;
    a.omega = c->dxf[L] / c->tau[L];
    if (sizeof(typename ST<T>::C) == 4) a.omega = (double)((float)c->dxf[L] / (float)c->tau[L]);
    a.u_ref = c->P.u_ref;
    a.bc_preset = c->P.bc_preset;
    a.mrt = (Q == 19 && c->P.collision == AGAL_MRT) ? 1 : 0;
    const double sv[5] = {c->P.s1, c->P.s2, c->P.s3, c->P.s5, c->P.s6};
    for (int k = 0; k < 5; k++) a.s[k] = (sizeof(typename ST<T>::C) == 4) ? (double)(float)sv[k] : sv[k];
    a.fix_count = c->fix_count;
    a.fix_list = c->fix_list;
    a.fix_cap = c->fix_cap;
    // the wall step rounds with the seed of its level step's main launch
    a.sr = (c->storage == AGAL_STORE_FP16 || c->storage == AGAL_STORE_BF16) &&
           c->P.half_rounding == AGAL_ROUND_STOCHASTIC;
    a.sr_ctr = c->d_sr;
    a.sr_salt = (unsigned)c->sr_salt;
    // LES: the eddy viscosity of the level's step (the wall step and the
    // force passes recompute the same collisions); the macro rows are written
    // by the wall step only (set by its launcher)
    a.nu_sgs = c->nu_sgs;
    a.nu = (sizeof(typename ST<T>::C) == 4) ? (double)(float)c->P.v0 : c->P.v0;
    a.dxL = (sizeof(typename ST<T>::C) == 4) ? (double)(float)c->dxf[L] : c->dxf[L];
    a.macro = nullptr;
    a.nmc = c->nmc;
    return a;
}

template <int DIM, int Q, typename T> struct RunWallStep {
    static int run(agal_ctx *c, int L, const void *fin, void *fout)
    {
        if constexpr (DIM != 3) {
            return AGAL_OK;
        } else {
            const int n = c->wall_n.empty() ? 0 : c->wall_n[L];
            if (n <= 0) return AGAL_OK;
            WallArgs w;
            w.s = base_args<DIM, Q, T>(c, L, fin, fout);
            w.s.macro = agal_les_macros(c) ? c->macro : nullptr;
            w.wall = c->wall_ids + c->wall_off[L];
            w.onb_solid = c->onb_solid;
            w.Xb = c->X_b;
            w.ncb = c->n_maxcells_b;
            w.bc_type = c->P.S_BC_TYPE;
            w.status = c->d_status;
            AGAL_CUDA(c, launch_pdl(k_step_wall<DIM, Q, T>, dim3(n), dim3(Geo<DIM>::MC), 0, c->stream, w));
            AGAL_CUDA(c, cudaGetLastError());
            return AGAL_OK;
        }
    }
};

template <int DIM, int Q, typename T> struct RunForces {
    static int run(agal_ctx *c, int L, int post)
    {
        if constexpr (DIM != 3) {
            return AGAL_OK;
        } else {
            const int n = c->wall_n.empty() ? 0 : c->wall_n[L];
            if (n <= 0 || !c->X_b || !c->Ff) return AGAL_OK;
            ForceArgs fa;
            fa.s = base_args<DIM, Q, T>(c, L, c->F[c->cur[L]], nullptr);
            fa.wall = c->wall_ids + c->wall_off[L];
            fa.onb_solid = c->onb_solid;
            fa.Xb = c->X_b;
            fa.ncb = c->n_maxcells_b;
            fa.nmb = c->nmb;
            // dvf_vec (solver_lbm_init.cu:21-27): dx_L^dim in ufloat_t.
            double dv = 1.0;
            for (int d = 0; d < DIM; d++) dv = (sizeof(typename ST<T>::C) == 4) ? (double)((float)dv * (float)c->dxf[L])
                                                                                 : dv * c->dxf[L];
            fa.dv = dv;
            fa.order = c->P.S_FORCE_ORDER;
            fa.post = post;
            fa.Ff = c->Ff;
            fa.status = c->d_status;
            AGAL_CUDA(c, launch_pdl(k_forces<DIM, Q, T>, dim3(n), dim3(Geo<DIM>::MC), 0, c->stream, fa));
            AGAL_CUDA(c, cudaGetLastError());
            return AGAL_OK;
        }
    }
};

// Control-volume forces (S_FORCE_TYPE 1; Cu_ComputeForcesCV,
// solver_lbm_kernels_forces.cu:13-245): per block of level L, over the cells
// whose centre lies strictly inside the box S_FORCEVOLUME_* and that are not
// solid, the momentum of the leaf blocks before the step (row 2d) and after it
// (row 2d+1), and, on the root level only, the momentum leaving through the
// box's surface: before the step the BGK post-collision value at the root
// level's relaxation rate of each direction that points out of the box, after
// it the population arriving from outside.  Block sums by a tree reduction,
// times dx_L^d; the pre-step pass writes the rows, the post-step pass adds.
struct CvArgs {
    const int *ids;
    int n;
    const void *f;            // level L's current buffer
    const int *cmask, *nbr_child;
    const float *fX;          // block lower corners [d][nmb]
    long long nmb;
    double dx, dv, omega0;    // dx_L, dx_L^d, dx_0 / tau_0 in the compute type
    int root, post;
    double box[6];            // xm, xM, ym, yM, zm, zM
    void *Ff;                 // [6][nmb] compute type
};

template <int DIM, int Q, typename T>
__global__ void __launch_bounds__(Geo<DIM>::MC) k_forces_cv(const CvArgs a)
{
    pdl_wait();
    using C = typename ST<T>::C;
    constexpr int MC = Geo<DIM>::MC, BLK = Q * MC;
    __shared__ C sP[3][MC], sM[3][MC];
    const int b = a.ids[blockIdx.x];
    const int t = threadIdx.x;
#pragma unroll
    for (int d = 0; d < 3; d++) sP[d][t] = sM[d][t] = C(0);
    const int mask = a.cmask[(long long)b * MC + t];
    const bool leaf = a.nbr_child[b] < 0;
    const int I = t & 3, J = (t >> 2) & 3, K = (DIM == 3) ? (t >> 4) : 0;
    const C dx = C(a.dx);
    const C x = C(a.fX[b]) + dx * (C(0.5) + C(I));
    const C y = C(a.fX[a.nmb + b]) + dx * (C(0.5) + C(J));
    const C z = DIM == 3 ? C(a.fX[2 * a.nmb + b]) + dx * (C(0.5) + C(K)) : C(0);
    auto inside = [&](C px, C py, C pz) {
        const bool in2 = px > C(a.box[0]) && px < C(a.box[1]) && py > C(a.box[2]) && py < C(a.box[3]);
        return DIM == 2 ? in2 : (in2 && pz > C(a.box[4]) && pz < C(a.box[5]));
    };
    const bool pv = inside(x, y, z) && mask != CELL_SOLID;
    const T *fin = static_cast<const T *>(a.f) + (long long)b * BLK + t;
    C f[Q];
    C rho = 0, ru = 0, rv = 0, rw = 0;
#pragma unroll
    for (int p = 0; p < Q; p++) {
        const C v = ST<T>::dec(fin[lat_pb(DIM, p) * MC]) + (ST<T>::OFF ? C(lat_w(Q, p)) : C(0));
        rho += v;
        ru += v * C(lat_c(DIM, 0, p));
        rv += v * C(lat_c(DIM, 1, p));
        if (DIM == 3) rw += v * C(lat_c(DIM, 2, p));
        f[p] = v;
    }
    if (pv && leaf) {
        C(*s)[MC] = a.post ? sM : sP;
        s[0][t] += ru;
        s[1][t] += rv;
        if (DIM == 3) s[2][t] += rw;
    }
    if (a.root) {
        const C om = C(a.omega0), omp = C(1) - om;
        if (!a.post) {
            ru = ru / rho;
            rv = rv / rho;
            rw = rw / rho;
        }
#pragma unroll
        for (int p = 1; p < Q; p++) {
            C v = f[p];
            // direction of the population leaving (pre-step) or arriving (post-step)
            const int q = a.post ? lat_pb(DIM, p) : p;
            if (!a.post) {
                const C uu = ru * ru + rv * rv + rw * rw;
                const C cu = C(lat_c(DIM, 0, p)) * ru + C(lat_c(DIM, 1, p)) * rv + C(lat_c(DIM, 2, p)) * rw;
                v = v * omp + (C(lat_w(Q, p)) * rho * (C(1) + C(3) * cu + C(4.5) * cu * cu - C(1.5) * uu)) * om;
            }
            const bool ps = !inside(x + C(lat_c(DIM, 0, q)) * dx, y + C(lat_c(DIM, 1, q)) * dx,
                                    z + C(lat_c(DIM, 2, q)) * dx);
            if (ps && pv) {
                sM[0][t] += v * C(lat_c(DIM, 0, q));
                sM[1][t] += v * C(lat_c(DIM, 1, q));
                if (DIM == 3) sM[2][t] += v * C(lat_c(DIM, 2, q));
            }
        }
    }
    __syncthreads();
    for (int st = MC / 2; st > 0; st >>= 1) {
        if (t < st)
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                sP[d][t] = sP[d][t] + sP[d][t + st];
                sM[d][t] = sM[d][t] + sM[d][t + st];
            }
        __syncthreads();
    }
    if (t == 0) {
        C *F = static_cast<C *>(a.Ff);
        const C dv = C(a.dv);
        for (int d = 0; d < DIM; d++) {
            C *fp = F + b + (long long)(2 * d) * a.nmb, *fm = F + b + (long long)(2 * d + 1) * a.nmb;
            if (!a.post) {
                *fp = sP[d][0] * dv;
                *fm = sM[d][0] * dv;
            } else {
                *fp += sP[d][0] * dv;
                *fm += sM[d][0] * dv;
            }
        }
    }
}

template <int DIM, int Q, typename T> struct RunForcesCv {
    static int run(agal_ctx *c, int L, int post)
    {
        const int n = c->n_ids[L];
        if (n <= 0 || !c->Ff) return AGAL_OK;
        using Cc = typename ST<T>::C;
        const bool f32 = sizeof(Cc) == 4;
        CvArgs a{};
        a.ids = c->id_set + (long long)L * c->nmb;
        a.n = n;
        a.f = c->F[c->cur[L]];
        a.cmask = c->cells_ID_mask;
        a.nbr_child = c->cblock_ID_nbr_child;
        a.fX = c->cblock_f_X;
        a.nmb = c->nmb;
        a.dx = c->dxf[L];
        double dv = 1.0;
        for (int d = 0; d < DIM; d++) dv = f32 ? (double)((float)dv * (float)c->dxf[L]) : dv * c->dxf[L];
        a.dv = dv;
        a.omega0 = f32 ? (double)((float)c->dxf[c->L0] / (float)c->tau[c->L0]) : c->dxf[c->L0] / c->tau[c->L0];
        a.root = L == c->L0;
        a.post = post;
        // The box snapped to root-block boundaries, 4 int(b Nxi / 4) dx_0
        // (solver_lbm_init.cu:36-41), stored in the compute type.
        const agal_params &P = c->P;
        const double box[6] = {P.S_FORCEVOLUME_Xm, P.S_FORCEVOLUME_XM, P.S_FORCEVOLUME_Ym,
                               P.S_FORCEVOLUME_YM, P.S_FORCEVOLUME_Zm, P.S_FORCEVOLUME_ZM};
        const int nxi[3] = {c->Nx, c->Ny, c->Nz};
        for (int k = 0; k < 6; k++) {
            const double v = 4.0 * (double)(int)(box[k] * (double)(nxi[k / 2] / 4)) * c->dxf[0];
            a.box[k] = f32 ? (double)(float)v : v;
        }
        a.Ff = c->Ff;
        AGAL_CUDA(c, launch_pdl(k_forces_cv<DIM, Q, T>, dim3(n), dim3(Geo<DIM>::MC), 0, c->stream, a));
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
};

// S_ReportForces sums (solver_lbm_compute.cu:166-201): every row of the
// partials over block IDs below id_max[MAX_LEVELS], in FP64, in one CTA.
template <typename C>
__global__ void __launch_bounds__(256) k_force_sums(const C *Ff, long long nmb, int n, double *out)
{
    __shared__ double s[256];
    for (int r = 0; r < 6; r++) {
        double acc = 0.0;
        for (int b = threadIdx.x; b < n; b += 256) acc += (double)Ff[b + r * nmb];
        s[threadIdx.x] = acc;
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[r] = s[0];
        __syncthreads();
    }
}

}  // namespace
}  // namespace agal

int agal_launch_wall_step(agal_ctx *c, int L, const void *fin, void *fout)
{
    if (!agal_wall_active(c)) return AGAL_OK;
    return agal::dispatch<agal::RunWallStep>(c, L, fin, fout);
}

int agal_launch_forces_cv(agal_ctx *c, int L, int post)
{
    if (c->rec)
        return agal_record_other(c, AGAL_OP_FORCES_CV, L, [L, post](agal_ctx *x) { return agal_launch_forces_cv(x, L, post); });
    if (c->P.S_FORCE_TYPE != 1) return AGAL_OK;
    return agal::dispatch<agal::RunForcesCv>(c, L, post);
}

int agal_launch_forces(agal_ctx *c, int L, int post)
{
    if (c->rec)
        return agal_record_other(c, AGAL_OP_FORCES, L, [L, post](agal_ctx *x) { return agal_launch_forces(x, L, post); });
    if (!c->onb_solid || !c->X_b || c->P.S_FORCE_TYPE != 0) return AGAL_OK;
    return agal::dispatch<agal::RunForces>(c, L, post);
}

extern "C" int agal_forces(agal_ctx *c, double *out)
{
    // Solver_LBM::S_ReportForces (solver_lbm_compute.cu:166-215): the sums
    // {Fpx, Fmx, Fpy, Fmy, Fpz, Fmz} of the MEA partials in FP64, then the
    // partials are reset.  The force is factor (Fp - Fm) with factor =
    // 1 / dx of the finest level (S_FORCE_TYPE 0).
    if (!c || !out) return AGAL_ERR_PARAM;
    for (int r = 0; r < 6; r++) out[r] = 0.0;
    if (!c->Ff) return AGAL_OK;
    double *d_out = nullptr;
    AGAL_CUDA(c, cudaMalloc(&d_out, sizeof(double) * 6));
    const int n = c->id_max[c->max_levels];
    if (c->storage == AGAL_STORE_FP64)
        agal::k_force_sums<double><<<1, 256, 0, c->stream>>>(static_cast<const double *>(c->Ff), c->nmb, n, d_out);
    else
        agal::k_force_sums<float><<<1, 256, 0, c->stream>>>(static_cast<const float *>(c->Ff), c->nmb, n, d_out);
    const size_t cs = (c->storage == AGAL_STORE_FP64) ? 8 : 4;
    cudaError_t e = cudaMemcpyAsync(out, d_out, sizeof(double) * 6, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->Ff, 0, cs * 6 * c->nmb, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_out);
    if (e != cudaSuccess) return agal_cuda_check(c, e, "agal_forces");
    return AGAL_OK;
}
