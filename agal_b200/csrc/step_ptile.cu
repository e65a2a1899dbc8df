// Push-tile form of the fused collide + boundary + stream step for the root
// level of 2D cases (variant 6).
//
// Why: in the plain push step (variant 1) every post-collision value is
// stored into its destination cell by its own thread, so a warp's 2-byte (or
// 4-byte) stores land in many partly written sectors of up to eight blocks:
// the L1-to-L2 request path and the issue slots spent on per-direction
// neighbour lookups bound the step, and FP16 takes as long as FP32 for half
// the bytes.  Here a CTA owns a tile of 8 x 4 cell-blocks (32 x 16 cells, one
// cell per thread):
//  1. each thread loads its cell's Q populations (as variant 1) and collides
//     them (collide_cell, the same arithmetic as every variant);
//  2. every post-collision value goes to shared memory at a compile-time
//     offset from the thread's own cell (slot planes of the tile and a
//     one-cell halo ring, row-major), so the pushes are uniform across the
//     warp; only blocks with a missing neighbour (the domain boundary) add
//     the bounce-back of their closed links (boundary hook included) into
//     their own cells;
//  3. after one barrier the tile's output is written block by block: every
//     16-byte chunk of a block's slot rows whose values all came from inside
//     the tile (or from bounce-back) is one vector store; a chunk with
//     values pushed in from a neighbouring tile writes only its own cells;
//     the halo ring's values go to the neighbouring tiles' blocks.
// Stochastic rounding is keyed by the source cell and direction, and the
// reference's stream guard is recorded in the fix-up list as in variant 1,
// so the output is bit-identical to every other variant.  DRAM traffic stays
// one read and one write of each population; no cell is collided twice.
//
// Requirements (else the launcher runs variant 1): a 2D case, the root level
// L0 holding the whole root grid (IDs 0.. in x-fastest order), root blocks per
// side a multiple of 8 in x and 4 in y, no geometry, no LES, FP32, FP16 or
// BF16 storage.
#include <cuda_runtime.h>

#include <type_traits>

#include "ctx.h"
#include "lattice.cuh"
#include "step_common.cuh"
#include "storage.cuh"

namespace agal {
namespace {

constexpr int PBX = 8, PBY = 4;               // cell-blocks per tile in x and y
constexpr int PCX = 4 * PBX, PCY = 4 * PBY;   // 32 x 16 cells
constexpr int PNB = PBX * PBY;                // 32 blocks
constexpr int PNT = PCX * PCY;                // 512 threads, one cell each

template <typename T> struct PTile {
    // Slot planes hold the tile and a one-cell halo ring: cell (x, y) of the
    // tile, x in -1..32, y in -1..16, sits at row y + 1, column x + 4, so
    // that the tile's rows start 8-byte (half) or 16-byte (float) aligned.
    // With 40 elements per row a warp's two 4 x 4-cell blocks push to
    // (nearly) distinct banks.
    static constexpr int RS = 40;
    static constexpr int X0 = 4, Y0 = 1;               // column / row of tile cell (0, 0)
    static constexpr int PS = RS * (PCY + 2);           // plane stride (elements)
    static constexpr int CH = 16 / (int)sizeof(T);      // cells per 16-byte chunk (8 or 4)
    static constexpr int CPB = 9 * 16 / CH;             // chunks per block
    static constexpr int NCH = PNB * CPB;               // chunks per tile
    static constexpr int NHALO = 2 * (PCX + 2) + 2 * PCY;   // halo cells (100)
    static_assert((PS * (int)sizeof(T)) % 16 == 0 && (RS * (int)sizeof(T)) % 16 == 0, "plane alignment");
};

template <typename T>
__device__ __forceinline__ void copy_chunk(T *__restrict__ dst, const T *src)
{
    if constexpr (sizeof(T) == 2) {
        // two rows of four cells, 8 bytes each, into one 16-byte store
        const uint2 r0 = *reinterpret_cast<const uint2 *>(src);
        const uint2 r1 = *reinterpret_cast<const uint2 *>(src + PTile<T>::RS);
        *reinterpret_cast<uint4 *>(dst) = make_uint4(r0.x, r0.y, r1.x, r1.y);
    } else {
        *reinterpret_cast<float4 *>(dst) = *reinterpret_cast<const float4 *>(src);
    }
}

template <typename T>
__global__ void __launch_bounds__(PNT, 3) k_step_ptile(const StepArgs a, int nbx)
{
    using C = typename ST<T>::C;
    constexpr int MC = 16, BLK = 9 * MC, W = Meta<2>::W;
    constexpr int RS = PTile<T>::RS, PS = PTile<T>::PS, CH = PTile<T>::CH, CPB = PTile<T>::CPB;
    constexpr int X0 = PTile<T>::X0, Y0 = PTile<T>::Y0;
    __shared__ __align__(16) T s_out[9 * PS];
    __shared__ int s_meta[PNB][W];
    const int tid = threadIdx.x, lb = tid >> 4, t = tid & 15;
    const int I = t & 3, J = t >> 2;
    const int lbx = lb % PBX, lby = lb / PBX;
    const int tiles_x = nbx / PBX;
    const int bx0 = (blockIdx.x % tiles_x) * PBX, by0 = (blockIdx.x / tiles_x) * PBY;
    const int b = (bx0 + lbx) + nbx * (by0 + lby);   // root-grid ID, x fastest

    // Metadata rows of the tile's blocks (written only by mesh passes, so
    // read before the wait on the predecessor).
    for (int i = tid; i < PNB * W; i += PNT) {
        const int k = i / W, j = i - k * W;
        const int bk = (bx0 + k % PBX) + nbx * (by0 + k / PBX);
        s_meta[k][j] = __ldg(&a.meta[(long long)bk * W + j]);
    }
    const T *__restrict__ f0 = static_cast<const T *>(a.fin) + (long long)b * BLK + t;
    pdl_wait();
    const unsigned seed = step_seed(a);
    C g[9];
#pragma unroll
    for (int p = 0; p < 9; p++) g[p] = ST<T>::dec(__ldg(f0 + lat_pb(2, p) * MC));
    __syncthreads();

    const int *nrow = s_meta[lb];
    const int flags = nrow[Meta<2>::FLAGS];
    C ux, uy, uz;
    collide_cell<2, 9, T>(g, a, ux, uy, uz);
    const int x = 4 * lbx + I, y = 4 * lby + J;
    T *own_s = s_out + (y + Y0) * RS + (x + X0);
    T *__restrict__ fo = static_cast<T *>(a.fout);
    const unsigned rc = a.sr ? sr_cell_of<2>(b, t, seed) : 0u;
    // Every value goes to the tile's planes (the halo ring for destinations
    // outside the tile): slot pb(p) of the cell x + c_p.
#pragma unroll
    for (int p = 0; p < 9; p++) {
        const int cx = lat_c(2, 0, p), cy = lat_c(2, 1, p);
        own_s[lat_pb(2, p) * PS + cy * RS + cx] = enc_r<T>(g[p], rc * sr_dir(p), a.sr);
    }
    // Blocks with a missing neighbour (the domain boundary): closed links
    // bounce back into slot p of the cell itself, through the boundary hook
    // on boundary blocks (push_cell's closed links).
    if (flags & META_CLOSED) {
        const bool hook = (flags & META_ONB) && a.bc_preset != AGAL_BC_NONE;
#pragma unroll
        for (int p = 1; p < 9; p++) {
            const int cx = lat_c(2, 0, p), cy = lat_c(2, 1, p);
            const int nb = nrow[nbr_slot(2, I + cx, J + cy, 0)];
            if (nb >= 0) continue;
            C v = g[p];
            if (hook && nb != N_SKIPID) {   // domain boundary: Cu_ImposeBC hook (kernels.cu:791-792)
                const C wp = C(lat_w(9, p));
                const C off = ST<T>::OFF ? wp : C(0);
                v = bc_hook<C>(a.bc_preset, nb, v + off, ux, uy, uz, wp, cx, cy, 0, C(a.u_ref)) - off;
            }
            own_s[p * PS] = enc_r<T>(v, rc * sr_dir(p), a.sr);
        }
    }
    // The stream guard of push_cell: the non-owning side of an open link
    // records it when its value is not positive (rare; the destination's
    // global index is worked out only then).
#pragma unroll
    for (int p = 1; p < 9; p++) {
        if (lat_half(2, p)) continue;
        if (g[p] + (ST<T>::OFF ? C(lat_w(9, p)) : C(0)) > C(0)) continue;
        const int cx = lat_c(2, 0, p), cy = lat_c(2, 1, p);
        const int nb = nrow[nbr_slot(2, I + cx, J + cy, 0)];
        if (nb < 0) continue;   // closed link: bounce-back, nothing to refuse
        const long long to = (long long)nb * BLK + lat_pb(2, p) * MC + nbr_cell(2, I + cx, J + cy, 0);
        const int k = atomicAdd(a.fix_count, 1);
        if (k < a.fix_cap) {
            a.fix_list[2 * k] = to;
            a.fix_list[2 * k + 1] = (long long)b * BLK + p * MC + t;
        }
    }
    __syncthreads();

    // Output 1: chunk k = 16 bytes of slot s of tile block kb.  Slot s of
    // cell X holds the value pushed from X + c_s; it is this tile's unless
    // X + c_s lies outside the tile in an existing block (that tile stores it).
    for (int k = tid; k < PTile<T>::NCH; k += PNT) {
        const int kb = k / CPB, r = k - kb * CPB;
        const int s = r / (16 / CH), c0 = (r - s * (16 / CH)) * CH;
        const int kbx = kb % PBX, kby = kb / PBX;
        const int cxs = lat_c(2, 0, s), cys = lat_c(2, 1, s);
        const int x0 = 4 * kbx, y0 = 4 * kby + (c0 >> 2);
        const T *src = s_out + s * PS + (y0 + Y0) * RS + (x0 + X0);
        T *dst = fo + ((long long)(bx0 + kbx) + (long long)nbx * (by0 + kby)) * BLK + s * MC + c0;
        const bool inside = x0 + cxs >= 0 && x0 + 3 + cxs < PCX && y0 + cys >= 0 && y0 + CH / 4 - 1 + cys < PCY;
        if (inside) {
            copy_chunk<T>(dst, src);
        } else {
#pragma unroll
            for (int c = 0; c < CH; c++) {
                const int cc = c0 + c, Ic = cc & 3, Jc = cc >> 2;
                const int xs = x0 + Ic + cxs, ys = 4 * kby + Jc + cys;
                const bool ext = !((unsigned)xs < (unsigned)PCX && (unsigned)ys < (unsigned)PCY) &&
                                 s_meta[kb][nbr_slot(2, Ic + cxs, Jc + cys, 0)] >= 0;
                if (!ext) dst[c] = src[(c >> 2) * RS + (c & 3)];
            }
        }
    }
    // Output 2: the halo ring, pushed into the neighbouring tiles' blocks.
    // Halo cell h (x in -1..32, y in -1..16 on the ring) receives, in slot
    // pb(p), the value of the tile cell h - c_p for each direction p whose
    // source lies in the tile.
    for (int k = tid; k < PTile<T>::NHALO; k += PNT) {
        int hx, hy;
        if (k < PCX + 2) {
            hx = k - 1, hy = -1;
        } else if (k < 2 * (PCX + 2)) {
            hx = k - (PCX + 2) - 1, hy = PCY;
        } else if (k < 2 * (PCX + 2) + PCY) {
            hx = -1, hy = k - 2 * (PCX + 2);
        } else {
            hx = PCX, hy = k - 2 * (PCX + 2) - PCY;
        }
#pragma unroll
        for (int p = 1; p < 9; p++) {
            const int cx = lat_c(2, 0, p), cy = lat_c(2, 1, p);
            const int sx = hx - cx, sy = hy - cy;   // source cell in the tile
            if (!((unsigned)sx < (unsigned)PCX && (unsigned)sy < (unsigned)PCY)) continue;
            const int sb = (sx >> 2) + PBX * (sy >> 2), Is = sx & 3, Js = sy & 3;
            const int nb = s_meta[sb][nbr_slot(2, Is + cx, Js + cy, 0)];
            if (nb < 0) continue;                     // closed link: bounced back in the tile
            fo[(long long)nb * BLK + lat_pb(2, p) * MC + nbr_cell(2, Is + cx, Js + cy, 0)] =
                s_out[lat_pb(2, p) * PS + (hy + Y0) * RS + (hx + X0)];
        }
    }
    if (a.fix_ticket) fused_fixup<T>(a);
}

}  // namespace

// Launch the push-tile step of the root level; AGAL_ERR_UNSUPPORTED when the
// case has no push tiles (the caller runs another variant).
template <int DIM, int Q, typename T>
int launch_step_ptile(agal_ctx *c, const StepArgs &a, int L)
{
    if constexpr (DIM != 2 || Q != 9 || std::is_same<T, double>::value) {
        return AGAL_ERR_UNSUPPORTED;
    } else {
        if (L != c->L0 || c->n_ptiles <= 0 || c->nu_sgs) return AGAL_ERR_UNSUPPORTED;
        AGAL_CUDA(c, launch_pdl(k_step_ptile<T>, dim3(c->n_ptiles), dim3(PNT), 0, c->stream, a, c->Nx / 4));
        AGAL_CUDA(c, cudaGetLastError());
        return AGAL_OK;
    }
}

#define AGAL_PTILE_INST(D, Q, T) template int launch_step_ptile<D, Q, T>(agal_ctx *, const StepArgs &, int);
AGAL_PTILE_INST(2, 9, float)
AGAL_PTILE_INST(2, 9, double)
AGAL_PTILE_INST(2, 9, __half)
AGAL_PTILE_INST(2, 9, __nv_bfloat16)
AGAL_PTILE_INST(3, 19, float)
AGAL_PTILE_INST(3, 19, double)
AGAL_PTILE_INST(3, 19, __half)
AGAL_PTILE_INST(3, 19, __nv_bfloat16)
AGAL_PTILE_INST(3, 27, float)
AGAL_PTILE_INST(3, 27, double)
AGAL_PTILE_INST(3, 27, __half)
AGAL_PTILE_INST(3, 27, __nv_bfloat16)

}  // namespace agal

// Number of push tiles of the root level (0 = variant 6 not available);
// called by agal_build_tiles after mesh changes.
int agal_count_ptiles(const agal_ctx *c)
{
    using namespace agal;
    if (c->dim != 2 || c->geometry_init) return 0;
    const int nbx = c->Nx / 4, nby = c->Ny / 4;
    if (nbx % PBX || nby % PBY || c->n_ids[c->L0] != nbx * nby) return 0;
    return (nbx / PBX) * (nby / PBY);
}
