// Context life cycle, root grid, host<->device array transfers and the
// advance entry points of the C ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "ctx.h"
#include "lattice.cuh"
#include "storage.cuh"

using namespace agal;

static std::string g_create_err;

int agal_set_err(agal_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg; else g_create_err = msg;
    return code;
}

int agal_cuda_check(agal_ctx *c, cudaError_t e, const char *what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return agal_set_err(c, AGAL_ERR_OOM, m);
    return agal_set_err(c, AGAL_ERR_CUDA, m);
}

namespace {

// Padded root-grid value (mesh_init.cu:406-460): boundaries are written z,
// then y, then x, so x wins at edges/corners; periodic faces wrap.
int root_padded_id(const agal_ctx *c, int bx, int by, int bz, int i, int j, int k)
{
    if (i < 1 || i > bx) {
        if (!c->P.PERIODIC_X) return (i < 1) ? -1 : -2;
        i = (i < 1) ? bx : 1;
    }
    if (j < 1 || j > by) {
        if (!c->P.PERIODIC_Y) return (j < 1) ? -3 : -4;
        j = (j < 1) ? by : 1;
    }
    if (c->dim == 3 && (k < 1 || k > bz)) {
        if (!c->P.PERIODIC_Z) return (k < 1) ? -5 : -6;
        k = (k < 1) ? bz : 1;
    }
    if (c->dim == 2) k = 1;
    return (i - 1) + bx * ((j - 1) + by * (k - 1));
}

template <typename T>
__global__ void k_fill(T *p, long long n, T v)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

template <typename T>
int fill(agal_ctx *c, T *p, long long n, T v)
{
    if (n <= 0) return AGAL_OK;
    k_fill<T><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(p, n, v);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

size_t compute_size(const agal_ctx *c) { return c->storage == AGAL_STORE_FP64 ? 8 : 4; }

}  // namespace

void agal_drop_graphs(agal_ctx *c)
{
    c->graph_steps = 0;
    c->graph_cur_in.clear();
    for (int k = 0; k < 2; k++) c->ml_graph_cur[k].clear();
}

void agal_free_graphs(agal_ctx *c)
{
    agal_drop_graphs(c);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
    for (int k = 0; k < 2; k++) {
        if (c->ml_graph[k]) cudaGraphExecDestroy(c->ml_graph[k]);
        c->ml_graph[k] = nullptr;
    }
}

namespace {

void release(agal_ctx *c)
{
    agal_free_graphs(c);
    agal_geometry_release(c);
    void *ptrs[] = {c->F[0], c->F[1], c->macro, c->cells_ID_mask, c->cblock_f_X, c->cblock_ID_mask,
                    c->cblock_ID_nbr, c->cblock_ID_nbr_child, c->cblock_ID_onb, c->cblock_ID_ref,
                    c->cblock_level, c->id_set, c->gap_set, c->red, c->red_out, c->d_status, c->meta,
                    c->amr, c->fix_count, c->fix_list, c->crit, c->iface_ids, c->nu_sgs, c->blk_solid,
                    c->tiles, c->xfer};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (c->h_small) cudaFreeHost(c->h_small);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
}

}  // namespace

extern "C" const char *agal_last_error(const agal_ctx *ctx)
{
    return ctx ? ctx->err.c_str() : g_create_err.c_str();
}

extern "C" int agal_ctx_create(const agal_params *p, agal_ctx **out)
{
    if (!p || !out) return agal_set_err(nullptr, AGAL_ERR_PARAM, "null argument");
    *out = nullptr;
    agal_ctx *c = new (std::nothrow) agal_ctx();
    if (!c) return agal_set_err(nullptr, AGAL_ERR_OOM, "host allocation failed");
    c->P = *p;
    switch (p->velocity_set) {
    case AGAL_D2Q9: c->dim = 2; c->Q = 9; break;
    case AGAL_D3Q19: c->dim = 3; c->Q = 19; break;
    case AGAL_D3Q27: c->dim = 3; c->Q = 27; break;
    default: delete c; return agal_set_err(nullptr, AGAL_ERR_PARAM, "velocity_set");
    }
    if (p->collision != AGAL_BGK && !(p->collision == AGAL_MRT && p->velocity_set == AGAL_D3Q19)) {
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_UNSUPPORTED, "collision operator: BGK, or MRT with D3Q19");
    }
    if (p->S_LES < 0 || p->S_LES > 3) { delete c; return agal_set_err(nullptr, AGAL_ERR_PARAM, "S_LES: 0..3"); }
    if (p->half_rounding != AGAL_ROUND_STOCHASTIC && p->half_rounding != AGAL_ROUND_NEAREST) {
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_PARAM, "half_rounding");
    }
    if (p->S_LES > 0 && p->collision != AGAL_BGK) {
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_UNSUPPORTED, "S_LES: built for BGK (Cu_CollideLES)");
    }
    c->Qmax = (c->dim == 2) ? 9 : 27;
    c->MC = (c->dim == 2) ? 16 : 64;
    c->NCH = (c->dim == 2) ? 4 : 8;
    c->storage = p->storage;
    switch (p->storage) {
    case AGAL_STORE_FP32: c->esize = 4; break;
    case AGAL_STORE_FP64: c->esize = 8; break;
    case AGAL_STORE_FP16:
    case AGAL_STORE_BF16: c->esize = 2; break;
    default: delete c; return agal_set_err(nullptr, AGAL_ERR_PARAM, "storage");
    }

    // mesh_init.cu:22-91
    const float Lx = (float)p->L_c;
    const float Ly = (float)(p->L_fy * Lx);
    const float Lz = (float)(p->L_fz * Lx);
    c->Nx = p->Nx;
    c->Ny = (int)(c->Nx * (Ly / Lx));
    c->Nz = (c->dim == 2) ? 1 : (int)(c->Nx * (Lz / Lx));
    if (c->Nx <= 0 || c->Nx % 4 || c->Ny <= 0 || c->Ny % 4 || (c->dim == 3 && (c->Nz <= 0 || c->Nz % 4))) {
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_PARAM, "grid sizes must be positive multiples of 4");
    }
    c->dx = Lx / (float)c->Nx;
    c->dx_cblock = 4.0f * c->dx;
    c->max_levels = std::max(p->MAX_LEVELS_WALL, p->MAX_LEVELS_INTERIOR);
    if (c->max_levels < 1 || c->max_levels > 16) { delete c; return agal_set_err(nullptr, AGAL_ERR_PARAM, "MAX_LEVELS"); }
    c->L0 = p->N_LEVEL_START;
    if (c->max_levels == 1) c->L0 = 0;
    if (c->L0 > c->max_levels - 1) c->L0 = c->max_levels - 1;
    const bool fp64 = (p->storage == AGAL_STORE_FP64);
    c->dxf.resize(c->max_levels);
    c->tau.resize(c->max_levels);
    for (int L = 0; L < c->max_levels; L++) {
        const double d = (double)c->dx / std::pow(2.0, (double)L);
        c->dxf[L] = fp64 ? d : (double)(float)d;
        // solver_lbm_init.cu:51: tau_L = v0*3 + 0.5*dx_L, rounded to ufloat_t.
        const double t = p->v0 * 3.0 + 0.5 * c->dxf[L];
        c->tau[L] = fp64 ? t : (double)(float)t;
    }

    const int bx = c->Nx / 4, by = c->Ny / 4, bz = (c->dim == 2) ? 1 : c->Nz / 4;
    const long long n_coarse = (long long)bx * by * bz;

    int rc;
    if (p->device >= 0 && cudaSetDevice(p->device) != cudaSuccess) {
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_CUDA, "cudaSetDevice failed");
    }
    if ((rc = cudaGetDevice(&c->device)) != cudaSuccess) { delete c; return agal_set_err(nullptr, AGAL_ERR_CUDA, "no CUDA device"); }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        release(c);
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_CUDA, "stream creation failed");
    }

    // Capacity: explicit, or from free memory like mesh_init.cu:155-169.
    const size_t per_block =
        (size_t)c->MC * (2 * c->Q * c->esize + (c->dim + 1) * compute_size(c) + sizeof(int)) +
        sizeof(float) * c->dim + sizeof(int) * (2 * c->Qmax + 5 + c->max_levels) +
        (c->max_levels > 1 ? 7 * sizeof(int) + sizeof(double) : 0) +
        (size_t)c->MC / 4 * 2 * sizeof(long long);   // stream-guard fix-up list
    if (p->n_maxcblocks > 0) {
        c->nmb = p->n_maxcblocks;
    } else {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        const double frac = (p->mem_frac > 0 && p->mem_frac < 1) ? p->mem_frac : 0.975;
        long long ncell = (long long)((double)fr * frac / (double)per_block) * c->MC;
        ncell = ((ncell + 1024) / 2048) * 2048;   // M_RNDOFF
        c->nmb = ncell / c->MC;
    }
    if (n_coarse > c->nmb) {
        release(c);
        delete c;
        return agal_set_err(nullptr, AGAL_ERR_OOM, "ERROR: Root grid size exceeds limits...");
    }
    c->nmc = c->nmb * c->MC;
    const long long nmb = c->nmb, nmc = c->nmc;

#define ALLOC(ptr, bytes)                                                              \
    do {                                                                               \
        if (cudaMalloc((void **)&(ptr), (bytes)) != cudaSuccess) {                     \
            cudaGetLastError();                                                        \
            release(c);                                                                \
            delete c;                                                                  \
            return agal_set_err(nullptr, AGAL_ERR_OOM, "device allocation failed: " #ptr); \
        }                                                                              \
    } while (0)
    ALLOC(c->F[0], c->esize * (size_t)c->Q * nmc);
    ALLOC(c->F[1], c->esize * (size_t)c->Q * nmc);
    ALLOC(c->macro, compute_size(c) * (size_t)(c->dim + 1) * nmc);
    ALLOC(c->cells_ID_mask, sizeof(int) * nmc);
    ALLOC(c->cblock_f_X, sizeof(float) * c->dim * nmb);
    ALLOC(c->cblock_ID_mask, sizeof(int) * nmb);
    ALLOC(c->cblock_ID_nbr, sizeof(int) * c->Qmax * nmb);
    ALLOC(c->cblock_ID_nbr_child, sizeof(int) * c->Qmax * nmb);
    ALLOC(c->cblock_ID_onb, sizeof(int) * nmb);
    ALLOC(c->cblock_ID_ref, sizeof(int) * nmb);
    ALLOC(c->cblock_level, sizeof(int) * nmb);
    ALLOC(c->id_set, sizeof(int) * c->max_levels * nmb);
    ALLOC(c->gap_set, sizeof(int) * nmb);
    ALLOC(c->red_out, sizeof(double) * 4);
    ALLOC(c->d_status, sizeof(int) * 4);
    ALLOC(c->meta, sizeof(int) * (size_t)(c->dim == 2 ? 12 : 28) * nmb);
    ALLOC(c->fix_count, sizeof(int) * 4);
    if (p->S_LES > 0) ALLOC(c->nu_sgs, (p->storage == AGAL_STORE_FP64 ? 8 : 4) * (size_t)nmb * c->MC);   // eddy viscosity
    if (p->S_FORCE_TYPE == 1) ALLOC(c->Ff, (p->storage == AGAL_STORE_FP64 ? 8 : 4) * 6 * (size_t)nmb);   // CV partials
    c->fix_cap = (int)std::min<long long>(std::max<long long>(nmc / 4, AGAL_FIX_CAP_MIN), 1LL << 26);
    ALLOC(c->fix_list, sizeof(long long) * 2 * (size_t)c->fix_cap);
    if (c->max_levels > 1) {
        const size_t na = agal_amr_scratch_ints(nmb);
        ALLOC(c->amr, sizeof(int) * na);
        c->amr_emap = c->amr;
        c->amr_first = c->amr + nmb;
        c->amr_a = c->amr + 2 * nmb;
        c->amr_b = c->amr + 3 * nmb;
        c->amr_snap = c->amr + 4 * nmb;
        c->amr_parts = c->amr + 5 * nmb;
        c->amr_small = c->amr + na - AGAL_AMR_SMALL;
        ALLOC(c->crit, sizeof(double) * nmb + sizeof(int) * 2 * 65536 + 256);
        if (cudaMallocHost((void **)&c->h_small, sizeof(int) * AGAL_AMR_SMALL) != cudaSuccess) {
            cudaGetLastError();
            c->h_small = nullptr;   // the readbacks fall back to pageable memory
        }
    }
#undef ALLOC
    cudaMemsetAsync(c->d_status, 0, sizeof(int) * 4, c->stream);
    c->d_sr = reinterpret_cast<unsigned *>(c->d_status + 2);
    cudaMemsetAsync(c->fix_count, 0, sizeof(int) * 4, c->stream);

    // Reset values, mesh_init.cu:285-304.
    if ((rc = fill<int>(c, c->cells_ID_mask, nmc, CELL_INTERIOR)) ||
        (rc = fill<int>(c, c->cblock_ID_mask, nmb, BLOCK_REGULAR)) ||
        (rc = fill<int>(c, c->cblock_ID_nbr, c->Qmax * nmb, N_SKIPID)) ||
        (rc = fill<int>(c, c->cblock_ID_nbr_child, c->Qmax * nmb, N_SKIPID)) ||
        (rc = fill<int>(c, c->cblock_ID_ref, nmb, REF_INACTIVE)) ||
        (rc = fill<int>(c, c->cblock_level, nmb, 0)) || (rc = fill<int>(c, c->cblock_ID_onb, nmb, 0)) ||
        // id_set / gap_set start zeroed as in the reference (mesh_init.cu
        // allocates them and fills only the live prefix); the refinement
        // pass reads slot 0 of an empty level as its id_max.
        (rc = fill<int>(c, c->id_set, c->max_levels * nmb, 0)) || (rc = fill<int>(c, c->gap_set, nmb, 0)) ||
        (rc = fill<float>(c, c->cblock_f_X, c->dim * nmb, 0.0f)) ||
        (c->amr && (rc = fill<int>(c, c->amr, 2 * nmb, -1)))) {
        std::string m = c->err;
        release(c);
        delete c;
        return agal_set_err(nullptr, rc, m);
    }
    cudaMemsetAsync(c->F[0], 0, c->esize * (size_t)c->Q * nmc, c->stream);
    cudaMemsetAsync(c->F[1], 0, c->esize * (size_t)c->Q * nmc, c->stream);
    cudaMemsetAsync(c->macro, 0, compute_size(c) * (size_t)(c->dim + 1) * nmc, c->stream);
    if (c->Ff) cudaMemsetAsync(c->Ff, 0, compute_size(c) * 6 * (size_t)nmb, c->stream);

    // Root grid (mesh_init.cu:354-516), built on the host and copied in.
    std::vector<int> nbr((size_t)c->Qmax * n_coarse), onb(n_coarse), ref(n_coarse, REF_UNREFINED);
    std::vector<float> fX((size_t)c->dim * n_coarse);
    for (int k = 1; k <= bz; k++)
        for (int j = 1; j <= by; j++)
            for (int i = 1; i <= bx; i++) {
                const int b = root_padded_id(c, bx, by, bz, i, j, k);
                fX[b] = (float)(i - 1) * c->dx_cblock;
                fX[b + n_coarse] = (float)(j - 1) * c->dx_cblock;
                if (c->dim == 3) fX[b + 2 * n_coarse] = (float)(k - 1) * c->dx_cblock;
                int on = 0;
                for (int q = 0; q < c->Qmax; q++) {
                    const int nb = root_padded_id(c, bx, by, bz, i + lat_c(c->dim, 0, q), j + lat_c(c->dim, 1, q),
                                                  k + lat_c(c->dim, 2, q));
                    nbr[b + (size_t)q * n_coarse] = nb;
                    if (nb < 0) on = 1;
                }
                onb[b] = on;
            }
    std::vector<int> gaps(nmb - n_coarse), ids(n_coarse);
    for (long long x = 0; x < n_coarse; x++) ids[x] = (int)x;
    for (long long x = 0; x < nmb - n_coarse; x++) gaps[x] = (int)((nmb - 1) - x);
#define H2D(dst, src, bytes) \
    do { cudaError_t e_ = cudaMemcpy((dst), (src), (bytes), cudaMemcpyHostToDevice); \
         if (e_ != cudaSuccess) { int r_ = agal_cuda_check(c, e_, "root grid copy"); std::string m = c->err; release(c); delete c; return agal_set_err(nullptr, r_, m); } } while (0)
    cudaStreamSynchronize(c->stream);
    H2D(c->cblock_ID_ref, ref.data(), sizeof(int) * n_coarse);
    for (int q = 0; q < c->Qmax; q++) {
        H2D(c->cblock_ID_nbr + (size_t)q * nmb, nbr.data() + (size_t)q * n_coarse, sizeof(int) * n_coarse);
        // nbr_child: boundary IDs copied, N_SKIPID elsewhere (mesh_init.cu:489)
        std::vector<int> ch(n_coarse);
        for (long long b = 0; b < n_coarse; b++) {
            const int v = nbr[b + (size_t)q * n_coarse];
            ch[b] = v < 0 ? v : N_SKIPID;
        }
        H2D(c->cblock_ID_nbr_child + (size_t)q * nmb, ch.data(), sizeof(int) * n_coarse);
    }
    H2D(c->cblock_ID_onb, onb.data(), sizeof(int) * n_coarse);
    for (int d = 0; d < c->dim; d++)
        H2D(c->cblock_f_X + (size_t)d * nmb, fX.data() + (size_t)d * n_coarse, sizeof(float) * n_coarse);
    H2D(c->id_set, ids.data(), sizeof(int) * n_coarse);
    if (!gaps.empty()) H2D(c->gap_set, gaps.data(), sizeof(int) * gaps.size());
#undef H2D
    c->n_ids.assign(c->max_levels + 1, 0);
    c->id_max.assign(c->max_levels + 1, 0);
    c->n_ids[0] = (int)n_coarse;
    c->id_max[0] = c->id_max[c->max_levels] = (int)n_coarse;
    c->n_gaps = (int)(nmb - n_coarse);
    c->cur.assign(c->max_levels, 0);
    if ((rc = agal_build_meta(c))) {
        std::string m = c->err;
        release(c);
        delete c;
        return agal_set_err(nullptr, rc, m);
    }
    *out = c;
    return AGAL_OK;
}

extern "C" int agal_ctx_destroy(agal_ctx *ctx)
{
    if (!ctx) return AGAL_ERR_PARAM;
    cudaStreamSynchronize(ctx->stream);
    release(ctx);
    delete ctx;
    return AGAL_OK;
}

extern "C" int agal_get_counts(const agal_ctx *c, int *n_ids, int *id_max, int *n_gaps, int64_t *n_maxcblocks,
                               int *max_levels)
{
    if (!c) return AGAL_ERR_PARAM;
    for (int L = 0; L <= c->max_levels; L++) {
        if (n_ids) n_ids[L] = c->n_ids[L];
        if (id_max) id_max[L] = c->id_max[L];
    }
    if (n_gaps) *n_gaps = c->n_gaps;
    if (n_maxcblocks) *n_maxcblocks = c->nmb;
    if (max_levels) *max_levels = c->max_levels;
    return AGAL_OK;
}

extern "C" int agal_set_counts(agal_ctx *c, const int *n_ids, const int *id_max, int n_gaps)
{
    if (!c || !n_ids || !id_max) return AGAL_ERR_PARAM;
    for (int L = 0; L <= c->max_levels; L++)
        if (n_ids[L] < 0 || n_ids[L] > c->nmb || id_max[L] > c->nmb)
            return agal_set_err(c, AGAL_ERR_PARAM, "agal_set_counts: count beyond the block pool");
    if (n_gaps < 0 || n_gaps > c->nmb) return agal_set_err(c, AGAL_ERR_PARAM, "agal_set_counts: n_gaps");
    for (int L = 0; L <= c->max_levels; L++) {
        c->n_ids[L] = n_ids[L];
        c->id_max[L] = id_max[L];
    }
    c->n_gaps = n_gaps;
    agal_drop_graphs(c);
    return agal_build_meta(c);
}

extern "C" int agal_sync(agal_ctx *c)
{
    if (!c) return AGAL_ERR_PARAM;
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    AGAL_CUDA(c, cudaGetLastError());
    // A bounded device wait that expired leaves its code in the status word.
    int st = 0;
    AGAL_CUDA(c, cudaMemcpy(&st, c->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) {
        cudaMemset(c->d_status, 0, sizeof(int));
        return agal_set_err(c, st, st == AGAL_ERR_TIMEOUT ? "a device wait timed out (pipeline stalled)"
                                                          : "stream-guard fix-up list overflowed in a step");
    }
    return AGAL_OK;
}

extern "C" int agal_get_stream(const agal_ctx *c, void **stream)
{
    if (!c || !stream) return AGAL_ERR_PARAM;
    *stream = (void *)c->stream;
    return AGAL_OK;
}

extern "C" int agal_autotune(agal_ctx *c, int L, int reps, float *ms, int *cells_per_thread)
{
    if (!c || L < 0 || L >= c->max_levels || reps <= 0) return AGAL_ERR_PARAM;
    agal_drop_graphs(c);   // launch shape changes
    int rc = agal_launch_tune(c, L, reps, ms);
    if (rc) return rc;
    if (cells_per_thread) *cells_per_thread = c->step_cpt;
    return AGAL_OK;
}

extern "C" int agal_set_tuning(agal_ctx *c, int cells_per_thread)
{
    if (!c || cells_per_thread < 1 || cells_per_thread > AGAL_STEP_VARIANTS) return AGAL_ERR_PARAM;
    agal_drop_graphs(c);
    int rc = agal_prepare_step(c);
    if (rc) return rc;
    c->step_cpt = cells_per_thread;
    return AGAL_OK;
}

extern "C" int agal_set_ic(agal_ctx *c, int L)
{
    if (!c || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    return agal_launch_set_ic(c, L);
}

extern "C" int agal_refresh(agal_ctx *c, int L)
{
    if (!c || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    return agal_launch_refresh(c, L);
}

extern "C" int agal_mass_momentum(agal_ctx *c, double *out)
{
    if (!c || !out) return AGAL_ERR_PARAM;
    return agal_launch_mass(c, out);
}

extern "C" int agal_mass_momentum_async(agal_ctx *c, double *out)
{
    if (!c || !out) return AGAL_ERR_PARAM;
    return agal_launch_mass_async(c, out);
}

// ---------------------------------------------------------------------------
// Level-interface transfers with the refresh the reference's S_Interpolate /
// S_Average perform first (solver_lbm_kernels_comm.cu:141-155, 351-370), so
// the macro array ends up as the reference's macro rows do.
extern "C" int agal_interpolate(agal_ctx *c, int L, int var)
{
    if (!c || L < 0 || L >= c->max_levels - 1) return AGAL_ERR_PARAM;
    if (var != AGAL_INTERP_INTERFACE && var != AGAL_INTERP_ADDED) return AGAL_ERR_PARAM;
    int rc = agal_launch_refresh(c, L);
    return rc ? rc : agal_launch_interp(c, L, var);
}

extern "C" int agal_average(agal_ctx *c, int L, int var)
{
    if (!c || L < 0 || L >= c->max_levels - 1) return AGAL_ERR_PARAM;
    if (var < AGAL_AVERAGE_INTERFACE || var > AGAL_AVERAGE_GRID) return AGAL_ERR_PARAM;
    int rc = agal_launch_refresh(c, L + 1);
    return rc ? rc : agal_launch_average(c, L, var);
}

extern "C" int agal_ref_criteria(agal_ctx *c)
{
    if (!c) return AGAL_ERR_PARAM;
    return agal_launch_criterion(c);
}

extern "C" int agal_refine_coarsen(agal_ctx *c)
{
    if (!c) return AGAL_ERR_PARAM;
    int rc = agal_refine_pass(c);
    if (rc) return rc;
    if (c->n_ref_last || c->n_coarse_last) agal_drop_graphs(c);   // launch sizes changed
    return AGAL_OK;
}

// Mesh::M_Advance_RefineWithSolution (mesh_advance.cu:185-243).
extern "C" int agal_refine_with_solution(agal_ctx *c)
{
    if (!c) return AGAL_ERR_PARAM;
    const int ML = c->max_levels;
    int rc;
    // mesh_advance.cu:191: not once the time average has started
    const bool averaging = c->P.N_PROBE_AVE != 0 && !(c->P.N_PROBE_AVE == 1 && c->iter + 1 <= c->P.N_PROBE_AVE_START);
    if (!(c->P.MAX_LEVELS_INTERIOR > 1) || averaging) return AGAL_OK;
    for (int L = ML - 2; L >= c->L0; L--)
        if ((rc = agal_average(c, L, AGAL_AVERAGE_GRID))) return rc;
    for (int L = c->L0; L < ML - 1; L++)
        if ((rc = agal_interpolate(c, L, AGAL_INTERP_INTERFACE))) return rc;
    if (c->learner) {
        if ((rc = agal_learn_marks(c))) return rc;
    } else if ((rc = agal_launch_criterion(c))) {
        return rc;
    }
    if ((rc = agal_refine_coarsen(c))) return rc;
    return c->learner ? agal_learn_after_regrid(c) : AGAL_OK;
}

// Mesh::M_Advance_RefineNearWall without geometry (mesh_advance.cu:54-122).
extern "C" int agal_refine_near_wall(agal_ctx *c)
{
    // Mesh::M_Advance_RefineNearWall (mesh_advance.cu:54-122), with the
    // voxelizer passes when a geometry is attached.
    if (!c) return AGAL_ERR_PARAM;
    const int ML = c->max_levels, MLW = c->P.MAX_LEVELS_WALL;
    const bool geo = c->geometry_init && c->faces;
    int rc;
    for (int L = 0; L < c->L0; L++) {
        if ((rc = agal_mark_level(c, L, 1))) return rc;
        if ((rc = agal_refine_coarsen(c))) return rc;
    }
    for (int L = c->L0; L < MLW; L++) {
        if (L < MLW - 1 && (rc = agal_mark_level(c, L, 0))) return rc;
        if (geo && (rc = agal_voxelize_s1(c, L))) return rc;
        if (ML > 1 && L < MLW - 1 && (rc = agal_refine_coarsen(c))) return rc;
        if (geo && (rc = agal_update_solid_children(c, L))) return rc;
        if ((rc = agal_launch_set_ic(c, L))) return rc;
    }
    if (geo) {
        for (int L = c->L0; L < MLW; L++)
            if ((rc = agal_voxelize_s2(c, L))) return rc;
        if ((rc = agal_voxelize_s3(c))) return rc;
        if (c->P.G_BIN_MAKE_LINKS)
            for (int L = c->L0; L < MLW; L++)
                if ((rc = agal_link_lengths(c, L))) return rc;
        // The wall flags of the step depend on the link lengths being present.
        if ((rc = agal_build_meta(c))) return rc;
    }
    if (ML > 1 && (rc = agal_freeze_refined(c))) return rc;
    return AGAL_OK;
}

extern "C" int agal_mesh_ref_criteria(agal_ctx *c, int L, int var)
{
    // Mesh::M_ComputeRefCriteria (mesh_criterion.cu:90-119).
    if (!c || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    switch (var) {
    case AGAL_MESH_REF_NW_CASES: return agal_mark_level(c, L, 0);
    case AGAL_MESH_REF_UNIFORM: return agal_mark_level(c, L, 1);
    case AGAL_MESH_REF_SOLUTION: return c->n_ids[L] > 0 ? agal_ref_criteria(c) : AGAL_OK;
    default: return agal_set_err(c, AGAL_ERR_PARAM, "mesh_ref_criteria: unknown var");
    }
}

extern "C" int agal_freeze_refined_cells(agal_ctx *c, int var)
{
    // Mesh::M_FreezeRefinedCells (mesh_amr.cu:2050-2074).
    if (!c || (var != 0 && var != 1)) return AGAL_ERR_PARAM;
    return agal_freeze_refined(c, var);
}

extern "C" int agal_refine_stats(const agal_ctx *c, long long *iter, int *n_refined, int *n_coarsened)
{
    if (!c) return AGAL_ERR_PARAM;
    if (iter) *iter = c->iter;
    if (n_refined) *n_refined = c->n_ref_last;
    if (n_coarsened) *n_coarsened = c->n_coarse_last;
    return AGAL_OK;
}

// ---------------------------------------------------------------------------
// Advance (solver_lbm_advance.cu:31-174).  Each sub-step of a level is one
// fused collide + boundary + stream kernel; each transfer between levels is
// one kernel.
static bool multi_level(const agal_ctx *c) { return c->max_levels > 1 && c->max_levels != c->L0 + 1; }

static int avg_mode(const agal_ctx *c)
{
    // solver_lbm_init.cu:94-97
    return (c->P.interp_order != AGAL_INTERP_LINEAR) ? AGAL_AVERAGE_BLOCK : AGAL_AVERAGE_INTERFACE;
}

// One sub-step of level L, with the MEA force passes around it when asked
// (before the stream from the current buffer, after it from the new one).
static int step_f(agal_ctx *c, int L, bool forces)
{
    int rc;
    if (forces && (rc = agal_launch_forces(c, L, 0))) return rc;
    if ((rc = agal_launch_step(c, L))) return rc;
    if (forces && (rc = agal_launch_forces(c, L, 1))) return rc;
    return AGAL_OK;
}

// S_Average inside the recursion: the refresh of level L+1 (LES macro mode),
// then the averaging.
static int average_rec(agal_ctx *c, int L, int var)
{
    const int rc = agal_les_refresh(c, L + 1);
    return rc ? rc : agal_launch_average(c, L, var);
}

// The interface interpolation of level L beside the step of level L: the
// interpolation reads F[cur[L]] and writes ghost cells of F[cur[L+1]], the
// step reads F[cur[L]] and writes level L's other buffer, so they are
// independent; the interpolation runs on the side stream, forked from and
// joined back into the case's stream (two branches of the captured graph).
static int interp_beside_step(agal_ctx *c, int L, bool forces)
{
    int rc;
    // The refresh of S_Interpolate (LES macro mode) precedes both branches:
    // the step's eddy viscosity reads the rows it writes.
    if ((rc = agal_les_refresh(c, L))) return rc;
    if (c->rec) {   // batch recording: the batch orders the launches itself
        if ((rc = agal_launch_interp(c, L, AGAL_INTERP_INTERFACE))) return rc;
        return step_f(c, L, forces);
    }
    AGAL_CUDA(c, cudaEventRecord(c->ev_fork, c->stream));
    AGAL_CUDA(c, cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    cudaStream_t main = c->stream;
    c->stream = c->side;
    rc = agal_launch_interp(c, L, AGAL_INTERP_INTERFACE);
    c->stream = main;
    if (rc) return rc;
    AGAL_CUDA(c, cudaEventRecord(c->ev_join, c->side));
    if ((rc = step_f(c, L, forces))) return rc;
    AGAL_CUDA(c, cudaStreamWaitEvent(c->stream, c->ev_join, 0));
    return AGAL_OK;
}

static int advance_rec(agal_ctx *c, int L)
{
    const int ML = c->max_levels;
    const bool mea = c->P.S_FORCE_TYPE == 0 && c->X_b;
    int rc;
    const bool cv = c->P.S_FORCE_TYPE == 1;
    if (!multi_level(c)) {                                  // :136-151
        if (cv && (rc = agal_launch_forces_cv(c, L, 0))) return rc;
        if ((rc = step_f(c, L, mea))) return rc;
        return cv ? agal_launch_forces_cv(c, L, 1) : AGAL_OK;
    }
    if (L == c->L0) {                                       // :39-70
        c->liter = 0;
        if (cv)
            for (int K = c->L0; K < ML; K++)
                if ((rc = agal_launch_forces_cv(c, K, 0))) return rc;
        if ((rc = interp_beside_step(c, L, false))) return rc;
        if ((rc = advance_rec(c, L + 1))) return rc;
        if ((rc = average_rec(c, L, avg_mode(c)))) return rc;
        if (cv) {
            // the control volume sees every level consistent: grid average,
            // interface interpolation, then the post-step pass
            for (int K = ML - 2; K >= c->L0; K--)
                if ((rc = average_rec(c, K, AGAL_AVERAGE_GRID))) return rc;
            for (int K = c->L0; K < ML - 1; K++)
                if ((rc = agal_les_refresh(c, K)) || (rc = agal_launch_interp(c, K, AGAL_INTERP_INTERFACE)))
                    return rc;
            for (int K = c->L0; K < ML; K++)
                if ((rc = agal_launch_forces_cv(c, K, 1))) return rc;
        }
        return AGAL_OK;
    }
    if (L < ML - 1) {                                                                       // :96-99
        if ((rc = interp_beside_step(c, L, false))) return rc;
    } else if ((rc = agal_launch_step(c, L))) {
        return rc;
    }
    if (L == ML - 1) c->liter++;
    // :114-126: the forces on the last finest sub-step of the coarse step.
    const bool f2 = mea && L == ML - 1 && c->liter == (1 << (ML - 1)) - 1;
    if (L < ML - 1) {                                                                       // :106-111
        if ((rc = advance_rec(c, L + 1))) return rc;
        if ((rc = average_rec(c, L, avg_mode(c)))) return rc;
        if ((rc = interp_beside_step(c, L, f2))) return rc;
    } else if ((rc = step_f(c, L, f2))) {
        return rc;
    }
    if (L == ML - 1) c->liter++;
    if (L < ML - 1) {                                                                       // :130-134
        if ((rc = advance_rec(c, L + 1))) return rc;
        if ((rc = average_rec(c, L, avg_mode(c)))) return rc;
    }
    return AGAL_OK;
}

namespace {
__global__ void k_sr_tick(unsigned *ctr) { *ctr += 1u; }
__global__ void k_sr_set(unsigned *ctr, unsigned v) { *ctr = v; }
}  // namespace

int agal_sr_tick(agal_ctx *c)
{
    // only the stochastic rounding of half-precision offsets reads the counter
    if (!((c->storage == AGAL_STORE_FP16 || c->storage == AGAL_STORE_BF16) &&
          c->P.half_rounding == AGAL_ROUND_STOCHASTIC))
        return AGAL_OK;
    if (c->rec) return agal_record_other(c, AGAL_OP_SR_TICK, 0, [](agal_ctx *x) { return agal_sr_tick(x); });
    k_sr_tick<<<1, 1, 0, c->stream>>>(c->d_sr);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

int agal_sr_set(agal_ctx *c, unsigned value)
{
    k_sr_set<<<1, 1, 0, c->stream>>>(c->d_sr, value);
    AGAL_CUDA(c, cudaGetLastError());
    return AGAL_OK;
}

extern "C" int agal_advance(agal_ctx *c, int L)
{
    if (!c || L < 0 || L >= c->max_levels) return AGAL_ERR_PARAM;
    c->sr_salt = 0;
    int rc = advance_rec(c, L);
    return rc ? rc : agal_sr_tick(c);
}

// One coarse step of M_Advance_Step (mesh_advance.cu:156-182): 2^N_LEVEL_START
// sub-steps from the starting level, then the tick of the rounding counter.
int agal_record_coarse_step(agal_ctx *c)
{
    const int mult = 1 << c->L0;
    c->sr_salt = 0;
    // On multi-level meshes the last launch of the coarse step is the
    // averaging of the starting level: it carries the tick (no launch of its
    // own), unless a control-volume pass follows or the batch records.
    const bool fold = multi_level(c) && c->P.S_FORCE_TYPE != 1 && !c->rec &&
                      (c->storage == AGAL_STORE_FP16 || c->storage == AGAL_STORE_BF16) &&
                      c->P.half_rounding == AGAL_ROUND_STOCHASTIC;
    c->tick_done = false;
    for (int j = 0; j < mult; j++) {
        c->tick_pending = fold && j == mult - 1;
        int rc = advance_rec(c, c->L0);
        c->tick_pending = false;
        if (rc) return rc;
    }
    if (c->tick_done) {
        c->tick_done = false;
        return AGAL_OK;
    }
    return agal_sr_tick(c);
}

// Capture `steps` coarse steps into *out: an existing executable is updated
// in place when the new graph has its topology (the usual case after a regrid:
// the same launches with new sizes and arguments), else replaced.
static int capture(agal_ctx *c, int steps, cudaGraphExec_t *out)
{
    std::vector<int> cur0 = c->cur;
    cudaGraph_t g = nullptr;
    AGAL_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = AGAL_OK;
    for (int i = 0; i < steps && rc == AGAL_OK; i++) rc = agal_record_coarse_step(c);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->cur = cur0;   // the capture only recorded the launches
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) return agal_cuda_check(c, e, "cudaStreamEndCapture");
    if (*out) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(*out, g, &info) == cudaSuccess) {
            cudaGraphDestroy(g);
            c->graph_updates++;
            return AGAL_OK;
        }
        cudaGetLastError();   // topology changed: rebuild
        cudaGraphExecDestroy(*out);
        *out = nullptr;
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return agal_cuda_check(c, e, "cudaGraphInstantiate");
    c->graph_builds++;
    return AGAL_OK;
}

extern "C" int agal_graph_stats(const agal_ctx *c, long long *builds, long long *updates)
{
    if (!c || !builds || !updates) return AGAL_ERR_PARAM;
    *builds = c->graph_builds;
    *updates = c->graph_updates;
    return AGAL_OK;
}

// Buffer parity after `steps` coarse steps.  Per coarse step the starting
// level L0 takes 2^L0 sub-steps and each finer level twice its parent's count
// (multi-level), or only L0 is stepped (single level); levels stepped an odd
// number of times flip.
void agal_advance_parity(agal_ctx *c, int steps)
{
    for (int L = 0; L < c->max_levels; L++) {
        long long k = 0;
        if (multi_level(c)) {
            if (L >= c->L0) k = (1LL << c->L0) << (L - c->L0);
        } else if (L == c->L0) {
            k = 1LL << c->L0;
        }
        if ((k * steps) & 1) c->cur[L] = 1 - c->cur[L];
    }
}

// n coarse steps of the M_AdvanceLoop body (mesh_advance.cu:421-463): a coarse
// step, then every P_REFINE steps the solution-based refinement.  use_graph
// replays a captured coarse step (captured once per mesh and buffer parity).
extern "C" int agal_advance_n(agal_ctx *c, int n, int use_graph)
{
    if (!c || n < 0) return AGAL_ERR_PARAM;
    int rc;
    if (!multi_level(c)) {
        if (!use_graph) {
            for (int i = 0; i < n; i++)
                if ((rc = agal_record_coarse_step(c))) return rc;
        } else if (n > 0) {
            if (!c->graph_exec || c->graph_steps != n || c->graph_cur_in != c->cur) {
                if ((rc = capture(c, n, &c->graph_exec))) return rc;
                c->graph_steps = n;
                c->graph_cur_in = c->cur;
            }
            AGAL_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
            agal_advance_parity(c, n);
        }
        c->iter += n;
        return AGAL_OK;
    }
    for (int s = 0; s < n; s++) {
        if (!use_graph) {
            if ((rc = agal_record_coarse_step(c))) return rc;
        } else {
            int k = (c->ml_graph[0] && c->ml_graph_cur[0] == c->cur)   ? 0
                    : (c->ml_graph[1] && c->ml_graph_cur[1] == c->cur) ? 1
                                                                       : -1;
            if (k < 0) {
                // a slot whose mesh changed (its executable is updated), else slot 1
                k = c->ml_graph_cur[0].empty() ? 0 : 1;
                if ((rc = capture(c, 1, &c->ml_graph[k]))) return rc;
                c->ml_graph_cur[k] = c->cur;
            }
            AGAL_CUDA(c, cudaGraphLaunch(c->ml_graph[k], c->stream));
            agal_advance_parity(c, 1);
        }
        const long long i = c->iter;
        if (c->P.P_REFINE > 0 && (i + 1) % c->P.P_REFINE == 0 && i > 0 && (rc = agal_refine_with_solution(c)))
            return rc;
        c->iter++;
    }
    return AGAL_OK;
}

// ---------------------------------------------------------------------------
// Array transfers.
extern "C" int agal_array_bytes(const agal_ctx *c, int which, size_t *bytes)
{
    if (!c || !bytes) return AGAL_ERR_PARAM;
    const size_t nmb = (size_t)c->nmb, nmc = (size_t)c->nmc;
    switch (which) {
    case AGAL_ARR_F: *bytes = sizeof(double) * (size_t)c->Q * nmc; break;
    case AGAL_ARR_MACROS: *bytes = sizeof(double) * (size_t)(c->dim + 1) * nmc; break;
    case AGAL_ARR_CELLS_ID_MASK: *bytes = sizeof(int) * nmc; break;
    case AGAL_ARR_CBLOCK_F_X: *bytes = sizeof(float) * (size_t)c->dim * nmb; break;
    case AGAL_ARR_CBLOCK_ID_MASK:
    case AGAL_ARR_CBLOCK_ID_ONB:
    case AGAL_ARR_CBLOCK_ID_REF:
    case AGAL_ARR_CBLOCK_LEVEL:
    case AGAL_ARR_GAP_SET: *bytes = sizeof(int) * nmb; break;
    case AGAL_ARR_CBLOCK_ID_NBR:
    case AGAL_ARR_CBLOCK_ID_NBR_CHILD: *bytes = sizeof(int) * (size_t)c->Qmax * nmb; break;
    case AGAL_ARR_ID_SET: *bytes = sizeof(int) * (size_t)c->max_levels * nmb; break;
    case AGAL_ARR_CBLOCK_ID_ONB_SOLID:
        if (!c->onb_solid) return AGAL_ERR_PARAM;
        *bytes = sizeof(int) * nmb;
        break;
    case AGAL_ARR_NU_SGS:
        if (!c->nu_sgs) return AGAL_ERR_PARAM;
        *bytes = sizeof(double) * nmc;
        break;
    case AGAL_ARR_CELLS_F_X_B:
        if (!c->X_b) return AGAL_ERR_PARAM;
        *bytes = sizeof(float) * 27 * (size_t)c->n_maxcells_b;
        break;
    case AGAL_ARR_CBLOCK_F_FF:
        if (!c->Ff) return AGAL_ERR_PARAM;
        *bytes = sizeof(double) * 6 * nmb;
        break;
    default: return AGAL_ERR_PARAM;
    }
    return AGAL_OK;
}

static void *int_array(agal_ctx *c, int which)
{
    switch (which) {
    case AGAL_ARR_CELLS_ID_MASK: return c->cells_ID_mask;
    case AGAL_ARR_CBLOCK_F_X: return c->cblock_f_X;
    case AGAL_ARR_CBLOCK_ID_MASK: return c->cblock_ID_mask;
    case AGAL_ARR_CBLOCK_ID_NBR: return c->cblock_ID_nbr;
    case AGAL_ARR_CBLOCK_ID_NBR_CHILD: return c->cblock_ID_nbr_child;
    case AGAL_ARR_CBLOCK_ID_ONB: return c->cblock_ID_onb;
    case AGAL_ARR_CBLOCK_ID_REF: return c->cblock_ID_ref;
    case AGAL_ARR_CBLOCK_LEVEL: return c->cblock_level;
    case AGAL_ARR_ID_SET: return c->id_set;
    case AGAL_ARR_GAP_SET: return c->gap_set;
    case AGAL_ARR_CBLOCK_ID_ONB_SOLID: return c->onb_solid;
    case AGAL_ARR_CELLS_F_X_B: return c->X_b;
    default: return nullptr;
    }
}

// Populations of blocks [0, nb) in the reference's slot-major layout
// (out[s][b * MC + cell], absolute values), each block from its level's
// current buffer; and the inverse, into both buffers.  Only the prefix of the
// pool crosses PCIe (restart files hold blocks below id_max).
int agal_read_blocks_F(agal_ctx *c, int nb, double *out)
{
    if (nb <= 0) return AGAL_OK;
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    return agal_f_to_host(c, nb, (long long)nb * c->MC, out);
}

int agal_write_blocks_F(agal_ctx *c, int nb, const double *in)
{
    if (nb <= 0) return AGAL_OK;
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    int rc = agal_f_from_host(c, nb, (long long)nb * c->MC, in);
    agal_drop_graphs(c);
    return rc;
}

extern "C" int agal_dump(agal_ctx *c, int which, void *host_buf, size_t bytes)
{
    size_t need = 0;
    int rc = agal_array_bytes(c, which, &need);
    if (rc) return rc;
    if (!host_buf || bytes != need) return agal_set_err(c, AGAL_ERR_PARAM, "dump size mismatch");
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (which == AGAL_ARR_CBLOCK_F_FF || which == AGAL_ARR_NU_SGS) {
        // compute-type arrays, widened to FP64
        double *o = static_cast<double *>(host_buf);
        const void *src = which == AGAL_ARR_NU_SGS ? c->nu_sgs : c->Ff;
        const size_t n = need / sizeof(double);
        if (c->storage == AGAL_STORE_FP64) {
            AGAL_CUDA(c, cudaMemcpy(o, src, n * 8, cudaMemcpyDeviceToHost));
        } else {
            std::vector<float> t(n);
            AGAL_CUDA(c, cudaMemcpy(t.data(), src, n * 4, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; i++) o[i] = t[i];
        }
        return AGAL_OK;
    }
    if (which == AGAL_ARR_F) {
        // Device layout F[b][s][c] -> reference layout cells_f_F[s][b*MC + c],
        // converted on the device.
        return agal_f_to_host(c, c->nmb, c->nmc, static_cast<double *>(host_buf));
    }
    if (which == AGAL_ARR_MACROS) {
        const size_t n = (size_t)(c->dim + 1) * c->nmc;
        double *o = static_cast<double *>(host_buf);
        if (c->storage == AGAL_STORE_FP64) {
            AGAL_CUDA(c, cudaMemcpy(o, c->macro, n * 8, cudaMemcpyDeviceToHost));
        } else {
            std::vector<float> t(n);
            AGAL_CUDA(c, cudaMemcpy(t.data(), c->macro, n * 4, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; i++) o[i] = t[i];
        }
        return AGAL_OK;
    }
    AGAL_CUDA(c, cudaMemcpy(host_buf, int_array(c, which), need, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

extern "C" int agal_load(agal_ctx *c, int which, const void *host_buf, size_t bytes)
{
    size_t need = 0;
    int rc = agal_array_bytes(c, which, &need);
    if (rc) return rc;
    if (!host_buf || bytes != need) return agal_set_err(c, AGAL_ERR_PARAM, "load size mismatch");
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (which == AGAL_ARR_F) {
        // The same values go to both buffers, converted on the device.
        return agal_f_from_host(c, c->nmb, c->nmc, static_cast<const double *>(host_buf));
    }
    if (which == AGAL_ARR_MACROS) return agal_set_err(c, AGAL_ERR_PARAM, "macros are derived, not loaded");
    if (which == AGAL_ARR_CBLOCK_F_FF) return agal_set_err(c, AGAL_ERR_PARAM, "force partials are derived, not loaded");
    if (which == AGAL_ARR_NU_SGS) return agal_set_err(c, AGAL_ERR_PARAM, "eddy viscosity is derived, not loaded");
    AGAL_CUDA(c, cudaMemcpy(int_array(c, which), host_buf, need, cudaMemcpyHostToDevice));
    if (which == AGAL_ARR_CELLS_ID_MASK) {
        // Geometry present when any cell is solid.
        std::vector<int> cm(c->nmc);
        std::memcpy(cm.data(), host_buf, need);
        c->geometry_init = std::any_of(cm.begin(), cm.end(), [](int v) { return v == CELL_SOLID; }) ? 1 : 0;
    }
    return agal_build_meta(c);
}
