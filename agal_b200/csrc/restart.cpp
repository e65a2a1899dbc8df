// Checkpoint / restart in the reference's restart.bin format
// (Mesh::M_Restart, mesh_restart.cu:45-225), so that checkpoints written by
// the reference can seed runs of this library and the other way round.
//
// Layout (native endianness, as the reference writes it):
//   int  n_maxcblocks
//   int  n_ids[MAX_LEVELS + 1]
//   int  n_gaps
//   int  id_max[MAX_LEVELS + 1]
//   int  cblocks_id_max = id_max[MAX_LEVELS]
//   long cells_id_max   = cblocks_id_max * M_CBLOCK          (8 bytes)
//   int  n_ids_probed
//   int  iter
//   int  id_set[L][0 .. n_ids[L])            for each level L
//   int  gap_set[0 .. n_gaps)
//   int  cells_ID_mask[0 .. cells_id_max)
//   R    cblock_f_X[d][0 .. cblocks_id_max)  for each dimension d
//   int  cblock_ID_mask[0 .. cblocks_id_max)
//   int  cblock_ID_nbr[p][..], cblock_ID_nbr_child[p][..]   interleaved per p < N_Q_max
//   int  cblock_ID_onb, cblock_ID_ref, cblock_level            [0 .. cblocks_id_max)
//   R    cells_f_F[p][0 .. cells_id_max)      p < Q + N_DIM + 1: the populations
//                                            (post-stream slots), then the macro
//                                            rows rho, u, v, (w) (the Mesh is
//                                            built with N_U = Q + N_DIM + 1 rows)
//   R    cells_f_U_probed_tn[d][n_ids_probed * M_CBLOCK]        d < N_DIM
//   R    cells_f_U_mean[d][n_ids[0] * M_CBLOCK]                 d < N_DIM + 1
// with R the reference's ufloat_t: float, or double for FP64 storage.  The
// macro rows are written as rho and u of the saved populations and skipped on
// load (derived data).  This library keeps no velocity probes or running
// means: it writes the reference's probe count (every N_PROBE_DENSITY-th root
// block per axis, mesh_init.cu:388-392) with zero velocities and a zero mean,
// and skips both on load.  The geometry arrays (wall slots, link lengths) are
// not part of the format, as in the reference.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"
#include "lattice.cuh"

namespace {

struct File {
    FILE *f = nullptr;
    explicit File(FILE *p) : f(p) {}
    ~File()
    {
        if (f) fclose(f);
    }
};

template <typename X>
bool put(FILE *f, const X *p, size_t n)
{
    return n == 0 || fwrite(p, sizeof(X), n, f) == n;
}

template <typename X>
bool get(FILE *f, X *p, size_t n)
{
    return n == 0 || fread(p, sizeof(X), n, f) == n;
}

// Prefix [0, n) of row r of a device array with rows of nmb elements.
template <typename X>
int d2h(agal_ctx *c, X *host, const X *dev, int r, long long n)
{
    if (n > 0) AGAL_CUDA(c, cudaMemcpy(host, dev + (size_t)r * c->nmb, sizeof(X) * (size_t)n, cudaMemcpyDeviceToHost));
    return AGAL_OK;
}

template <typename X>
int h2d(agal_ctx *c, X *dev, const X *host, int r, long long n)
{
    if (n > 0) AGAL_CUDA(c, cudaMemcpy(dev + (size_t)r * c->nmb, host, sizeof(X) * (size_t)n, cudaMemcpyHostToDevice));
    return AGAL_OK;
}

// The block arrays of the format, prefix [0, cb) of every row.
struct Blocks {
    std::vector<int> cmask, bmask, nbr, child, onb, ref, lev;   // nbr / child: [p][cb]
    std::vector<float> fx;                                      // [d][cb]
};

int read_blocks(agal_ctx *c, int cb, Blocks &k)
{
    const long long cells = (long long)cb * c->MC;
    k.cmask.resize(cells);
    k.bmask.resize(cb);
    k.onb.resize(cb);
    k.ref.resize(cb);
    k.lev.resize(cb);
    k.nbr.resize((size_t)c->Qmax * cb);
    k.child.resize((size_t)c->Qmax * cb);
    k.fx.resize((size_t)c->dim * cb);
    int rc;
    if (cells > 0) AGAL_CUDA(c, cudaMemcpy(k.cmask.data(), c->cells_ID_mask, sizeof(int) * cells, cudaMemcpyDeviceToHost));
    if ((rc = d2h(c, k.bmask.data(), c->cblock_ID_mask, 0, cb)) || (rc = d2h(c, k.onb.data(), c->cblock_ID_onb, 0, cb)) ||
        (rc = d2h(c, k.ref.data(), c->cblock_ID_ref, 0, cb)) || (rc = d2h(c, k.lev.data(), c->cblock_level, 0, cb)))
        return rc;
    for (int p = 0; p < c->Qmax; p++)
        if ((rc = d2h(c, k.nbr.data() + (size_t)p * cb, c->cblock_ID_nbr, p, cb)) ||
            (rc = d2h(c, k.child.data() + (size_t)p * cb, c->cblock_ID_nbr_child, p, cb)))
            return rc;
    for (int d = 0; d < c->dim; d++)
        if ((rc = d2h(c, k.fx.data() + (size_t)d * cb, c->cblock_f_X, d, cb))) return rc;
    return AGAL_OK;
}

int write_blocks(agal_ctx *c, int cb, const Blocks &k)
{
    const long long cells = (long long)cb * c->MC;
    int rc;
    if (cells > 0) AGAL_CUDA(c, cudaMemcpy(c->cells_ID_mask, k.cmask.data(), sizeof(int) * cells, cudaMemcpyHostToDevice));
    if ((rc = h2d(c, c->cblock_ID_mask, k.bmask.data(), 0, cb)) || (rc = h2d(c, c->cblock_ID_onb, k.onb.data(), 0, cb)) ||
        (rc = h2d(c, c->cblock_ID_ref, k.ref.data(), 0, cb)) || (rc = h2d(c, c->cblock_level, k.lev.data(), 0, cb)))
        return rc;
    for (int p = 0; p < c->Qmax; p++)
        if ((rc = h2d(c, c->cblock_ID_nbr, k.nbr.data() + (size_t)p * cb, p, cb)) ||
            (rc = h2d(c, c->cblock_ID_nbr_child, k.child.data() + (size_t)p * cb, p, cb)))
            return rc;
    for (int d = 0; d < c->dim; d++)
        if ((rc = h2d(c, c->cblock_f_X, k.fx.data() + (size_t)d * cb, d, cb))) return rc;
    return AGAL_OK;
}

template <typename R>
int save_as(agal_ctx *c, FILE *f, int iter)
{
    const int ML = c->max_levels, MC = c->MC, dim = c->dim;
    const int cb = c->id_max[ML];
    const long cells = (long)cb * MC;
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    Blocks k;
    std::vector<std::vector<int>> ids(ML);
    std::vector<int> gap(std::max(c->n_gaps, 1));
    std::vector<double> F((size_t)c->Q * cells + 1);
    int rc;
    for (int L = 0; L < ML; L++) {
        ids[L].resize(std::max(c->n_ids[L], 1));
        if ((rc = d2h(c, ids[L].data(), c->id_set, L, c->n_ids[L]))) return rc;
    }
    if ((rc = d2h(c, gap.data(), c->gap_set, 0, c->n_gaps)) || (rc = read_blocks(c, cb, k)) ||
        (rc = agal_read_blocks_F(c, cb, F.data())))
        return rc;
    // The reference's probe count: root blocks whose padded grid indices
    // i-1, j-1 (and k-1 in 3D) are multiples of N_PROBE_DENSITY.
    const int D = c->P.N_PROBE_DENSITY > 0 ? c->P.N_PROBE_DENSITY : 1;
    const int nbx = c->Nx / 4, nby = c->Ny / 4, nbz = dim == 3 ? c->Nz / 4 : 1;
    const int probed = ((nbx + D - 1) / D) * ((nby + D - 1) / D) * (dim == 3 ? (nbz + D - 1) / D : 1);
    const int nmb_i = (int)c->nmb;
    bool ok = put(f, &nmb_i, 1) && put(f, c->n_ids.data(), ML + 1) && put(f, &c->n_gaps, 1) &&
              put(f, c->id_max.data(), ML + 1) && put(f, &cb, 1) && put(f, &cells, 1) && put(f, &probed, 1) &&
              put(f, &iter, 1);
    for (int L = 0; L < ML && ok; L++) ok = put(f, ids[L].data(), c->n_ids[L]);
    ok = ok && put(f, gap.data(), c->n_gaps) && put(f, k.cmask.data(), cells);
    std::vector<R> buf((size_t)std::max<long>(cells, cb) + 1);
    for (int d = 0; d < dim && ok; d++) {
        for (int i = 0; i < cb; i++) buf[i] = (R)k.fx[(size_t)d * cb + i];
        ok = put(f, buf.data(), cb);
    }
    ok = ok && put(f, k.bmask.data(), cb);
    for (int p = 0; p < c->Qmax && ok; p++)
        ok = put(f, k.nbr.data() + (size_t)p * cb, cb) && put(f, k.child.data() + (size_t)p * cb, cb);
    ok = ok && put(f, k.onb.data(), cb) && put(f, k.ref.data(), cb) && put(f, k.lev.data(), cb);
    for (int p = 0; p < c->Q && ok; p++) {
        for (long i = 0; i < cells; i++) buf[i] = (R)F[(size_t)p * cells + i];
        ok = put(f, buf.data(), cells);
    }
    // macro rows: rho, u, v, (w) of the saved populations (slot s holds f_pb(s))
    for (int m = 0; m < dim + 1 && ok; m++) {
        for (long i = 0; i < cells; i++) {
            double r = 0, j = 0;
            for (int sl = 0; sl < c->Q; sl++) {
                const double fv = F[(size_t)sl * cells + i];
                r += fv;
                if (m > 0) j += agal::lat_c(dim, m - 1, agal::lat_pb(dim, sl)) * fv;
            }
            buf[i] = (R)(m == 0 ? r : j / r);
        }
        ok = put(f, buf.data(), cells);
    }
    // zero probe velocities and running mean of level 0
    const std::vector<R> zp((size_t)probed * MC, R(0)), zm((size_t)c->n_ids[0] * MC, R(0));
    for (int d = 0; d < dim && ok; d++) ok = put(f, zp.data(), zp.size());
    for (int d = 0; d < dim + 1 && ok; d++) ok = put(f, zm.data(), zm.size());
    if (!ok) return agal_set_err(c, AGAL_ERR_IO, "restart: write failed");
    return AGAL_OK;
}

template <typename R>
int load_as(agal_ctx *c, FILE *f, int *iter)
{
    const int ML = c->max_levels, MC = c->MC, dim = c->dim;
    const long long nmb = c->nmb;
    int nmb_old = 0, n_gaps = 0, cb = 0, probed = 0, it = 0;
    long cells = 0;
    std::vector<int> n_ids(ML + 1), id_max(ML + 1);
    if (!(get(f, &nmb_old, 1) && get(f, n_ids.data(), ML + 1) && get(f, &n_gaps, 1) && get(f, id_max.data(), ML + 1) &&
          get(f, &cb, 1) && get(f, &cells, 1) && get(f, &probed, 1) && get(f, &it, 1)))
        return agal_set_err(c, AGAL_ERR_IO, "restart: short header");
    if (nmb_old <= 0 || cb < 0 || probed < 0 || n_gaps < 0 || n_gaps > nmb_old || cells != (long)cb * MC)
        return agal_set_err(c, AGAL_ERR_IO, "restart: inconsistent header");
    for (int L = 0; L <= ML; L++)
        if (n_ids[L] < 0 || n_ids[L] > nmb_old || id_max[L] < 0 || id_max[L] > nmb_old)
            return agal_set_err(c, AGAL_ERR_IO, "restart: inconsistent counts");
    if (id_max[ML] > nmb || cb > nmb) return agal_set_err(c, AGAL_ERR_OOM, "Insufficient memory allocation...");
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    bool ok = true;
    std::vector<std::vector<int>> ids(ML);
    for (int L = 0; L < ML && ok; L++) {
        ids[L].resize(std::max(n_ids[L], 1));
        ok = get(f, ids[L].data(), n_ids[L]);
    }
    std::vector<int> gaps_old(std::max(n_gaps, 1));
    ok = ok && get(f, gaps_old.data(), n_gaps);
    Blocks k;
    k.cmask.resize(cells);
    k.bmask.resize(cb);
    k.onb.resize(cb);
    k.ref.resize(cb);
    k.lev.resize(cb);
    k.nbr.resize((size_t)c->Qmax * cb);
    k.child.resize((size_t)c->Qmax * cb);
    k.fx.resize((size_t)dim * cb);
    ok = ok && get(f, k.cmask.data(), cells);
    std::vector<R> buf((size_t)std::max<long>(cells, cb) + 1);
    for (int d = 0; d < dim && ok; d++) {
        ok = get(f, buf.data(), cb);
        for (int i = 0; i < cb && ok; i++) k.fx[(size_t)d * cb + i] = (float)buf[i];
    }
    ok = ok && get(f, k.bmask.data(), cb);
    for (int p = 0; p < c->Qmax && ok; p++)
        ok = get(f, k.nbr.data() + (size_t)p * cb, cb) && get(f, k.child.data() + (size_t)p * cb, cb);
    ok = ok && get(f, k.onb.data(), cb) && get(f, k.ref.data(), cb) && get(f, k.lev.data(), cb);
    std::vector<double> F((size_t)c->Q * cells + 1);
    for (int p = 0; p < c->Q && ok; p++) {
        ok = get(f, buf.data(), cells);
        for (long i = 0; i < cells && ok; i++) F[(size_t)p * cells + i] = (double)buf[i];
    }
    for (int m = 0; m < dim + 1 && ok; m++) ok = get(f, buf.data(), cells);   // macro rows: derived
    if (!ok) return agal_set_err(c, AGAL_ERR_IO, "restart: short data");
    // The gap stack moved to this pool's size (mesh_restart.cu:174-179): a
    // larger pool keeps the fresh pool's top IDs below the old stack, a
    // smaller one drops the bottom of the old stack (its highest IDs).
    const long long shift = nmb - nmb_old;
    const long long n_gaps_new = n_gaps + shift;
    if (n_gaps_new < 0) return agal_set_err(c, AGAL_ERR_OOM, "restart: the gap stack does not fit the block pool");
    std::vector<int> gap((size_t)std::max<long long>(n_gaps_new, 1));
    if (shift >= 0) {
        for (long long x = 0; x < shift; x++) gap[x] = (int)(nmb - 1 - x);
        std::memcpy(gap.data() + shift, gaps_old.data(), sizeof(int) * (size_t)n_gaps);
    } else {
        std::memcpy(gap.data(), gaps_old.data() + (-shift), sizeof(int) * (size_t)n_gaps_new);
    }
    int rc;
    for (int L = 0; L < ML; L++)
        if ((rc = h2d(c, c->id_set, ids[L].data(), L, n_ids[L]))) return rc;
    if ((rc = h2d(c, c->gap_set, gap.data(), 0, n_gaps_new)) || (rc = write_blocks(c, cb, k)) ||
        (rc = agal_write_blocks_F(c, cb, F.data())))
        return rc;
    if ((rc = agal_set_counts(c, n_ids.data(), id_max.data(), (int)n_gaps_new))) return rc;
    // The file holds the loop index of the last step taken; the loop resumes
    // at the next one (M_Advance_LoadRestartFile, mesh_advance.cu:124-134).
    c->iter = (long long)it + 1;
    if (iter) *iter = it;
    // The stochastic-rounding counter of a run advanced by agal_advance_n is
    // its coarse-step count: the loaded state continues as the saved run.
    return agal_sr_set(c, (unsigned)c->iter);
}

}  // namespace

extern "C" int agal_restart_save(agal_ctx *c, const char *path, int iter)
{
    if (!c || !path) return AGAL_ERR_PARAM;
    File f(fopen(path, "wb"));
    if (!f.f) return agal_set_err(c, AGAL_ERR_IO, std::string("restart: cannot open ") + path);
    return c->storage == AGAL_STORE_FP64 ? save_as<double>(c, f.f, iter) : save_as<float>(c, f.f, iter);
}

extern "C" int agal_restart_load(agal_ctx *c, const char *path, int *iter)
{
    if (!c || !path) return AGAL_ERR_PARAM;
    File f(fopen(path, "rb"));
    if (!f.f) return agal_set_err(c, AGAL_ERR_IO, std::string("restart: cannot open ") + path);
    return c->storage == AGAL_STORE_FP64 ? load_as<double>(c, f.f, iter) : load_as<float>(c, f.f, iter);
}
