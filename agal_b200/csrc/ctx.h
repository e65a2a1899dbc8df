// Private state of one simulation case (the object behind agal_ctx*).
//
// Device layout in HBM, per case:
//   F[2]            two population buffers, each Q slots x n_maxcells of the
//                   storage type (float, double, or half/bf16 weight offsets),
//                   slot s of a cell holding f_{pb(s)} (the reference's
//                   post-stream convention, solver_lbm_kernels.cu:67/251).
//                   Level L's current buffer is cur[L]; a step of level L
//                   reads F[cur[L]] and writes F[1-cur[L]].
//   macro           (dim+1) x n_maxcells float/double, written on demand.
//   block arrays    structure-of-arrays over n_maxcblocks exactly as
//                   inc/mesh.h:366-459 (neighbours [Qmax][n_maxcblocks], ...).
//   id_set          [MAX_LEVELS][n_maxcblocks], sorted block IDs per level.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "../../include/agal_b200.h"

// One CSR set of face bins on the device (Bins::binned_face_ids_{n,N,},
// geometry_bins.h:66-86): n = faces per bin, N = start, ids = face IDs.
struct agal_bins_d {
    int density = 0, n_bins = 0;
    float sx = 0.f, sy = 0.f, sz = 0.f;   // bins per unit length along x, y, z
    long long n_entries = 0;
    int *n = nullptr, *N = nullptr, *ids = nullptr;
};

struct agal_ctx {
    agal_params P{};
    int dim = 2, Q = 9, Qmax = 9, MC = 16, NCH = 4;
    int storage = AGAL_STORE_FP32;
    size_t esize = 4;                  // bytes per stored population
    int64_t nmb = 0, nmc = 0;          // n_maxcblocks, n_maxcells
    int max_levels = 1, L0 = 0;
    int Nx = 0, Ny = 0, Nz = 1;
    float dx = 0.f, dx_cblock = 0.f;
    std::vector<double> dxf;           // dxf_vec (rounded to the compute type)
    std::vector<double> tau;           // tau_vec (rounded to the compute type)
    // host mirrors (authoritative for launch sizes, as in the reference)
    std::vector<int> n_ids, id_max;
    int n_gaps = 0;
    int geometry_init = 0;
    // device arrays
    void *F[2] = {nullptr, nullptr};
    std::vector<int> cur;              // current population buffer per level
    void *macro = nullptr;
    int *cells_ID_mask = nullptr;
    float *cblock_f_X = nullptr;
    int *cblock_ID_mask = nullptr;
    int *cblock_ID_nbr = nullptr;
    int *cblock_ID_nbr_child = nullptr;
    int *cblock_ID_onb = nullptr;
    int *cblock_ID_ref = nullptr;
    int *cblock_level = nullptr;
    int *id_set = nullptr;
    int *gap_set = nullptr;
    double *red = nullptr;             // reduction scratch for FP64 sums
    int red_len = 0;
    double *red_out = nullptr;
    cudaStream_t stream = nullptr;
    // Side stream for the level interpolations that run beside the step of
    // the same level (forked from and joined back into `stream`).
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int device = 0;
    // graph of n coarse steps (agal_advance_n)
    cudaGraphExec_t graph_exec = nullptr;
    // multi-level: graphs of one coarse step, keyed on cur[] at entry (the
    // coarse level's parity alternates, the finer levels' returns)
    cudaGraphExec_t ml_graph[2] = {nullptr, nullptr};
    std::vector<int> ml_graph_cur[2];
    int graph_steps = 0;
    std::vector<int> graph_cur_in;     // cur[] the graph was captured with
    long long graph_builds = 0, graph_updates = 0;   // instantiations / in-place updates
    int liter = 0;                     // global_Liter (solver_lbm_advance.cu:6)
    int step_cpt = 1;                  // step kernel variant, 1..AGAL_STEP_VARIANTS (autotuned)
    int *d_status = nullptr;           // device status word: AGAL_ERR_TIMEOUT from bounded waits
    // Stochastic rounding of half-precision offsets: the coarse-step counter
    // in device memory (d_status[2]; one tick per coarse step, equal to iter
    // under agal_advance_n and restored by restart loads) and the ordinal of
    // the next step launch within the coarse step being recorded.
    unsigned *d_sr = nullptr;
    int sr_salt = 0;
    // The tick folded into the coarse step's last averaging launch (its last
    // CTA increments the counter, d_status[3] its CTA ticket): pending while
    // the last sub-step of a multi-level coarse step is recorded, done once
    // that launch carries it.
    bool tick_pending = false, tick_done = false;
    int *meta = nullptr;               // per-block step metadata rows (step_common.cuh Meta<DIM>)
    int *blk_solid = nullptr;          // [nmb] 1 = the block holds a solid cell (geometry cases)
    int *tiles = nullptr;              // root-level tile table of the 2D tile step (step_tile.cu)
    int n_tiles = 0;                   // 0 = the tile step is not available
    int n_ptiles = 0;                  // push tiles of the root level (step_ptile.cu); 0 = not available
    // Batch recording (batch.cu): while set, the launchers of a coarse step
    // append what they would launch to this list instead of launching.
    struct agal_oplist *rec = nullptr;
    void *xfer = nullptr;              // 64 MiB FP64 staging of the population dumps and loads (xfer.cu)
    int *fix_count = nullptr;          // stream-guard fix-ups of the running step (k_stream_fixup)
    long long *fix_list = nullptr;
    int fix_cap = 0;
    // refine/coarsen pass scratch (multi-level cases only), one allocation:
    int *amr = nullptr;
    int *amr_emap = nullptr;           // efficient map (mesh_amr.cu c_tmp_8), -1 = absent
    int *amr_first = nullptr;          // first-child ID of each marked block, -1 = none
    int *amr_a = nullptr, *amr_b = nullptr, *amr_snap = nullptr;   // compaction / snapshot buffers
    int *amr_parts = nullptr;          // per-CTA partial counts of the compactions
    int *amr_small = nullptr;          // small counters read back by the host
    int *h_small = nullptr;            // [AGAL_AMR_SMALL] pinned host copy of them (a readback per pass stage)
    void *crit = nullptr;              // percentile criterion: block values, histograms, selection state
    long long iter = 0;                // coarse steps taken (M_AdvanceLoop counter i)
    int n_ref_last = 0, n_coarse_last = 0;   // marks acted on by the last refinement pass
    // Geometry (geometry.cu): faces, bins, solid-boundary state, MEA partials.
    int n_faces = 0;
    float *faces = nullptr;            // [9][n_faces] v1x v1y v1z v2x .. v3z
    int n_bin_levels = 0, bin_level_md = -1;
    agal_bins_d bins[16], bins_md;
    long long n_solida = 0, n_maxcells_b = 0;
    int n_solidb = 0;
    int *onb_solid = nullptr;          // [nmb] wall-block slot (cblock_ID_onb_solid), -1 = none
    float *X_b = nullptr;              // [27][n_maxcells_b] link lengths (cells_f_X_b), -1 = none
    int *vox_tmp = nullptr;            // [nmb] near-wall marking scratch (c_tmp_1), -1 at rest
    unsigned long long *bnd_bits = nullptr;   // [nmb] boundary-cell flags of Voxelize_S2
    void *nu_sgs = nullptr;            // [nmb][MC] LES eddy viscosity (S_LES > 0), compute type
    void *Ff = nullptr;                // [6][nmb] MEA partials (cblock_f_Ff), compute type
    int *geo_small = nullptr, *geo_parts = nullptr;   // counters / compaction partials
    // Wall blocks (onb == 1 and a wall slot) per level for the interpolated
    // bounce-back and the forces: wall_ids[wall_off[L] .. + wall_n[L]).
    int *wall_ids = nullptr;
    std::vector<int> wall_off, wall_n;
    // Interface parents per level (block mask INTERFACE with children), the
    // only blocks the per-step interpolation and averaging touch:
    // iface_ids[iface_off[L] .. + iface_n[L]), in ID-set order.
    int *iface_ids = nullptr;
    std::vector<int> iface_off, iface_n;
    // Learned refinement predictor attached to this case (learn.cu).
    struct agal_learn *learner = nullptr;
    int learn_mode = 0;                // 1 = collect labelled snapshots, 2 = predict (judged)
    std::string err;
};

// Stream-guard fix-ups (refused swaps) one step of a context can hold:
// n_maxcells / 4, at least AGAL_FIX_CAP_MIN (every wall link of a geometry is
// one refused swap per step).
#define AGAL_FIX_CAP_MIN 65536
// Step launches over at most this many blocks apply their fix-ups in the
// kernel's last CTA instead of a separate launch.
#define AGAL_FUSED_FIXUP_BLOCKS 8192

// Step kernel variants: 1 and 2 cells per thread (one-shot grid), 3 the
// TMA-staged persistent pipeline, 4 one x-row of four cells per thread with
// vector loads and stores (step_row.cu), 5 the root-level tile step of 2D
// cases (step_tile.cu; other levels and cases run variant 4 in its place).
#define AGAL_STEP_VARIANTS 6

// Error helpers shared by the translation units.
int agal_set_err(agal_ctx *c, int code, const std::string &msg);
int agal_cuda_check(agal_ctx *c, cudaError_t e, const char *what);
#define AGAL_CUDA(c, call)                                             \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) return agal_cuda_check((c), e_, #call); \
    } while (0)

// Kernel launchers (step_kernels.cu).
int agal_launch_set_ic(agal_ctx *c, int L);
int agal_launch_step(agal_ctx *c, int L);
int agal_launch_tune(agal_ctx *c, int L, int reps, float *ms);
int agal_prepare_step(agal_ctx *c);
int agal_build_meta(agal_ctx *c);   // after any change of the block arrays
int agal_build_tiles(agal_ctx *c);  // root-level tile table (agal_build_meta calls it)
int agal_count_ptiles(const agal_ctx *c);   // root-level push tiles, 0 if not available
int agal_launch_refresh(agal_ctx *c, int L);

// Multi-level LES: the eddy viscosity reads the macro rows as the reference
// leaves them -- refreshed by every interpolation (level L) and averaging
// (level L+1) and by the initial condition, rewritten by every collide from
// its pre-collision populations -- instead of the current populations
// (S_Collide refreshes first only when MAX_LEVELS is 1,
// solver_lbm_kernels.cu:467-471).
inline bool agal_les_macros(const agal_ctx *c) { return c->nu_sgs && c->max_levels > 1; }
// The refresh a transfer performs first (level L), in that mode only.
int agal_les_refresh(agal_ctx *c, int L);
int agal_launch_mass(agal_ctx *c, double *out);
// Enqueue the FP64 sums and their copy into host memory (pinned for a truly
// asynchronous copy); the values are valid once the stream has reached it.
int agal_launch_mass_async(agal_ctx *c, double *host_out);
// Multi-level path (amr_kernels.cu, amr_pass.cu).
int agal_launch_interp(agal_ctx *c, int L, int var);
int agal_launch_average(agal_ctx *c, int L, int var);
int agal_launch_criterion(agal_ctx *c);
// Decisions of the percentile rule for listed blocks (k_pct_decide); select = 1
// first computes the block values and quantiles on the current macros, 0
// reuses those of the last criterion launch.
int agal_percentile_decisions(agal_ctx *c, int select, const int *ids, const int *lvl0, int n, float *Y, float *Wt);
int agal_refine_pass(agal_ctx *c);          // Mesh::M_RefineAndCoarsenBlocks
int agal_mark_level(agal_ctx *c, int L, int uniform);
int agal_freeze_refined(agal_ctx *c, int thaw = 0);
int agal_build_iface_lists(agal_ctx *c);    // after any mesh change (multi-level cases)
size_t agal_amr_scratch_ints(int64_t nmb);  // the last AGAL_AMR_SMALL ints are amr_small
#define AGAL_AMR_SMALL 192
// After any change of the mesh or launch shapes: the captured graphs no
// longer match; their executables are kept and updated in place from the next
// capture (cudaGraphExecUpdate, same topology), else rebuilt.
void agal_drop_graphs(agal_ctx *c);
void agal_free_graphs(agal_ctx *c);          // destroys them (context release)
// One coarse step's launches on the context's stream (flips cur[] as it
// records), and the buffer-parity bookkeeping of replaying `steps` of them.
int agal_record_coarse_step(agal_ctx *c);
// Advance the device coarse-step counter of the stochastic rounding by one
// (stream-ordered), or set it.
int agal_sr_tick(agal_ctx *c);
int agal_sr_set(agal_ctx *c, unsigned value);
void agal_advance_parity(agal_ctx *c, int steps);
// Populations of the first nb blocks in the reference's slot-major layout
// (restart I/O without copying the whole pool).
int agal_read_blocks_F(agal_ctx *c, int nb, double *out);
int agal_write_blocks_F(agal_ctx *c, int nb, const double *in);
// Device-side conversions behind them (xfer.cu): blocks [0, nb) to / from
// host[s * pitch + b * M_CBLOCK + c] (FP64, absolute values).
int agal_f_to_host(agal_ctx *c, long long nb, long long pitch, double *host);
int agal_f_from_host(agal_ctx *c, long long nb, long long pitch, const double *host);
// Geometry (geometry.cu, wall_kernels.cu).
void agal_geometry_release(agal_ctx *c);
int agal_build_wall_lists(agal_ctx *c);     // after the mesh or the wall slots change
int agal_wall_active(const agal_ctx *c);    // interpolated bounce-back in force
int agal_launch_wall_step(agal_ctx *c, int L, const void *fin, void *fout);
int agal_launch_forces(agal_ctx *c, int L, int post);
int agal_launch_forces_cv(agal_ctx *c, int L, int post);   // S_FORCE_TYPE 1
// Batch recording (batch.cu): a fused step (its StepArgs as bytes, the
// batched-kernel key of agal_step_batch_key, the level's block count and the
// buffers of the wall step that follows it), or any other launch as a
// closure that issues it on the context's stream.
int agal_record_step(agal_ctx *c, int L, const void *args, size_t bytes, int key, int n_blocks, const void *fin,
                     void *fout);
int agal_record_other(agal_ctx *c, int tag, int L, std::function<int(agal_ctx *)> fn);
// A transfer (interpolation or averaging): its argument structure, the key of
// its batched kernel and its block count.
int agal_record_args(agal_ctx *c, int kind, int L, const void *args, size_t bytes, int key, int n_items);
int agal_transfer_batch_key(const agal_ctx *c, bool cubic);
int agal_launch_transfer_batch(int kind, int key, cudaStream_t s, const void *args, const int *start, int n, int total);
size_t agal_transfer_args_size(int kind);
enum { AGAL_OP_INTERP = 1, AGAL_OP_AVERAGE, AGAL_OP_FORCES, AGAL_OP_FORCES_CV, AGAL_OP_SR_TICK };
int agal_step_batch_key(const agal_ctx *c);
int agal_launch_step_batch(int key, cudaStream_t s, const void *dev_args, const int *dev_start, int n, int total,
                           int fixup_only);
// Learned predictor hooks of the solution-based refinement (learn.cu).
int agal_learn_marks(agal_ctx *c);          // instead of the criterion when a learner is attached
int agal_learn_after_regrid(agal_ctx *c);   // after the refine/coarsen pass
