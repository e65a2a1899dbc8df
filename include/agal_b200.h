/*
 * agal_b200.h - C ABI of the B200-native octree-AMR lattice Boltzmann time step.
 *
 * The library (agal_b200/libagal_b200.so) owns every device array of one
 * simulation case in an opaque context.  All entry points take plain pointers
 * and sizes, return an int status (AGAL_OK or a negative AGAL_ERR_* code) and
 * never call exit().  Kernels run on the context's CUDA stream.
 *
 * Reference interface replaced (paths relative to the AGAL source tree):
 *   Solver<...> virtuals          inc/solver.h:62-71
 *   Solver_LBM<...> routines      inc/solver_lbm.h:153-179
 *   Mesh<...> AMR/advance entry   inc/mesh.h:676-727
 *   Parser input.txt maps          inc/parser.h:58-183
 */
#ifndef AGAL_B200_H
#define AGAL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The library is built with -fvisibility=hidden; the entry points declared
   here are the only exported symbols. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- status codes ------------------------------------------------------ */
#define AGAL_OK                 0
#define AGAL_ERR_PARAM         -1   /* invalid argument or input.txt value       */
#define AGAL_ERR_OOM           -2   /* device allocation failed / capacity short  */
#define AGAL_ERR_GAPS          -3   /* block-ID gap set exhausted during refine   */
#define AGAL_ERR_TIMEOUT       -4   /* a bounded device wait gave up              */
#define AGAL_ERR_CUDA          -5   /* CUDA runtime error (see agal_last_error)   */
#define AGAL_ERR_IO            -6   /* file missing, unreadable or corrupt        */
#define AGAL_ERR_STATE         -7   /* call not valid in the context's state      */
#define AGAL_ERR_UNSUPPORTED   -8   /* option combination not built               */

/* ---- enumerations (runtime forms of the reference's compile-time packs) -- */
/* velocity set: inc/solver_lbm.h:13-18 */
#define AGAL_D2Q9   0
#define AGAL_D3Q19  1
#define AGAL_D3Q27  2
/* collision operator: inc/solver_lbm.h:19-24 (TRT not built) */
#define AGAL_BGK    0
#define AGAL_MRT    2
/* interpolation order: inc/solver_lbm.h:25-30 */
#define AGAL_INTERP_LINEAR 0
#define AGAL_INTERP_CUBIC  2
/* population storage in HBM */
#define AGAL_STORE_FP32 0
#define AGAL_STORE_FP64 1
#define AGAL_STORE_FP16 2   /* weight offsets g = f - w_p, collided in FP32 */
#define AGAL_STORE_BF16 3
/* agal_params.half_rounding */
#define AGAL_ROUND_STOCHASTIC 0
#define AGAL_ROUND_NEAREST 1   /* weight offsets g = f - w_p, collided in FP32 */
/* boundary-condition presets of the Cu_ImposeBC hook, inc/custom.h:79-117 */
#define AGAL_BC_NONE    0   /* plain half-way bounce-back on every wall        */
#define AGAL_BC_LDC2D   1   /* moving lid on boundary -4 (y+), custom.h:80-84   */
#define AGAL_BC_LDC3D   2   /* moving lid on boundary -6 (z+), custom.h:100-104 */
#define AGAL_BC_FPSC2D  3   /* inflow -1,-3,-4; outflow -2, custom.h:87-97      */
#define AGAL_BC_FPSC3D  4   /* inflow -1,-3..-6; outflow -2, custom.h:107-117   */
/* initial-condition presets of the Cu_ComputeIC hook, inc/custom.h:50-60 */
#define AGAL_IC_REST    0   /* rho = 1, u = 0                                   */
#define AGAL_IC_UNIFORM 1   /* rho = 1, u = (u_ref, 0, 0) (+ seeded noise)      */
/* near-wall refinement regions of the Cu_RefineRegion hook, inc/custom.h:17-42,
   evaluated on a block's bounds (x + 1e-5, x + 4 dx_L - 1e-5) as
   mesh_criterion.cu:28-50 passes them */
#define AGAL_REGION_NONE     0   /* no block (the shipped hook returns false)     */
#define AGAL_REGION_BOUNDARY 1   /* blocks on the domain boundary (onb == 1)      */
#define AGAL_REGION_BOX      2   /* blocks inside [0.25, 0.75]^d (coordinates)    */

/* S_CRITERION values: solver_lbm_criterion.cu:572-575 (0, 1) and the
   percentile mode of this library (2) */
#define AGAL_CRITERION_VORTICITY  0
#define AGAL_CRITERION_Q          1
#define AGAL_CRITERION_PERCENTILE 2
#define AGAL_CRITERION_LEARNED    3   /* network predictions, percentile rule as the judge (agal_learn_attach) */

/* interpolation / averaging modes, inc/mesh.h:58-62 */
#define AGAL_INTERP_INTERFACE 0
#define AGAL_INTERP_ADDED     1
#define AGAL_AVERAGE_INTERFACE 0
#define AGAL_AVERAGE_BLOCK     1
#define AGAL_AVERAGE_GRID      2

/* array selectors for agal_dump / agal_load */
#define AGAL_ARR_F              0  /* populations, reference slot layout [Q][n_maxcells], float64, solid = -1 */
#define AGAL_ARR_MACROS         1  /* rho,u,v(,w) [dim+1][n_maxcells], float64 (after agal_refresh)          */
#define AGAL_ARR_CELLS_ID_MASK  2  /* int32 [n_maxcells]                      mesh.h:366                     */
#define AGAL_ARR_CBLOCK_F_X     3  /* float32 [dim][n_maxcblocks]             mesh.h:389                     */
#define AGAL_ARR_CBLOCK_ID_MASK 4  /* int32 [n_maxcblocks]                    mesh.h:393                     */
#define AGAL_ARR_CBLOCK_ID_NBR  5  /* int32 [N_Q_max][n_maxcblocks]           mesh.h:397                     */
#define AGAL_ARR_CBLOCK_ID_NBR_CHILD 6 /* int32 [N_Q_max][n_maxcblocks]       mesh.h:404                     */
#define AGAL_ARR_CBLOCK_ID_ONB  7  /* int32 [n_maxcblocks]                    mesh.h:407                     */
#define AGAL_ARR_CBLOCK_ID_REF  8  /* int32 [n_maxcblocks]                    mesh.h:416                     */
#define AGAL_ARR_CBLOCK_LEVEL   9  /* int32 [n_maxcblocks]                    mesh.h:419                     */
#define AGAL_ARR_ID_SET        10  /* int32 [MAX_LEVELS][n_maxcblocks]        mesh.h:428                     */
#define AGAL_ARR_GAP_SET       11  /* int32 [n_maxcblocks] (first n_gaps valid) mesh.h:459                   */
#define AGAL_ARR_CBLOCK_ID_ONB_SOLID 12 /* int32 [n_maxcblocks] wall-block slot, -1 = none  mesh.h:515      */
#define AGAL_ARR_CELLS_F_X_B   13  /* float32 [N_Q_max][n_maxcells_b] link lengths, -1 = none   mesh.h:491   */
#define AGAL_ARR_CBLOCK_F_FF   14  /* float64 [6][n_maxcblocks] MEA force partials per block   mesh.h:518    */
#define AGAL_ARR_NU_SGS        15  /* float64 [n_maxcells] LES eddy viscosity (S_LES > 0), field row N_Q+4 */

/* ---- parameters: every input.txt key of inc/parser.h:62-144 ------------- */
typedef struct agal_params {
    /* MESH (integer keys) */
    int MAX_LEVELS_WALL, MAX_LEVELS_INTERIOR, N_ITER_TOTAL, N_LEVEL_START, Nx, N_RESTART;
    int PERIODIC_X, PERIODIC_Y, PERIODIC_Z;
    /* GEOMETRY (integer keys) */
    int G_LOADTYPE, G_PRINT, G_VIS_TREE, G_BIN_DENSITY, G_BIN_APPROACH, G_BIN_LEVELS, G_BIN_SPEC, G_BIN_MAKE_LINKS;
    /* SOLVER (integer keys) */
    /* S_LES: 0 none, 1 Smagorinsky, 2 WALE, 3 Vreman (inc/solver_lbm.h:31-37,
       solver_lbm_kernels_les.cu); with BGK (one or several levels, walls
       included), else agal_create returns AGAL_ERR_UNSUPPORTED */
    int S_COLLISION, S_INTERP, S_INTERP_HYBRID, S_AVERAGE, S_CRITERION, S_LES, S_FORCE_ORDER, S_FORCE_TYPE, S_BC_TYPE;
    /* REFINEMENT / PROBING / OUTPUT (integer keys) */
    int P_REFINE, N_PROBE, N_PROBE_DENSITY, N_PROBE_FREQUENCY, N_PROBE_FORCE, N_PROBE_F_START, N_PROBE_F_FREQUENCY;
    int N_PROBE_AVE, N_PROBE_AVE_FREQUENCY, N_PROBE_AVE_START;
    int N_PRINT_LEVELS, N_PRINT_LEVELS_VTHB, N_PRINT_LEVELS_PATCH, N_PRINT_LEVELS_IMAGE, P_OUTPUT, N_OUTPUT, N_OUTPUT_START;
    int VOL_I_MIN, VOL_I_MAX, VOL_J_MIN, VOL_J_MAX, VOL_K_MIN, VOL_K_MAX, USE_CPU;
    /* double keys */
    double L_c, L_fy, L_fz, v0, G_NEAR_WALL_DISTANCE, s1, s2, s3, s4, s5, s6, V_PROBE_TOL;
    double N_REFINE_START, N_REFINE_INC, N_REFINE_MAX;
    double S_FORCEVOLUME_Xm, S_FORCEVOLUME_XM, S_FORCEVOLUME_Ym, S_FORCEVOLUME_YM, S_FORCEVOLUME_Zm, S_FORCEVOLUME_ZM;
    /* string keys */
    char I_DIR_NAME[256], P_DIR_NAME[256], G_FILENAME[256];

    /* Runtime selections that the reference fixes at compile time
       (main.cu:48-77 ArgsPack/LBMPack, custom.h hooks). */
    int velocity_set;     /* AGAL_D2Q9 / AGAL_D3Q19 / AGAL_D3Q27 */
    int collision;        /* AGAL_BGK / AGAL_MRT                 */
    int interp_order;     /* AGAL_INTERP_LINEAR / AGAL_INTERP_CUBIC */
    int storage;          /* AGAL_STORE_*                        */
    int bc_preset;        /* AGAL_BC_*                           */
    int ic_preset;        /* AGAL_IC_*                           */
    int region_preset;    /* AGAL_REGION_*                       */
    /* S_CRITERION = AGAL_CRITERION_PERCENTILE: leaf blocks whose maximum
       vorticity magnitude lies above the ref_pct_hi quantile of all leaf
       blocks are refined, refined blocks below the ref_pct_lo quantile
       coarsened (no reference counterpart). */
    double ref_pct_hi, ref_pct_lo;
    double u_ref;         /* velocity of the presets (custom.h hard-codes 0.05) */
    double ic_noise;      /* relative amplitude of seeded IC noise (0 = none)   */
    uint64_t seed;        /* seed of the IC noise                               */
    /* Capacity in cell-blocks.  0 = size from free device memory with
       mem_frac, as mesh_init.cu:155-169 does with M_FRAC = 0.975. */
    int64_t n_maxcblocks;
    double mem_frac;
    /* CUDA device ordinal of the context (-1 = the calling thread's current device). */
    int device;
    /* Rounding of the FP16/BF16 weight offsets written by the step kernels:
       AGAL_ROUND_STOCHASTIC (default) or AGAL_ROUND_NEAREST.  Round-to-nearest
       loses every per-step change below half a unit in the last place, so a
       slowly developing flow stagnates (FP16 velocity 9e-3 from FP64 after
       10,000 steps of a 256^2 cavity at Re 100).  Stochastic rounding rounds
       up with probability equal to the discarded fraction, so the stored
       value is unbiased; its random bits are a hash of the value's cell and
       direction and of the coarse-step counter, so results are deterministic,
       identical across step kernel variants, and continue bit for bit from a
       restart.  No reference counterpart (the reference stores FP32/FP64). */
    int half_rounding;
} agal_params;

typedef struct agal_ctx agal_ctx;

/* Defaults of inc/parser.h:62-144 plus D2Q9/BGK/cubic/FP32/no-BC presets. */
int agal_params_default(agal_params *p);
/* sizeof(agal_params), for foreign-function bindings to check their layout. */
size_t agal_params_size(void);
/* Parse <input_dir>/input.txt with the reference's rules (parser.h:146-180):
   '#' comments, "A*Nx" integer factors, unknown keys reported and skipped.
   Starts from the values already in *p. */
int agal_params_read(const char *input_dir, agal_params *p);
/* Set one key by name from its text value (same rules as a file line). */
int agal_params_set(agal_params *p, const char *key, const char *value);

/* Mesh::M_Init (mesh_init.cu:11-567) + Solver_LBM::S_Init (solver_lbm_init.cu:4-102):
   allocate the block pool, build the root grid, set tau per level. */
int agal_ctx_create(const agal_params *p, agal_ctx **out);
int agal_ctx_destroy(agal_ctx *ctx);
/* Text of the last error on this context (or of the last failed create). */
const char *agal_last_error(const agal_ctx *ctx);

/* Host mirrors: n_ids[MAX_LEVELS+1], id_max[MAX_LEVELS+1], n_gaps, capacity. */
int agal_get_counts(const agal_ctx *ctx, int *n_ids, int *id_max, int *n_gaps,
                    int64_t *n_maxcblocks, int *max_levels);
/* Restore the host mirrors after loading a mesh with agal_load, as the
   restart reader does (mesh_restart.cu:111-121): n_ids[MAX_LEVELS+1],
   id_max[MAX_LEVELS+1], n_gaps.  Rebuilds the step metadata of the loaded
   blocks.  AGAL_ERR_PARAM if a count exceeds the pool. */
int agal_set_counts(agal_ctx *ctx, const int *n_ids, const int *id_max, int n_gaps);

/* Solver::S_SetIC (solver_lbm_kernels.cu:79-98). */
int agal_set_ic(agal_ctx *ctx, int L);
/* Solver::S_RefreshVariables (solver_lbm_kernels.cu:161-175): macros of level L. */
int agal_refresh(agal_ctx *ctx, int L);
/* Solver::S_Advance(i_dev, L, tmp) (solver_lbm_advance.cu:31-174): one step of
   level L and, recursively, of every finer level.  L = N_LEVEL_START is one
   coarse step. */
int agal_advance(agal_ctx *ctx, int L);
/* n coarse steps of the M_AdvanceLoop body (mesh_advance.cu:421-463): each a
   2^N_LEVEL_START-fold S_Advance from N_LEVEL_START, then, on a multi-level
   mesh, the solution-based refinement every P_REFINE steps (counted over the
   context's life).  With use_graph != 0 a coarse step is captured once per
   mesh and buffer parity into a CUDA graph and replayed (same kernels). */
int agal_advance_n(agal_ctx *ctx, int n, int use_graph);

/* ---- multi-level mesh ------------------------------------------------------ */
/* Solver_LBM::S_Interpolate (solver_lbm_kernels_comm.cu:141-155, 642-658):
   refresh the macros of level L, then interpolate from level L into the ghost
   cells of its children (AGAL_INTERP_INTERFACE) or into every cell of the
   children of blocks marked for refinement (AGAL_INTERP_ADDED). */
int agal_interpolate(agal_ctx *ctx, int L, int var);
/* Solver_LBM::S_Average (solver_lbm_kernels_comm.cu:351-370): refresh level
   L+1, then average it into level L (AGAL_AVERAGE_INTERFACE/_BLOCK/_GRID). */
int agal_average(agal_ctx *ctx, int L, int var);
/* Solver_LBM::S_ComputeRefCriteria (solver_lbm_criterion.cu:595-613): marks
   blocks for refinement/coarsening from the macros of the last refresh
   (S_CRITERION, N_REFINE_START/_INC/_MAX, MAX_LEVELS_INTERIOR). */
int agal_ref_criteria(agal_ctx *ctx);
/* Mesh::M_RefineAndCoarsenBlocks (mesh_amr.cu:2162-2744): acts on the marks;
   block IDs from the gap stack, ID sets, neighbour lists, masks rebuilt. */
int agal_refine_coarsen(agal_ctx *ctx);
/* Mesh::M_Advance_RefineWithSolution (mesh_advance.cu:185-243): grid
   average, interface interpolation, criterion, refine/coarsen. */
int agal_refine_with_solution(agal_ctx *ctx);
/* Mesh::M_ComputeRefCriteria (mesh_criterion.cu:90-119) on level L:
   AGAL_MESH_REF_NW_CASES marks the unrefined blocks of the Cu_RefineRegion
   preset (region_preset), AGAL_MESH_REF_UNIFORM every unrefined block,
   AGAL_MESH_REF_SOLUTION runs agal_ref_criteria when level L has blocks. */
#define AGAL_MESH_REF_NW_CASES 0
#define AGAL_MESH_REF_UNIFORM  2
#define AGAL_MESH_REF_SOLUTION 3
int agal_mesh_ref_criteria(agal_ctx *ctx, int L, int var);
/* Mesh::M_FreezeRefinedCells (mesh_amr.cu:2050-2074): var 0 makes refined
   blocks permanent (not coarsened), var 1 releases them. */
int agal_freeze_refined_cells(agal_ctx *ctx, int var);
/* Mesh::M_Advance_RefineNearWall (mesh_advance.cu:54-122) without geometry:
   uniform refinement to N_LEVEL_START, Cu_RefineRegion marks (region_preset)
   up to MAX_LEVELS_WALL with S_SetIC per level, refined blocks frozen. */
int agal_refine_near_wall(agal_ctx *ctx);
/* Coarse steps taken by agal_advance_n and the number of blocks refined /
   coarsened by the last refine/coarsen pass (mesh_amr.cu:2714-2744 prints
   them).  Pointers may be NULL. */
int agal_refine_stats(const agal_ctx *ctx, long long *iter, int *n_refined, int *n_coarsened);
/* CUDA graphs of agal_advance_n built (instantiated) and updated in place
   (after a regrid the captured step usually keeps its topology and only its
   launch sizes and arguments change).  No reference counterpart. */
int agal_graph_stats(const agal_ctx *ctx, long long *builds, long long *updates);

/* ---- Geometry (3D velocity sets) -------------------------------------------
   agal_set_geometry: faces = n_faces x 9 floats (v1x v1y v1z v2x v2y v2z v3x
   v3y v3z, unit-length domain coordinates), as Geometry imports and splits them
   (geometry_import.cu:11-83, geometry_refine.cu:178-238).  Builds the
   voxelizer bins of every bin level and, with G_BIN_MAKE_LINKS, the link bins
   (Geometry::G_InitBins, geometry_bins.h:106-203; Bins::G_MakeBinsGPU and
   _MD, geometry_bins_gpu.cu:587-1300), then attaches the geometry to the mesh
   (Mesh::M_AddGeometry, mesh_init.cu:570-577): agal_refine_near_wall then
   voxelizes and computes link lengths, and the step imposes the wall
   (interpolated bounce-back with S_BC_TYPE 1) and sums MEA forces
   (S_FORCE_TYPE 0).  The bin grid spans the unit cube, as the reference's
   does (its cell and bin indexing assume L_c = L_fy = L_fz = 1); a face whose
   bins fall outside it is refused (AGAL_ERR_PARAM). */
int agal_set_geometry(agal_ctx *ctx, const float *faces, long long n_faces);
/* Geometry import on the host, no device needed (faces n x 9 floats; with
   faces NULL only *n is set; AGAL_ERR_PARAM if cap is too small, *n then
   holding the size needed):
   agal_geometry_read_stl   - ASCII STL as G_ImportSTL_ASCII (geometry_import.cu:11-83),
                              degenerate facets dropped;
   agal_geometry_read_text  - the primitives of a geometry.txt
                              (G_ImportBoundariesFromTextFile + G_Convert_IndexListsToCoordList,
                              geometry_add.cu:539-666): BOX, PRISM, SPHERE; the 2D shapes
                              and NACA profiles give AGAL_ERR_UNSUPPORTED;
   agal_geometry_refine_length - G_RefineFaces_Length (geometry_refine.cu): faces longer than
                              0.95 G_BIN_SPEC min(L) / (2^(G_BIN_LEVELS-1) G_BIN_DENSITY)
                              split at the edge midpoints, in place;
   agal_import_geometry     - main.cu:94-101 for a context: G_LOADTYPE 0 reads
                              I_DIR_NAME/geometry/G_FILENAME, 1 reads I_DIR_NAME/geometry.txt,
                              then the length refinement and agal_set_geometry. */
int agal_geometry_read_stl(const char *path, float *faces, long long cap, long long *n);
int agal_geometry_read_text(const agal_params *p, const char *path, float *faces, long long cap, long long *n);
int agal_geometry_refine_length(const agal_params *p, float *faces, long long cap, long long *n);
int agal_import_geometry(agal_ctx *ctx);
/* CSR bins of voxelizer bin level `level`, or of the link bins for level -1
   (binned_face_ids_n/N/ids).  Array pointers may be NULL (sizes first). */
int agal_bins_get(agal_ctx *ctx, int level, int *density, int *n_bins, long long *n_entries, int *n, int *N,
                  int *ids);
int agal_voxelize_s1(agal_ctx *ctx, int L);          /* Mesh::M_Geometry_Voxelize_S1, mesh_voxelizer.cu:34-156  */
int agal_update_solid_children(agal_ctx *ctx, int L);/* Mesh::M_UpdateSolidChildren, mesh_voxelizer.cu:247-259  */
int agal_voxelize_s2(agal_ctx *ctx, int L);          /* Mesh::M_Geometry_Voxelize_S2, mesh_voxelizer.cu:158-189  */
int agal_voxelize_s3(agal_ctx *ctx);                 /* Mesh::M_Geometry_Voxelize_S3, mesh_voxelizer.cu:191-245  */
int agal_link_lengths(agal_ctx *ctx, int L);         /* Mesh::M_LinkLengthComputation, mesh_voxelizer.cu:261-294 */
/* out = {n_faces, n_solida, n_solidb, n_maxcells_b} (mesh.h:304-307). */
int agal_geometry_counts(const agal_ctx *ctx, long long *out);
/* Solver_LBM::S_ReportForces (solver_lbm_compute.cu:166-215): out = {Fpx, Fmx,
   Fpy, Fmy, Fpz, Fmz}, the FP64 sums of the per-block MEA partials over block
   IDs below id_max[MAX_LEVELS]; the partials are reset.  The force is
   (Fp - Fm) / dx of the finest level. */
int agal_forces(agal_ctx *ctx, double *out);

/* ---- Batches of independent cases (no reference counterpart: AGAL runs one
   case per process) ------------------------------------------------------------
   agal_batch_advance_n advances every case of the batch by n coarse steps (each
   with its own refinement every P_REFINE steps) as one CUDA graph per coarse
   step whose branches are the cases, so small cases run concurrently.  Each
   case ends exactly where agal_advance_n would have left it.  The contexts stay
   owned by the caller and must outlive the batch; all on one device. */
/* ---- Learned refinement predictor (no reference counterpart) ----------------
   agal_learn_gemm_bf16: D[M x N] = A[M x K] . B[N x K]^T with BF16 inputs (bit
   patterns) and FP32 accumulation on the tensor cores (tcgen05), host buffers;
   N <= 32, K a multiple of 16.  The kernel behind the network's layers. */
int agal_learn_gemm_bf16(const uint16_t *A, const uint16_t *B, float *D, int M, int N, int K);

/* The predictor: per block of 4^d cells, 8 input channels ((rho-1)/U^2, u/U,
   v/U, w/U, 2^L |curl u|/U, level/(ML-1), refined flag, 1), three 3^d
   convolutions 8 -> 32 -> 32 -> 2 (ReLU between, zero padding at the block
   faces), the last averaged over the block: logits of the percentile rule's
   two decisions at the next regrid (a leaf block's value above the upper
   quantile, a block's value below the lower one; the marks follow with the
   rule's admissibility).  BF16 weights and activations, FP32 accumulation
   (tcgen05), Adam on FP32 master weights.  Snapshots live on the device:
   agal_learn_record stores the features of a case's current blocks and the
   rule's decisions on that state, agal_learn_label labels the latest
   unlabelled snapshot with the decisions of the rule's last run. */
typedef struct agal_learn agal_learn;
int agal_learn_create(int dim, unsigned long long seed, agal_learn **out);
int agal_learn_destroy(agal_learn *m);
const char *agal_learn_last_error(const agal_learn *m);
int agal_learn_num_params(const agal_learn *m, long long *n);
/* Parameters W1 [32][K1p], b1 [32], W2 [32][K2], b2 [32], W3 [2][K2], b3 [2];
   K2 = 32 T, K1p = 16 ceil(8 T / 16), T = 3^d, column = tap * channels +
   channel, tap = (dx+1) + 3 (dy+1) + 9 (dz+1); W1's padding columns are 0. */
int agal_learn_get_params(agal_learn *m, float *out, long long n);
int agal_learn_set_params(agal_learn *m, const float *in, long long n);
int agal_learn_record(agal_learn *m, agal_ctx *ctx);
int agal_learn_label(agal_learn *m, agal_ctx *ctx);
/* {snapshots, labelled, regrids seen, judged regrids, plain refinement marks
   at judged regrids, of those not predicted by the network} */
int agal_learn_counts(const agal_learn *m, long long *out);
/* Host copies of snapshot k: n blocks, X [n*4^d][8], labels [n][2], weights [n]. */
int agal_learn_snapshot(agal_learn *m, int k, int *n_blocks, float *X, float *Y, float *Wt);
/* The percentile rule's decisions [n][2] on snapshot k's own state. */
int agal_learn_snapshot_decisions(agal_learn *m, int k, float *D);
/* Weights of the positive class in the loss of the two outputs (refinement,
   coarsening marks are rare): per block and output
   wt (pw y softplus(-z) + (1 - y) softplus(z)); default 1, 1. */
int agal_learn_set_class_weights(agal_learn *m, double refine, double coarsen);
/* Mean binary cross entropy of snapshot k and its gradient w.r.t. the parameters. */
int agal_learn_gradients(agal_learn *m, int k, float *grad, long long n, double *loss);
/* Adam over labelled snapshots [first, last), `epochs` passes in seeded order. */
int agal_learn_train(agal_learn *m, int first, int last, int epochs, double lr, unsigned long long seed, double *loss);
/* Logits [n][2] of snapshot k's blocks. */
int agal_learn_predict_snapshot(agal_learn *m, int k, float *out);
/* Couple a predictor with a case's solution-based refinement: mode 1 collects
   labelled snapshots (plain criterion), mode 2 predicts (the marks of a regrid
   are the network's, made after the previous regrid, for probabilities above
   `threshold`; every judge_every-th regrid the percentile rule also runs and
   the refinements the network missed are counted and applied); mode 0
   detaches.  The predictor must outlive the coupling. */
int agal_learn_attach(agal_ctx *ctx, agal_learn *m, int mode, int judge_every, double threshold);
/* Look-ahead (horizon 1..64; 0, the default, is the one-regrid-delayed
   mode above).  In mode 1 a snapshot is taken at each regrid before its
   refinement pass and labelled with the rule's decisions at that regrid and
   the next horizon - 1: refine if any of them refines a block, coarsen only
   if all of them coarsen it, weight 0 for a block that changes level in
   between.  In mode 2 the network predicts from the state at a regrid and its
   marks apply at that same regrid, so they cover the next `horizon` periods
   and a predicting case can regrid `horizon` times less often (its P_REFINE
   times `horizon`).  Set it before collecting. */
int agal_learn_set_horizon(agal_learn *m, int horizon);
/* Inference convolutions as implicit GEMMs (on = 1, the default: the im2col
   columns are gathered into the tcgen05 GEMM's shared-memory stages) or
   through materialised columns (0).  The logits are the same bit for bit. */
int agal_learn_set_implicit(agal_learn *m, int on);
/* Separate probability thresholds of the refinement and coarsening outputs in
   predict mode (after agal_learn_attach, which sets both to `threshold`). */
int agal_learn_set_thresholds(agal_learn *m, double refine, double coarsen);

typedef struct agal_batch agal_batch;
int agal_batch_create(agal_ctx *const *cases, int n_cases, agal_batch **out);
int agal_batch_destroy(agal_batch *batch);
int agal_batch_advance_n(agal_batch *batch, int n, int use_graph);
int agal_batch_sync(agal_batch *batch);
int agal_batch_get_stream(const agal_batch *batch, void **stream);
const char *agal_batch_last_error(const agal_batch *batch);
/* Work-list mode (on by default where every case allows it: no LES, no
   control-volume forces): each coarse step of the batch runs the fused steps
   of all cases as one persistent kernel per phase over a global list of
   (case, chunk of blocks), each case's arguments read from a device table,
   followed by one batched fix-up launch; interpolation and averaging phases
   are one launch each over (case, parent block) items; forces and the
   rounding counter run per case.  0 returns to one graph branch per case.  Results are identical
   either way.  AGAL_ERR_UNSUPPORTED when a case does not allow it. */
int agal_batch_set_worklist(agal_batch *batch, int on);
/* Autotuner of the batch's launch mode: times `steps` graph-replayed coarse
   steps in work-list mode (where allowed) and with one branch per case, each
   after two warm-up steps, and keeps the faster.  The cases really advance
   (2 x (steps + 2) coarse steps, regrids included).  ms[2] (may be NULL)
   receives the per-step times {branches, work list (-1 if not allowed)},
   *mode (may be NULL) 1 for the work list, 0 for branches. */
int agal_batch_autotune(agal_batch *batch, int steps, float *ms, int *mode);

/* Device <-> host transfers of one mesh/solver array (AGAL_ARR_*).
   bytes must equal the size reported by agal_array_bytes. */
int agal_array_bytes(const agal_ctx *ctx, int which, size_t *bytes);
/* Checkpoint / restart in the reference's restart.bin format
   (Mesh::M_Restart SAVE / LOAD, mesh_restart.cu:45-225): the counts, ID sets,
   gap stack, cell masks, block arrays and populations up to id_max, as floats
   (doubles for FP64 storage).  Load adapts the gap stack to this context's
   n_maxcblocks like the reference, restores the counts and the coarse-step
   counter (`iter` is the M_AdvanceLoop index of the last step taken; the
   loop resumes at iter + 1), and refuses a state beyond the
   block pool (AGAL_ERR_OOM).  No velocity probes are kept: save writes none
   and a zero running mean, load skips them.  Geometry arrays are not part of
   the format.  The file holds f = w + g in FP32: for FP16 storage (offsets
   g stored times 2^10) the smallest offsets are finer than FP32 resolves
   near the weights, so a load reproduces FP16 states to that rounding (FP32,
   FP64 and BF16 states exactly). */
int agal_restart_save(agal_ctx *ctx, const char *path, int iter);
int agal_restart_load(agal_ctx *ctx, const char *path, int *iter);

/* Headless uniform-grid output in the reference's out_direct.dat format
   (header: mesh_init.cu:114-150; frames: Mesh::M_RenderAndPrint_Uniform,
   mesh_print_uniform.cu:96-188).  The box is VOL_{I,J,K}_{MIN,MAX} (cells,
   rounded down to root blocks) at the resolution of level N_PRINT_LEVELS-1;
   each output cell takes the macros of the cell of the deepest block (up to
   that level) covering it.  agal_uniform_header creates the file;
   agal_uniform_frame prepares the state as M_Advance_PrintData does (grid
   average, interface interpolation, refresh of every level) and appends
   t = iter / Nx and the fields rho, u, v, w, level, block ID (doubles, x
   fastest).  agal_uniform_render fills out[6][nz][ny][nx] from the current
   macros without preparing; agal_uniform_append appends a frame of the
   current macros without preparing (M_RenderAndPrint_Uniform alone);
   agal_uniform_dims gives {nx, ny, nz}. */
int agal_uniform_dims(const agal_ctx *ctx, int *dims);
int agal_uniform_render(agal_ctx *ctx, double *out, long long n);
int agal_uniform_header(agal_ctx *ctx, const char *path);
int agal_uniform_frame(agal_ctx *ctx, const char *path, int iter);
int agal_uniform_append(agal_ctx *ctx, const char *path, int iter);
int agal_dump(agal_ctx *ctx, int which, void *host_buf, size_t bytes);
int agal_load(agal_ctx *ctx, int which, const void *host_buf, size_t bytes);

/* FP64 sums over every fluid leaf cell: out[0] = mass, out[1..dim] = momentum.
   Reads the macros of agal_refresh-free state (computes them itself).  The
   partial sums are reduced on the device in a fixed order (deterministic).
   No reference counterpart (the reference has no global conservation check;
   its per-cell macros are S_ComputeProperties, solver_lbm_compute.cu:5). */
int agal_mass_momentum(agal_ctx *ctx, double *out);
/* The same sums enqueued on the context's stream without waiting: out[0..3]
   (four doubles; out[3] = 0 in 2D) is written when the stream reaches the
   copy, so it is valid after agal_sync.  Pass pinned host memory
   (cudaHostAlloc / cudaHostRegister) for an asynchronous copy; with pageable
   memory the copy waits.  Successive calls may share one buffer only if the
   caller reads it in between. */
int agal_mass_momentum_async(agal_ctx *ctx, double *out);

/* Same sums as agal_mass_momentum, for callers that must not allocate device
   memory (a memory-capped serving process, a pool that is fully reserved, a
   code path between other libraries' allocations): the partial sums live in a
   fixed static device array of AGAL_MASS_NOALLOC_MAX_PARTIALS x 4 doubles
   (8 MiB), and no call allocates or frees.  One partial covers 256 active
   cells of one level, so a mesh of more than 67,108,864 active cells (summed
   per level, each level rounded up to 256) is rejected with AGAL_ERR_PARAM.
   Every call looks the array up (cudaGetSymbolAddress, no allocation) with
   the context's device current, so a device reset between calls is
   followed; the first call on a device may load the module and belongs
   before any stream capture.  The array is
   shared by every context of the device: calls that overlap in time race
   and must be serialised by the caller.  No reference counterpart. */
#define AGAL_MASS_NOALLOC_MAX_PARTIALS 262144
int agal_mass_momentum_noalloc(agal_ctx *ctx, double *out);

/* Autotuner of the fused step kernel.  Variants: 1 = one cell per thread,
   2 = two cells per thread (one-shot grids), 3 = persistent pipeline with the
   cell-blocks staged in shared memory by TMA bulk copies, 4 = one x-row of
   four cells per thread with vector loads and stores (FP64 and LES contexts
   run variant 1 in its place), 5 = the root level of 2D cases as tiles of
   8 x 8 cell-blocks per CTA, each output block written whole (root blocks per
   side a multiple of 8, no geometry, no LES; elsewhere variant 4 runs in its
   place), 6 = the root level of 2D cases as tiles of 8 x 4 cell-blocks
   whose in-tile pushes go through shared memory and whose output block rows
   are written with 16-byte stores (root blocks per side a multiple of 8 in x
   and 4 in y, no geometry, no LES; elsewhere variant 1 runs in its place).
   Times each variant reps times on level L's current state without
   advancing it (the step writes only the scratch population buffer) and
   keeps the fastest for the context.  ms[6] (may be NULL) receives the
   per-launch times, *variant (may be NULL) the choice.
   All variants give bit-identical populations.  No reference counterpart:
   the reference launches one fixed 16/64-thread shape (cppspec.h:96). */
int agal_autotune(agal_ctx *ctx, int L, int reps, float *ms, int *variant);
/* Set the step kernel variant explicitly (1..6, as for agal_autotune). */
int agal_set_tuning(agal_ctx *ctx, int variant);

/* Synchronise the context's stream; returns the first pending CUDA error, or
   AGAL_ERR_TIMEOUT if a bounded wait inside a kernel expired. */
int agal_sync(agal_ctx *ctx);
/* The context's cudaStream_t (as void*), so that callers can order their own
   work and CUDA events with the library's kernels. */
int agal_get_stream(const agal_ctx *ctx, void **stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* AGAL_B200_H */
