/*
 * ORACLE - CPU restatement of AGAL's octree-AMR lattice Boltzmann time step.
 *
 * This is test infrastructure: the checker that the CUDA product is compared
 * against, and the timed CPU baseline of bench.py.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.  The
 * product library never links or calls it.
 *
 * It restates the reference algorithm step by step in plain C with OpenMP,
 * using the reference's own data layout (structure-of-arrays populations with
 * the in-place swap-streaming slot convention) so that its arrays compare
 * element-wise with dumps of the reference CUDA build and of the product.
 *
 * Parity: the integer arrays of the root grid and the lattice tables are
 * pinned to golden vectors extracted from the reference sources
 * (tests/golden/make_golden.py).  The floating-point path is pinned against
 * the reference's own CUDA build when that build has been run (oracle/_ref);
 * otherwise it is "parity unpinned" for floating point.
 */
#ifndef AGAL_ORACLE_H
#define AGAL_ORACLE_H

#include <stddef.h>
#include <stdint.h>
#include "../include/agal_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_case orc_case;

/* Mesh::M_Init root grid (mesh_init.cu:325-516) and Solver_LBM::S_Init
   (solver_lbm_init.cu:4-76) with a fixed capacity of n_maxcblocks blocks.
   fp64 != 0 runs the arithmetic in double (ufloat_t = double). */
orc_case *orc_create(const agal_params *p, int64_t n_maxcblocks, int fp64);
void orc_destroy(orc_case *c);

/* Number of OpenMP threads used by the step routines (0 = library default). */
void orc_set_threads(int n);

int orc_get_counts(const orc_case *c, int *n_ids, int *id_max, int *n_gaps,
                   int64_t *n_maxcblocks, int *max_levels);

/* Restore n_ids[MAX_LEVELS+1], id_max[MAX_LEVELS+1] and n_gaps after
   orc_load, as the restart reader does (mesh_restart.cu:111-121). */
int orc_set_counts(orc_case *c, const int *n_ids, const int *id_max, int n_gaps);
/* Solver_LBM::S_SetIC (solver_lbm_kernels.cu:15-98). */
int orc_set_ic(orc_case *c, int L);
/* Solver_LBM::S_RefreshVariables (solver_lbm_kernels.cu:112-175). */
int orc_refresh(orc_case *c, int L);
/* Single phases of one level. */
int orc_collide(orc_case *c, int L);    /* solver_lbm_kernels.cu:206-289, 465-510 */
int orc_impose_bc(orc_case *c, int L);  /* solver_lbm_kernels.cu:693-920 */
int orc_stream(orc_case *c, int L);     /* solver_lbm_kernels.cu:534-660 */
/* S_Interpolate / S_Average with their refresh (solver_lbm_kernels_comm.cu). */
int orc_interpolate(orc_case *c, int L, int var);
int orc_average(orc_case *c, int L, int var);
/* Solver_LBM::S_ComputeRefCriteria (solver_lbm_criterion.cu:440-613). */
int orc_ref_criteria(orc_case *c);
/* Mesh::M_RefineAndCoarsenBlocks (mesh_amr.cu:2162-2744). */
int orc_refine_coarsen(orc_case *c);
/* Mesh::M_Advance_RefineWithSolution (mesh_advance.cu:185-243). */
int orc_refine_with_solution(orc_case *c);
/* Mesh::M_Advance_RefineNearWall without geometry (mesh_advance.cu:54-122):
   uniform refinement to N_LEVEL_START, Cu_RefineRegion marks (region_preset)
   up to MAX_LEVELS_WALL, S_SetIC per level, then the refined blocks frozen. */
int orc_refine_near_wall(orc_case *c);
/* Solver_LBM::S_Advance (solver_lbm_advance.cu:31-174). */
int orc_advance(orc_case *c, int L);
/* n coarse steps of the M_AdvanceLoop body (mesh_advance.cu:421-463):
   S_Advance from N_LEVEL_START, then every P_REFINE steps the
   solution-based refinement. */
int orc_advance_n(orc_case *c, int n);

/* Array sizes and copies with the AGAL_ARR_* selectors of agal_b200.h. */
size_t orc_array_bytes(const orc_case *c, int which);
int orc_dump(const orc_case *c, int which, void *buf, size_t bytes);
int orc_load(orc_case *c, int which, const void *buf, size_t bytes);

/* FP64 mass and momentum over fluid cells of leaf blocks (all levels). */
int orc_mass_momentum(orc_case *c, double *out);

/* ---- geometry (3D) ------------------------------------------------------
   faces: n_faces x 9 floats (v1x v1y v1z v2x v2y v2z v3x v3y v3z), as
   imported (geometry_import.cu:11-83) and length-refined
   (geometry_refine.cu:178-238).  Builds the bins of every bin level and, with
   G_BIN_MAKE_LINKS, the link bins (Geometry::G_InitBins); attaches the
   geometry to the mesh (Mesh::M_AddGeometry, mesh_init.cu:570-577), after
   which orc_refine_near_wall voxelizes and orc_advance imposes the wall. */
int orc_set_geometry(orc_case *c, const float *faces, int n_faces);
/* level >= 0: voxelizer bins of that bin level; level = -1: link bins. */
int orc_bins_info(const orc_case *c, int level, int *density, int *n_bins, int64_t *n_entries);
int orc_bins_copy(const orc_case *c, int level, int *n, int *N, int *ids);
int orc_voxelize_s1(orc_case *c, int L);          /* mesh_voxelizer.cu:34-156   */
int orc_update_solid_children(orc_case *c, int L);/* mesh_voxelizer.cu:247-259  */
int orc_voxelize_s2(orc_case *c, int L);          /* mesh_voxelizer.cu:158-189  */
int orc_voxelize_s3(orc_case *c);                 /* mesh_voxelizer.cu:191-245  */
int orc_link_lengths(orc_case *c, int L);         /* mesh_voxelizer.cu:261-294  */
/* out = {n_faces, n_solida, n_solidb, n_maxcells_b} */
int orc_geometry_counts(const orc_case *c, int64_t *out);
/* MEA force sums {Fpx, Fmx, Fpy, Fmy, Fpz, Fmz}; resets the partials. */
int orc_forces(orc_case *c, double *out);

#ifdef __cplusplus
}
#endif
#endif
