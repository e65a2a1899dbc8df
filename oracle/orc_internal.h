/* ORACLE (test infrastructure only): private state of a CPU oracle case. */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H

#include <stdint.h>
#include "agal_oracle.h"
#include "orc_lattice.h"

#define ORC_MAXL 16

/* Constants of inc/mesh.h:34-105 and inc/cppspec.h:124-125. */
#define ORC_N_SKIPID (-999)
#define ORC_N_SPECID (-998)
#define ORC_REF_UNREFINED 0
#define ORC_REF_REFINED 1
#define ORC_REF_REFINED_WCHILD 2
#define ORC_REF_REFINED_PERM 3
#define ORC_REF_MARK_REFINE 4
#define ORC_REF_MARK_COARSEN 5
#define ORC_REF_NEW 6
#define ORC_REF_REMOVE 7
#define ORC_REF_INACTIVE 8
#define ORC_REF_UNREFINED_VIO 9
#define ORC_REF_REFINED_WCHILD_PERM 10
#define ORC_CELL_INTERIOR 0
#define ORC_CELL_INTERFACE 1
#define ORC_CELL_GHOST 2
#define ORC_CELL_SOLID (-1)
#define ORC_CELL_BOUNDARY (-6)
#define ORC_BLOCK_REGULAR 0
#define ORC_BLOCK_INTERFACE 1
#define ORC_BLOCK_SOLIDB (-1)
#define ORC_BLOCK_SOLIDA (-2)
#define ORC_BLOCK_SOLID (-3)
/* Voxelizer cell states (inc/mesh.h:88-96) and the near-wall marking
   states (mesh.h:45-46). */
#define ORC_CELL_GUARD (-2)
#define ORC_CELL_LL (-10)
#define ORC_CELL_LR (-11)
#define ORC_CELL_RL (-12)
#define ORC_CELL_RR (-13)
#define ORC_REF_INDET_E 11
#define ORC_REF_INDET_O 12

/* One CSR set of face bins (Bins::binned_face_ids_{n,N,}, geometry_bins.h:66-86). */
typedef struct orc_bins {
    int density, n_bins;
    float sx, sy, sz;   /* bins per unit length along x, y, z (density / L) */
    int64_t n_entries;
    int *n, *N, *ids;
} orc_bins;

struct orc_case {
    agal_params P;
    int fp64;
    int dim, Q, Qmax, MC, NCH;
    int64_t nmb, nmc;
    int max_levels, L0;
    int Nx, Ny, Nz;
    float dx, dx_cblock;
    float dxf[ORC_MAXL];     /* dxf_vec as ufloat_t = float */
    double dxf_d[ORC_MAXL];  /* dxf_vec as ufloat_t = double */
    double tau[ORC_MAXL];    /* tau_vec, rounded to the case's ufloat_t */
    const int *cx, *cy, *cz, *pb, *map;
    const double *w;
    /* mesh arrays, layouts of inc/mesh.h:366-459 */
    int *cells_ID_mask;      /* [nmc] */
    float *cblock_f_X;       /* [dim][nmb] */
    int *cblock_ID_mask;     /* [nmb] */
    int *cblock_ID_nbr;      /* [Qmax][nmb] */
    int *cblock_ID_nbr_child;/* [Qmax][nmb] */
    int *cblock_ID_onb;      /* [nmb] */
    int *cblock_ID_ref;      /* [nmb] */
    int *cblock_level;       /* [nmb] */
    int *id_set;             /* [max_levels][nmb] */
    int *gap_set;            /* [nmb] */
    int n_ids[ORC_MAXL + 1], id_max[ORC_MAXL + 1], n_gaps;
    int geometry_init;
    void *F;                 /* [(Q + dim + 1)][nmc] of float or double */
    int liter;               /* global_Liter of solver_lbm_advance.cu:6 */
    int *emap;               /* [nmb] efficient map of the refinement pass (c_tmp_8), -1 = absent */
    int *first_child;        /* [nmb] scattered first-child IDs (c_tmp_2), -1 = none */
    long iter;               /* coarse steps taken (M_AdvanceLoop counter i) */
    int n_ref_last, n_coarse_last;  /* marks acted on by the last refinement pass */
    /* Geometry (geometry.h, geometry_bins.h; mesh.h:304-307, 491-518). */
    int n_faces;
    float *faces;            /* [9][n_faces]: v1x v1y v1z v2x .. v3z */
    int n_bin_levels, bin_level_md;
    orc_bins bins[ORC_MAXL], bins_md;
    int64_t n_solida, n_maxcells_b;
    int n_solidb;
    int *onb_solid;          /* [nmb] cblock_ID_onb_solid, -1 = none */
    float *X_b;              /* [Qmax][n_maxcells_b] cells_f_X_b, -1 = no link */
    int *tmp_1, *tmp_2;      /* [nmb] c_tmp_1 / c_tmp_2 scratch of the voxelizer */
    int *cells_mask_hi;      /* [nmc] upper half of cells_ID_mask (mesh_init.cu:241) */
    void *Ff;                /* [6][nmb] cblock_f_Ff, ufloat_t */
};

/* orc_geometry.c */
int orc_geometry_alloc(orc_case *c);
void orc_geometry_free(orc_case *c);

static inline int orc_half(int dim, int p)
{
    /* Half set of directions that own a swap pair (kernels.cu:597, 769). */
    if (dim == 2) return p == 1 || (p + 1) % 3 == 0;
    return p == 26 || ((p - 1) % 2 == 0 && p < 25);
}

static inline int orc_nbrslot(int dim, int I, int J, int K)
{
    /* inc/util_index.h:45-66 */
    int S = (I >= 4) ? 2 : (I >= 0 ? 1 : 0);
    S += 3 * ((J >= 4) ? 2 : (J >= 0 ? 1 : 0));
    if (dim == 3) S += 9 * ((K >= 4) ? 2 : (K >= 0 ? 1 : 0));
    return S;
}

static inline int orc_nbrcell(int dim, int I, int J, int K)
{
    /* inc/util_index.h:88-98 */
    I = (4 + (I % 4)) % 4;
    J = (4 + (J % 4)) % 4;
    if (dim == 3) K = (4 + (K % 4)) % 4; else K = 0;
    return I + 4 * J + 16 * K;
}

#endif
