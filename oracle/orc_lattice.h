/*
 * ORACLE (test infrastructure only): lattice tables restated from AGAL.
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline; never by
 * the product path.
 *
 * Direction order, opposite map and weights follow
 *   inc/util.h:94-101            (V_CONN_ID_2D/3D, V_CONN_ID_PB, V_CONN_MAP)
 *   src/solver_lbm/solver_lbm_init.cu:79-91 (LBMw, LBMpb)
 * D3Q19 is the first 19 directions of the D3Q27 order.
 */
#ifndef ORC_LATTICE_H
#define ORC_LATTICE_H

static const int ORC_C2[3][9] = {
    {0, 1, 0, -1, 0, 1, -1, -1, 1},
    {0, 0, 1, 0, -1, 1, 1, -1, -1},
    {0, 0, 0, 0, 0, 0, 0, 0, 0}};
static const int ORC_PB2[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const double ORC_W2[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                                 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};

static const int ORC_C3[3][27] = {
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1},
    {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1}};
static const int ORC_PB3[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13,
                                16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
static const double ORC_W19[19] = {1.0 / 3.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                                   1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                   1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                   1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
static const double ORC_W27[27] = {8.0 / 27.0, 2.0 / 27.0, 2.0 / 27.0, 2.0 / 27.0, 2.0 / 27.0,
                                   2.0 / 27.0, 2.0 / 27.0, 1.0 / 54.0, 1.0 / 54.0, 1.0 / 54.0,
                                   1.0 / 54.0, 1.0 / 54.0, 1.0 / 54.0, 1.0 / 54.0, 1.0 / 54.0,
                                   1.0 / 54.0, 1.0 / 54.0, 1.0 / 54.0, 1.0 / 54.0, 1.0 / 216.0,
                                   1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0, 1.0 / 216.0,
                                   1.0 / 216.0, 1.0 / 216.0};

/* Neighbour-slot map: lexicographic slot S = sx + 3 sy (+ 9 sz), s = 0 for
   index -1, 1 inside [0,4), 2 for 4 -> index into the block-neighbour array
   (inc/util.h:100-101 V_CONN_MAP, inc/util_index.h:45-66 Cu_NbrMap). */
static const int ORC_MAP2[9] = {7, 4, 8, 3, 0, 1, 6, 2, 5};
static const int ORC_MAP3[27] = {20, 12, 26, 10, 6, 15, 24, 17, 21, 8, 4, 13, 2, 0,
                                 1, 14, 3, 7, 22, 18, 23, 16, 5, 9, 25, 11, 19};

#endif
