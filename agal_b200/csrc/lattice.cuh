// Lattice tables and block-local index maths for the device kernels.
//
// The direction order, opposite map and weights must be those of the
// reference (inc/util.h:94-101, solver_lbm_init.cu:79-91): they define the slot
// convention of the population arrays that callers read and write.  All
// functions are constexpr so that, inside fully unrolled loops over p, every
// table lookup folds to an immediate.
#pragma once

#include <cstdint>

namespace agal {

constexpr int N_SKIPID = -999;   // cppspec.h:125
constexpr int N_SPECID = -998;   // cppspec.h:124

// Reference enumerations (inc/mesh.h:34-105).
constexpr int REF_UNREFINED = 0, REF_REFINED = 1, REF_REFINED_WCHILD = 2, REF_REFINED_PERM = 3,
              REF_MARK_REFINE = 4, REF_MARK_COARSEN = 5, REF_NEW = 6, REF_REMOVE = 7,
              REF_INACTIVE = 8, REF_UNREFINED_VIO = 9, REF_REFINED_WCHILD_PERM = 10,
              REF_INDET_E = 11, REF_INDET_O = 12;
constexpr int CELL_INTERIOR = 0, CELL_INTERFACE = 1, CELL_GHOST = 2, CELL_SOLID = -1,
              CELL_GUARD = -2, CELL_BOUNDARY = -6;
constexpr int BLOCK_REGULAR = 0, BLOCK_INTERFACE = 1, BLOCK_SOLIDB = -1, BLOCK_SOLIDA = -2,
              BLOCK_SOLID = -3;

template <int DIM> struct Geo;
template <> struct Geo<2> { static constexpr int MC = 16, QMAX = 9, NCH = 4; };
template <> struct Geo<3> { static constexpr int MC = 64, QMAX = 27, NCH = 8; };

// The tables are packed into integer constants: a lookup at an index that is
// not known at compile time is then a shift and a mask in registers instead
// of a table built in local memory on every call.
namespace lat_tab {
constexpr int c2[3][9] = {{0, 1, 0, -1, 0, 1, -1, -1, 1},
                          {0, 0, 1, 0, -1, 1, 1, -1, -1},
                          {0, 0, 0, 0, 0, 0, 0, 0, 0}};
constexpr int c3[3][27] = {
    {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1},
    {0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1},
    {0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1}};
constexpr int m2[9] = {7, 4, 8, 3, 0, 1, 6, 2, 5};
constexpr int m3[27] = {20, 12, 26, 10, 6, 15, 24, 17, 21, 8, 4, 13, 2, 0,
                        1, 14, 3, 7, 22, 18, 23, 16, 5, 9, 25, 11, 19};
// c + 1 in 2 bits per direction
template <int N> constexpr unsigned long long pack_c(const int (&c)[N])
{
    unsigned long long w = 0;
    for (int p = 0; p < N; p++) w |= (unsigned long long)(c[p] + 1) << (2 * p);
    return w;
}
// 5 bits per entry, entries [lo, lo + 9)
template <int N> constexpr unsigned long long pack_m(const int (&m)[N], int lo)
{
    unsigned long long w = 0;
    for (int i = lo; i < lo + 9 && i < N; i++) w |= (unsigned long long)m[i] << (5 * (i - lo));
    return w;
}
constexpr unsigned long long C2X = pack_c(c2[0]), C2Y = pack_c(c2[1]), C2Z = pack_c(c2[2]);
constexpr unsigned long long C3X = pack_c(c3[0]), C3Y = pack_c(c3[1]), C3Z = pack_c(c3[2]);
constexpr unsigned long long M2 = pack_m(m2, 0), M3A = pack_m(m3, 0), M3B = pack_m(m3, 9), M3C = pack_m(m3, 18);
}  // namespace lat_tab

__host__ __device__ constexpr int lat_c(int dim, int axis, int p)
{
    const unsigned long long w = dim == 2 ? (axis == 0 ? lat_tab::C2X : axis == 1 ? lat_tab::C2Y : lat_tab::C2Z)
                                          : (axis == 0 ? lat_tab::C3X : axis == 1 ? lat_tab::C3Y : lat_tab::C3Z);
    return (int)((w >> (2 * p)) & 3ull) - 1;
}

// Opposite direction: D2Q9 pairs {1,3}, {2,4}, {5,7}, {6,8}; D3Q19/D3Q27
// pairs {2k-1, 2k}.
__host__ __device__ constexpr int lat_pb(int dim, int p)
{
    return p == 0 ? 0
         : dim == 2 ? (p < 5 ? ((p + 1) & 3) + 1 : ((p - 3) & 3) + 5)
                    : ((p & 1) ? p + 1 : p - 1);
}

// Weights: D2Q9 4/9,1/9,1/36; D3Q19 1/3,1/18,1/36; D3Q27 8/27,2/27,1/54,1/216.
__host__ __device__ constexpr double lat_w(int Q, int p)
{
    return Q == 9 ? (p == 0 ? 4.0 / 9.0 : (p < 5 ? 1.0 / 9.0 : 1.0 / 36.0))
         : Q == 19 ? (p == 0 ? 1.0 / 3.0 : (p < 7 ? 1.0 / 18.0 : 1.0 / 36.0))
         : (p == 0 ? 8.0 / 27.0 : (p < 7 ? 2.0 / 27.0 : (p < 19 ? 1.0 / 54.0 : 1.0 / 216.0)));
}

// Neighbour-array index of the lexicographic neighbour slot S (util.h:100-101).
__host__ __device__ constexpr int lat_map(int dim, int S)
{
    const unsigned long long w = dim == 2 ? lat_tab::M2 : (S < 9 ? lat_tab::M3A : S < 18 ? lat_tab::M3B : lat_tab::M3C);
    return (int)((w >> (5 * (dim == 2 ? S : S % 9))) & 31ull);
}

// Lexicographic neighbour slot of a cell index in {-1..4}^dim (util_index.h:45-66).
__host__ __device__ constexpr int nbr_slot(int dim, int I, int J, int K)
{
    return ((I >= 4) ? 2 : (I >= 0 ? 1 : 0)) + 3 * ((J >= 4) ? 2 : (J >= 0 ? 1 : 0)) +
           (dim == 3 ? 9 * ((K >= 4) ? 2 : (K >= 0 ? 1 : 0)) : 0);
}
// Cell id after wrapping into the neighbour block (util_index.h:88-98).
__host__ __device__ constexpr int nbr_cell(int dim, int I, int J, int K)
{
    return ((I + 4) & 3) + 4 * ((J + 4) & 3) + (dim == 3 ? 16 * ((K + 4) & 3) : 0);
}
__host__ __device__ constexpr int center_slot(int dim) { return dim == 2 ? 4 : 13; }

// Directions that own a swap pair in the in-place stream (kernels.cu:597, 769):
// the stream visits p in this half set and swaps with pb(p) of the neighbour.
__host__ __device__ constexpr bool lat_half(int dim, int p)
{
    return dim == 2 ? (p == 1 || (p + 1) % 3 == 0) : (p == 26 || ((p - 1) % 2 == 0 && p < 25));
}

// The packed forms agree with the tables (checked at compile time).
namespace lat_tab {
constexpr bool check()
{
    constexpr int pb2[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    constexpr int pb3[27] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13,
                             16, 15, 18, 17, 20, 19, 22, 21, 24, 23, 26, 25};
    for (int a = 0; a < 3; a++) {
        for (int p = 0; p < 9; p++)
            if (lat_c(2, a, p) != c2[a][p]) return false;
        for (int p = 0; p < 27; p++)
            if (lat_c(3, a, p) != c3[a][p]) return false;
    }
    for (int p = 0; p < 9; p++)
        if (lat_pb(2, p) != pb2[p] || lat_map(2, p) != m2[p]) return false;
    for (int p = 0; p < 27; p++)
        if (lat_pb(3, p) != pb3[p] || lat_map(3, p) != m3[p]) return false;
    return true;
}
static_assert(check(), "packed lattice tables");
}  // namespace lat_tab

}  // namespace agal
