// ORACLE (test infrastructure only): the reference's own time loop driven
// through the drop-in facade include/agal_solver_b200.hpp.
//
// Compiled by oracle/Makefile (targets `_ref/facade_*`) from the AGAL sources
// where they lie, exactly as src/main.cu includes them, plus the facade
// header; linked against the B200 library.  main() is src/main.cu:80-120 with
// the solver lines enabled and Solver_LBM replaced by Solver_B200: Parser ->
// Mesh<..., &agal_b200::AP2D/AP3D> -> Solver_B200 -> M_AddSolver ->
// M_AdvanceLoop (mesh_advance.cu:386-466, the reference's code).  Afterwards
// every mesh array and the populations of the library context are written to
// <dump_prefix>.<array>.bin for comparison with a run of the same input
// through the C ABI.
//
// usage: facade_agal <input_dir/> <dump_prefix|-> <n_maxcblocks> [bc ic region storage]
//   bc, ic, region, storage: AGAL_BC_*, AGAL_IC_*, AGAL_REGION_*, AGAL_STORE_*
//   (-1 storage: from the solution type).
#include "cppspec.h"
#include "parser.h"
#include "geometry.h"
#include "geometry_bins.h"
#include "mesh.h"
#include "solver_lbm.h"

#include "geometry_add.cu"
#include "geometry_bins.cu"
#include "geometry_bins_cpu.cu"
#include "geometry_bins_gpu.cu"
#include "geometry_bins_draw.cu"
#include "geometry_convert.cu"
#include "geometry_dest.cu"
#include "geometry_import.cu"
#include "geometry_init.cu"
#include "geometry_print.cu"
#include "geometry_refine.cu"
#include "mesh_advance.cu"
#include "mesh_amr.cu"
#include "mesh_comm.cu"
#include "mesh_voxelizer.cu"
#include "mesh_criterion.cu"
#include "mesh_dest.cu"
#include "mesh_init.cu"
#include "mesh_output.cu"
#include "mesh_print_uniform.cu"
#include "mesh_restart.cu"
#include "solver_lbm_advance.cu"
#include "solver_lbm_compute_macro.cu"
#include "solver_lbm_compute.cu"
#include "solver_lbm_criterion.cu"
#include "solver_lbm_init.cu"
#include "solver_lbm_kernels.cu"
#include "solver_lbm_kernels_les.cu"
#include "solver_lbm_kernels_comm.cu"
#include "solver_lbm_kernels_forces.cu"
#include "solver_lbm_kernels_debug.cu"

#include "agal_solver_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#if defined(USED2Q9)
constexpr const ArgsPack *APf = &agal_b200::AP2D;
constexpr LBMPack LPf = LBMPack(&agal_b200::AP2D, VelocitySet::D2Q9, CollisionOperator::BGK, InterpOrder::Cubic);
#elif defined(USED3Q19)
constexpr const ArgsPack *APf = &agal_b200::AP3D;
constexpr LBMPack LPf = LBMPack(&agal_b200::AP3D, VelocitySet::D3Q19, CollisionOperator::BGK, InterpOrder::Linear);
#else
constexpr const ArgsPack *APf = &agal_b200::AP3D;
constexpr LBMPack LPf = LBMPack(&agal_b200::AP3D, VelocitySet::D3Q27, CollisionOperator::BGK, InterpOrder::Linear);
#endif
typedef float REAL_f;

// Every array of the context with its selector, in the order the test reads.
static const struct { int which; const char *name; } kArrays[] = {
    {AGAL_ARR_F, "F"},
    {AGAL_ARR_CELLS_ID_MASK, "cells_ID_mask"},
    {AGAL_ARR_CBLOCK_F_X, "cblock_f_X"},
    {AGAL_ARR_CBLOCK_ID_MASK, "cblock_ID_mask"},
    {AGAL_ARR_CBLOCK_ID_NBR, "cblock_ID_nbr"},
    {AGAL_ARR_CBLOCK_ID_NBR_CHILD, "cblock_ID_nbr_child"},
    {AGAL_ARR_CBLOCK_ID_ONB, "cblock_ID_onb"},
    {AGAL_ARR_CBLOCK_ID_REF, "cblock_ID_ref"},
    {AGAL_ARR_CBLOCK_LEVEL, "cblock_level"},
    {AGAL_ARR_ID_SET, "id_set"},
    {AGAL_ARR_GAP_SET, "gap_set"},
};

static int write_file(const std::string &path, const void *data, size_t bytes)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return 1;
    const bool ok = bytes == 0 || std::fwrite(data, 1, bytes, f) == bytes;
    std::fclose(f);
    return ok ? 0 : 1;
}

// The context's counts and every array, one file each.
static int dump_context(agal_ctx *ctx, const std::string &prefix)
{
    int n_ids[64], id_max[64], n_gaps = 0, ml = 0;
    int64_t nmb = 0;
    if (agal_get_counts(ctx, n_ids, id_max, &n_gaps, &nmb, &ml) != AGAL_OK) return 1;
    std::vector<long long> counts;
    counts.push_back(ml);
    counts.push_back(nmb);
    counts.push_back(n_gaps);
    for (int L = 0; L <= ml; L++) counts.push_back(n_ids[L]);
    for (int L = 0; L <= ml; L++) counts.push_back(id_max[L]);
    if (write_file(prefix + ".counts.bin", counts.data(), counts.size() * sizeof(long long))) return 1;
    for (const auto &a : kArrays) {
        size_t bytes = 0;
        if (agal_array_bytes(ctx, a.which, &bytes) != AGAL_OK) return 1;
        std::vector<unsigned char> buf(bytes);
        if (agal_dump(ctx, a.which, buf.data(), bytes) != AGAL_OK) return 1;
        if (write_file(prefix + "." + a.name + ".bin", buf.data(), bytes)) return 1;
    }
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s input_dir/ dump_prefix|- n_maxcblocks [bc ic region storage]\n", argv[0]);
        return 2;
    }
    const std::string input_dir = argv[1], prefix = argv[2];
    agal_b200::Options opt;
    opt.n_maxcblocks = std::atoll(argv[3]);
    if (argc > 4) opt.bc_preset = std::atoi(argv[4]);
    if (argc > 5) opt.ic_preset = std::atoi(argv[5]);
    if (argc > 6) opt.region_preset = std::atoi(argv[6]);
    if (argc > 7) opt.storage = std::atoi(argv[7]);
    try {
        // src/main.cu:88-120 with the solver enabled.
        Parser parser(input_dir);
        const int N_U = LPf.N_Q + APf->N_DIM + 1;
        Mesh<REAL_f, REAL_f, APf> mesh(&parser, N_U);
        Solver_B200<REAL_f, REAL_f, APf, &LPf> solver(&mesh, opt);
        mesh.M_AddSolver(&solver);
        mesh.M_AdvanceLoop();
        if (agal_sync(solver.context()) != AGAL_OK) {
            std::fprintf(stderr, "agal_sync: %s\n", agal_last_error(solver.context()));
            return 4;
        }
        if (prefix != "-" && dump_context(solver.context(), prefix)) {
            std::fprintf(stderr, "dump to %s failed\n", prefix.c_str());
            return 5;
        }
        const double *F = solver.last_force();
        std::printf("{\"facade\": true, \"n_ids0\": %d, \"force\": [%.17g, %.17g, %.17g]}\n", mesh.n_ids[0][0], F[0],
                    F[1], F[2]);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    return 0;
}
