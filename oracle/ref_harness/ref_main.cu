// ORACLE (test infrastructure only): driver for the reference's own CUDA
// build.  Compiled by oracle/Makefile (target `ref`) against the AGAL sources
// where they lie; the binaries go to oracle/_ref/ and run on the GPU box to
// produce golden dumps and the reference's own timing.
//
// It does what the reference's src/main.cu would do with the solver enabled
// (main.cu:108-120 commented lines): Parser -> Mesh(N_U = N_Q + N_DIM + 1) ->
// Solver_LBM -> M_AddSolver, then the loop body of M_AdvanceLoop
// (mesh_advance.cu:381-466) without printing, and writes a binary dump of the
// active blocks.
//
// usage: ref_agal <input_dir/> <dump_file|-> <n_steps> <keep_mb> [n_timed]
//   keep_mb  device memory left free for the reference's own sizing: the
//            rest is taken by a ballast allocation first, because M_Init sizes
//            its pool to 97.5% of free memory (mesh_init.cu:155-169).
//   n_timed  extra steps timed with CUDA events after the dump (MLUPS line).
#include "ref_hooks.h"

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

#include <cstdint>
#include <cstdio>
#include <set>
#include <vector>

// VTK writers are not built (VTK is absent); these stubs replace
// mesh_print_vthb.cu, mesh_print_vthb_patch.cu and mesh_print_image.cu.
template <typename ufloat_t, typename ufloat_g_t, const ArgsPack *AP>
int Mesh<ufloat_t, ufloat_g_t, AP>::M_Print_VTHB(int, int) { return 0; }
template <typename ufloat_t, typename ufloat_g_t, const ArgsPack *AP>
int Mesh<ufloat_t, ufloat_g_t, AP>::M_Print_VTHB_Patch(int, int) { return 0; }
template <typename ufloat_t, typename ufloat_g_t, const ArgsPack *AP>
int Mesh<ufloat_t, ufloat_g_t, AP>::M_Print_ImageData(int, int) { return 0; }

// Argument packs as in main.cu:48-57.
constexpr ArgsPack AP2D_H = ArgsPack(2, 128, 1, 1, 1, 24, 2048);
constexpr ArgsPack AP3D_H = ArgsPack(3, 128, 1, 1, 1, 24, 2048);
#ifndef REF_INTERP2D
#define REF_INTERP2D InterpOrder::Cubic
#endif
#ifndef REF_INTERP3D
#define REF_INTERP3D InterpOrder::Linear
#endif
#ifndef REF_LES
#define REF_LES LESModel::None
#endif
#if defined(USED2Q9)
constexpr ArgsPack APh = AP2D_H;
constexpr LBMPack LPh = LBMPack(&AP2D_H, VelocitySet::D2Q9, CollisionOperator::BGK, REF_INTERP2D, REF_LES);
#elif defined(USED3Q19)
constexpr ArgsPack APh = AP3D_H;
constexpr LBMPack LPh = LBMPack(&AP3D_H, VelocitySet::D3Q19, CollisionOperator::BGK, REF_INTERP3D, REF_LES);
#else
constexpr ArgsPack APh = AP3D_H;
constexpr LBMPack LPh = LBMPack(&AP3D_H, VelocitySet::D3Q27, CollisionOperator::BGK, REF_INTERP3D, REF_LES);
#endif
typedef float REAL_h;

template <typename T>
static void put(FILE *f, const T *p, size_t n) { fwrite(p, sizeof(T), n, f); }

template <typename T>
static std::vector<T> d2h(const T *d, size_t n)
{
    std::vector<T> h(n);
    if (n) cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost);
    return h;
}

// Gather rows [r][blk*width .. +width) of an SoA array for the listed blocks:
// out[(i*rows + r)*width + k] = in[r*stride + blk[i]*width + k].
template <typename T>
__global__ void k_gather(const T *in, long long stride, int rows, int width, const int *blk, int n, T *out)
{
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)n * rows * width;
    if (g >= tot) return;
    int k = (int)(g % width);
    long long t = g / width;
    int r = (int)(t % rows);
    int i = (int)(t / rows);
    out[g] = in[(long long)r * stride + (long long)blk[i] * width + k];
}

template <typename T>
static std::vector<T> gather(const T *d_in, long long stride, int rows, int width, const int *d_blk, int n)
{
    const size_t tot = (size_t)n * rows * width;
    T *d_out = nullptr;
    std::vector<T> h(tot);
    if (!tot) return h;
    cudaMalloc(&d_out, tot * sizeof(T));
    k_gather<T><<<(unsigned)((tot + 255) / 256), 256>>>(d_in, stride, rows, width, d_blk, n, d_out);
    cudaMemcpy(h.data(), d_out, tot * sizeof(T), cudaMemcpyDeviceToHost);
    cudaFree(d_out);
    return h;
}

int main(int argc, char **argv)
{
    if (argc < 5) {
        fprintf(stderr, "usage: %s input_dir/ dump_file|- n_steps keep_mb [n_timed]\n", argv[0]);
        return 2;
    }
    const std::string input_dir = argv[1];
    const std::string dump_file = argv[2];
    const int n_steps = atoi(argv[3]);
    const long long keep_mb = atoll(argv[4]);
    const int n_timed = argc > 5 ? atoi(argv[5]) : 0;

    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    void *ballast = nullptr;
    const size_t keep = (size_t)keep_mb << 20;
    if (fr > keep + (256ull << 20)) {
        if (cudaMalloc(&ballast, fr - keep) != cudaSuccess) { fprintf(stderr, "ballast failed\n"); return 3; }
    }

    if (const char *rg = getenv("REF_REGION")) {
        const int v = atoi(rg);
        cudaMemcpyToSymbol(g_ref_region, &v, sizeof(int));
    }

    Parser parser(input_dir);
    // REF_GEOM=1: import the STL named by G_FILENAME and bin it as main.cu:94-106
    // does, then attach it to the mesh (mesh_init.cu:570-577).
    const bool geom = getenv("REF_GEOM") && atoi(getenv("REF_GEOM")) == 1;
    Geometry<REAL_h, REAL_h, &APh> *geometry = nullptr;
    if (geom) {
        geometry = new Geometry<REAL_h, REAL_h, &APh>(&parser);
        // main.cu:95-101: STL, or the primitives of geometry.txt
        if (geometry->G_LOADTYPE == static_cast<int>(LoadType::STL)) {
            geometry->G_ImportSTL_ASCII(geometry->G_FILENAME);
        } else {
            geometry->G_ImportBoundariesFromTextFile();
            geometry->G_Convert_IndexListsToCoordList();
        }
        geometry->G_Init_Arrays_CoordsList_CPU();
        geometry->G_InitBins(BinMake::GPU, 0);
    }
    // With an LES model the field also holds the eddy viscosity, which the
    // kernels write to row N_Q + 4 in 2D and 3D alike
    // (solver_lbm_kernels_les.cu:450, 597).  main.cu:109's commented size,
    // N_Q + N_DIM + 2, ends one row short of it in 2D, so the field is sized
    // N_Q + 5 whenever a model is on.
    const int N_U = (LPh.LM != LESModel::None) ? LPh.N_Q + 5 : LPh.N_Q + APh.N_DIM + 1;
    Mesh<REAL_h, REAL_h, &APh> mesh(&parser, N_U);
    if (geom) mesh.M_AddGeometry(geometry);
    Solver_LBM<REAL_h, REAL_h, &APh, &LPh> solver(&mesh);
    mesh.M_AddSolver(&solver);
    for (int L = 0; L < mesh.MAX_LEVELS; L++) solver.S_SetIC(0, L);
    cudaDeviceSynchronize();

    // Loop body of M_AdvanceLoop (mesh_advance.cu:403-463) without output.
    const int iter_mult = (int)pow(2.0, (double)mesh.N_LEVEL_START);
    // With a geometry the near-wall pass also voxelizes a uniform grid
    // (M_AdvanceLoop calls it unconditionally, mesh_advance.cu:395).
    if (mesh.MAX_LEVELS > 1 || geom) mesh.M_Advance_RefineNearWall();
    if (geom && n_steps > 0 && mesh.n_solidb > 0) {
        // The wall kernels read the populations of the cell behind a
        // boundary cell without checking that its block exists
        // (solver_lbm_kernels.cu:808-815, 859-866; forces.cu:428-436).
        // Refuse to step a case where any boundary cell of a wall block has
        // a missing neighbour block along a lattice direction.
        const long long nmb = mesh.n_maxcblocks;
        const int dim = APh.N_DIM, Q = LPh.N_Q, MC = APh.M_CBLOCK, Qmax = APh.N_Q_max;
        auto onb = d2h(mesh.c_cblock_ID_onb[0], (size_t)nmb);
        auto onbs = d2h(mesh.c_cblock_ID_onb_solid[0], (size_t)nmb);
        auto nbr = d2h(mesh.c_cblock_ID_nbr[0], (size_t)nmb * Qmax);
        auto cm = d2h(mesh.c_cells_ID_mask[0], (size_t)mesh.n_maxcells);
        long long bad = 0;
        for (int L = 0; L < mesh.MAX_LEVELS; L++) {
            auto ids = d2h(&mesh.c_id_set[0][(size_t)L * nmb], mesh.n_ids[0][L]);
            for (int b : ids) {
                if (onb[b] != 1 || onbs[b] < 0) continue;
                for (int t = 0; t < MC; t++) {
                    if (cm[(size_t)b * MC + t] != -6) continue;
                    const int I = t % 4, J = (t / 4) % 4, K = dim == 3 ? t / 16 : 0;
                    for (int p = 1; p < Q; p++) {
                        const int Ip = I + V_CONN_ID_H[p], Jp = J + V_CONN_ID_H[p + 27];
                        const int Kp = dim == 3 ? K + V_CONN_ID_H[p + 54] : 0;
                        const int bx = Ip < 0 ? 0 : (Ip < 4 ? 1 : 2), by = Jp < 0 ? 0 : (Jp < 4 ? 1 : 2);
                        const int bz = dim == 3 ? (Kp < 0 ? 0 : (Kp < 4 ? 1 : 2)) : 0;
                        const int S = bx + 3 * by + 9 * bz;
                        if (nbr[(size_t)b + (size_t)V_CONN_MAP_H[S] * nmb] < 0) bad++;
                    }
                }
            }
        }
        if (bad) {
            fprintf(stderr, "geometry guard: %lld boundary-cell links without a neighbour block\n", bad);
            return 6;
        }
    }
    // REF_SKIP_LAST_REGRID=1 stops before the refinement of the last step, so
    // the dump is the input of that refinement.
    const bool skip_last = getenv("REF_SKIP_LAST_REGRID") && atoi(getenv("REF_SKIP_LAST_REGRID")) == 1;
    for (int i = 0; i < n_steps; i++) {
        mesh.M_Advance_Step(i, 0, iter_mult);
        if (skip_last && i == n_steps - 1) break;
        if (mesh.MAX_LEVELS > 1 && (mesh.MAX_LEVELS != mesh.N_LEVEL_START + 1) && (i + 1) % mesh.P_REFINE == 0 && i > 0)
            mesh.M_Advance_RefineWithSolution(i, 0);
    }
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) { fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(err)); return 4; }
    // REF_UNIFORM=1: one frame of the reference's uniform-grid output
    // (M_Advance_PrintData, mesh_advance.cu:296-334: grid average, interface
    // interpolation, refresh, M_RetrieveFromGPU, M_RenderAndPrint_Uniform)
    // appended to <P_DIR_NAME>out_direct.dat, whose header M_Init wrote.
    if (getenv("REF_UNIFORM") && atoi(getenv("REF_UNIFORM")) == 1) {
        if (mesh.MAX_LEVELS > 1) {
            for (int L = mesh.MAX_LEVELS - 2; L >= 0; L--) solver.S_Average(0, L, V_AVERAGE_GRID);
            for (int L = 0; L < mesh.MAX_LEVELS - 1; L++) solver.S_Interpolate(0, L, V_INTERP_INTERFACE);
        }
        for (int L = 0; L < mesh.MAX_LEVELS; L++) solver.S_RefreshVariables(0, L);
        cudaDeviceSynchronize();
        mesh.M_RetrieveFromGPU();
        mesh.M_RenderAndPrint_Uniform(0, n_steps);
        mesh.output_file_direct->flush();
    }
    // REF_RESTART=1: the reference's own checkpoint of this state
    // (M_RetrieveFromGPU, then M_Restart SAVE as at the end of M_AdvanceLoop,
    // mesh_advance.cu:316-324) into <P_DIR_NAME>restart.bin.
    if (getenv("REF_RESTART") && atoi(getenv("REF_RESTART")) == 1) {
        mesh.M_RetrieveFromGPU();
        int it = n_steps - 1;
        mesh.M_Restart(0, V_MESH_RESTART_SAVE, &it);
    }

    if (dump_file != "-") {
        const int dim = APh.N_DIM, Q = LPh.N_Q, Qmax = APh.N_Q_max, MC = APh.M_CBLOCK, ML = mesh.MAX_LEVELS;
        const long long nmb = mesh.n_maxcblocks, nmc = mesh.n_maxcells;
        FILE *f = fopen(dump_file.c_str(), "wb");
        if (!f) { fprintf(stderr, "cannot open %s\n", dump_file.c_str()); return 5; }
        fwrite("AGALREF1", 1, 8, f);
        int hdr[6] = {dim, Q, Qmax, MC, ML, n_steps};
        put(f, hdr, 6);
        long long hdr2[2] = {nmb, nmc};
        put(f, hdr2, 2);
        put(f, mesh.n_ids[0], ML + 1);
        put(f, mesh.id_max[0], ML + 1);
        put(f, &mesh.n_gaps[0], 1);
        std::set<int> act;
        for (int L = 0; L < ML; L++) {
            auto ids = d2h(&mesh.c_id_set[0][(size_t)L * nmb], mesh.n_ids[0][L]);
            put(f, ids.data(), ids.size());
            act.insert(ids.begin(), ids.end());
        }
        const int n_gap_keep = std::min(mesh.n_gaps[0], 65536);
        auto gaps = d2h(&mesh.c_gap_set[0][mesh.n_gaps[0] - n_gap_keep], n_gap_keep);
        put(f, &n_gap_keep, 1);
        put(f, gaps.data(), gaps.size());
        std::vector<int> blk(act.begin(), act.end());
        const int n_act = (int)blk.size();
        put(f, &n_act, 1);
        put(f, blk.data(), blk.size());
        // Only the active blocks travel to the host (the pool spans GBs).
        int *d_blk = nullptr;
        cudaMalloc(&d_blk, sizeof(int) * std::max(n_act, 1));
        if (n_act) cudaMemcpy(d_blk, blk.data(), sizeof(int) * n_act, cudaMemcpyHostToDevice);
        auto fX = gather(mesh.c_cblock_f_X[0], nmb, dim, 1, d_blk, n_act);
        auto bm = gather(mesh.c_cblock_ID_mask[0], nmb, 1, 1, d_blk, n_act);
        auto nb = gather(mesh.c_cblock_ID_nbr[0], nmb, Qmax, 1, d_blk, n_act);
        auto nc = gather(mesh.c_cblock_ID_nbr_child[0], nmb, Qmax, 1, d_blk, n_act);
        auto onb = gather(mesh.c_cblock_ID_onb[0], nmb, 1, 1, d_blk, n_act);
        auto ref = gather(mesh.c_cblock_ID_ref[0], nmb, 1, 1, d_blk, n_act);
        auto lev = gather(mesh.c_cblock_level[0], nmb, 1, 1, d_blk, n_act);
        auto cm = gather(mesh.c_cells_ID_mask[0], nmc, 1, MC, d_blk, n_act);
        auto F = gather(mesh.c_cells_f_F[0], nmc, N_U, MC, d_blk, n_act);
        std::vector<int> onb_s;
        std::vector<REAL_h> Ff;
        if (geom) {
            if (mesh.n_solidb > 0) onb_s = gather(mesh.c_cblock_ID_onb_solid[0], nmb, 1, 1, d_blk, n_act);
            Ff = gather(mesh.c_cblock_f_Ff[0], nmb, 6, 1, d_blk, n_act);
        }
        cudaFree(d_blk);
        for (int i = 0; i < n_act; i++) {
            put(f, &fX[(size_t)i * dim], dim);
            put(f, &bm[i], 1);
            put(f, &nb[(size_t)i * Qmax], Qmax);
            put(f, &nc[(size_t)i * Qmax], Qmax);
            put(f, &onb[i], 1);
            put(f, &ref[i], 1);
            put(f, &lev[i], 1);
            put(f, &cm[(size_t)i * MC], MC);
            put(f, &F[(size_t)i * N_U * MC], (size_t)N_U * MC);
        }
        if (geom) {
            // Geometry section: faces after import/refinement (SoA rows 0..8 of
            // geom_f_face_X), the 3D bins of every bin level and the link
            // bins (CSR: count, start, ids), the solid-boundary counts and
            // map, the link lengths and the per-block MEA force partials.
            fwrite("GEOM", 1, 4, f);
            const long long nf = geometry->n_faces, nfa = geometry->n_faces_a;
            put(f, &nf, 1);
            for (int r = 0; r < 9; r++) put(f, &geometry->geom_f_face_X[(size_t)r * nfa], (size_t)nf);
            auto *bins = geometry->bins;
            const int nbl = bins->n_bin_levels;
            put(f, &nbl, 1);
            for (int L = 0; L < nbl; L++) {
                const int dens = bins->n_bin_density[L], nb = bins->n_bins_3D[L];
                long long ne = 0;
                for (int k = 0; k < nb; k++) ne += bins->binned_face_ids_n_3D[L][k];
                put(f, &dens, 1);
                put(f, &nb, 1);
                put(f, &ne, 1);
                put(f, bins->binned_face_ids_n_3D[L], nb);
                put(f, bins->binned_face_ids_N_3D[L], nb);
                put(f, bins->binned_face_ids_3D[L], (size_t)ne);
            }
            const int mk = bins->make_links;
            put(f, &mk, 1);
            if (mk) {
                const int lmd = bins->n_bin_level_MD, dens = bins->n_bin_density_MD, nb = bins->n_bins_MD;
                long long ne = 0;
                for (int k = 0; k < nb; k++) ne += bins->binned_face_ids_n_MD[k];
                put(f, &lmd, 1);
                put(f, &dens, 1);
                put(f, &nb, 1);
                put(f, &ne, 1);
                put(f, bins->binned_face_ids_n_MD, nb);
                put(f, bins->binned_face_ids_N_MD, nb);
                put(f, bins->binned_face_ids_MD, (size_t)ne);
            }
            const long long sa = mesh.n_solida, sb = mesh.n_solidb, mcb = mesh.n_maxcells_b;
            put(f, &sa, 1);
            put(f, &sb, 1);
            put(f, &mcb, 1);
            if (sb > 0) put(f, onb_s.data(), onb_s.size());
            long long nxb = (sb > 0 && mk) ? mcb * Qmax : 0;
            put(f, &nxb, 1);
            if (nxb) {
                auto xb = d2h(mesh.c_cells_f_X_b[0], (size_t)nxb);
                put(f, xb.data(), xb.size());
            }
            put(f, Ff.data(), Ff.size());
        }
        fclose(f);
    }

    if (n_timed > 0) {
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, mesh.streams[0]);
        for (int i = 0; i < n_timed; i++) mesh.M_Advance_Step(n_steps + i, 0, iter_mult);
        cudaEventRecord(e1, mesh.streams[0]);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        // Cell updates per coarse step as solver_lbm_advance.cu:74-89 counts them.
        long long cells = 0;
        int mult = 1;
        for (int L = mesh.N_LEVEL_START; L < mesh.MAX_LEVELS - 1; L++) {
            cells += (long long)mult * (mesh.n_ids[0][L] - mesh.n_ids[0][L + 1] / APh.N_CHILDREN);
            mult *= 2;
        }
        cells += (long long)mult * mesh.n_ids[0][mesh.MAX_LEVELS - 1];
        cells *= APh.M_CBLOCK;
        const double mlups = (double)cells * n_timed / (ms * 1e-3) / 1e6;
        printf("{\"ref_timing\": true, \"steps\": %d, \"ms\": %.4f, \"cell_updates_per_step\": %lld, \"mlups\": %.3f}\n",
               n_timed, ms, cells, mlups);
    }
    if (ballast) cudaFree(ballast);
    return 0;
}
