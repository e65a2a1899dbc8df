/*
 * agal_solver_b200.hpp - drop-in solver and mesh adaptor that run the AGAL
 * time loop on the B200 library (libagal_b200.so, C ABI in agal_b200.h).
 *
 * The AGAL driver builds a Mesh, attaches a Solver_LBM and calls
 * Mesh::M_AdvanceLoop (src/main.cu:108-120, mesh_advance.cu:386-466).  This
 * header supplies the two pieces that let that unchanged loop drive the
 * library instead:
 *
 *   Solver_B200<ufloat_t, ufloat_g_t, AP, LP>
 *       a subclass of the reference's abstract Solver (inc/solver.h:20-90)
 *       with the template signature of Solver_LBM (inc/solver_lbm.h:82).  It
 *       owns one library context, built from the Parser's maps and the
 *       LBMPack, and maps every S_* virtual to the C entry point of the same
 *       routine.
 *
 *   the mesh adaptor
 *       explicit specialisations of the Mesh members that own device data
 *       (M_Init, M_RefineAndCoarsenBlocks, M_ComputeRefCriteria, the
 *       voxelizer passes, M_Restart, the printers ...) for the argument packs
 *       agal_b200::AP2D and agal_b200::AP3D.  A Mesh of those packs allocates
 *       no block pool of its own: the context holds the mesh, and the
 *       reference's own M_AdvanceLoop, M_Advance_Step,
 *       M_Advance_RefineNearWall, M_Advance_RefineWithSolution and
 *       M_Advance_PrintData run unchanged on top of it.
 *
 * Use: include after the AGAL headers and sources (the #include list of
 * src/main.cu), then, in main():
 *
 *     constexpr LBMPack LP = LBMPack(&agal_b200::AP2D, VelocitySet::D2Q9,
 *                                    CollisionOperator::BGK, InterpOrder::Cubic);
 *     Parser parser("../input/");
 *     Mesh<float, float, &agal_b200::AP2D> mesh(&parser, LP.N_Q + 3);
 *     agal_b200::Options opt;
 *     opt.bc_preset = AGAL_BC_LDC2D;              // the custom.h hooks in use
 *     Solver_B200<float, float, &agal_b200::AP2D, &LP> solver(&mesh, opt);
 *     mesh.M_AddSolver(&solver);
 *     mesh.M_AdvanceLoop();
 *
 * The Cu_ImposeBC / Cu_ComputeIC / Cu_RefineRegion device hooks of
 * inc/custom.h are not compiled into the library; Options selects the
 * library's presets of them.  Errors of the library throw
 * std::runtime_error with the context's error text (the reference exits on
 * CUDA errors through gpuErrchk).  Other argument packs can be adapted with
 * AGAL_B200_MESH_ADAPTOR(ufloat_t, ufloat_g_t, &pack).
 */
#ifndef AGAL_SOLVER_B200_HPP
#define AGAL_SOLVER_B200_HPP

#include <sys/stat.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "agal_b200.h"

namespace agal_b200 {

// Argument packs of the adapted meshes (the values of AP2D_DEF / AP3D_DEF,
// cppspec.h:119-120).
inline constexpr ArgsPack AP2D = ArgsPack(2);
inline constexpr ArgsPack AP3D = ArgsPack(3);

// Selections the reference makes by editing inc/custom.h or by the solution
// type, and the library's own capacity and precision controls.
struct Options {
    int bc_preset = AGAL_BC_NONE;          // Cu_ImposeBC preset
    int ic_preset = AGAL_IC_REST;          // Cu_ComputeIC preset
    int region_preset = AGAL_REGION_NONE;  // Cu_RefineRegion preset
    double u_ref = 0.05;                   // preset velocity (custom.h hard-codes 0.05)
    int storage = -1;                      // AGAL_STORE_*; -1: FP32 for float, FP64 for double
    int half_rounding = AGAL_ROUND_STOCHASTIC;
    int64_t n_maxcblocks = 0;              // 0: sized from free memory with mem_frac
    double mem_frac = 0.975;               // M_FRAC of mesh.h
    int device = -1;                       // -1: the current device
    int step_variant = 0;                  // 0: library default, 1..5: agal_set_tuning
};

inline void check(const agal_ctx *ctx, int rc, const char *what)
{
    if (rc == AGAL_OK) return;
    const char *e = agal_last_error(ctx);
    throw std::runtime_error(std::string("agal_b200: ") + what + " failed (" + std::to_string(rc) +
                             "): " + (e ? e : ""));
}

// agal_params from the Parser's maps (parser.h:62-144): every key the parser
// holds, as text, through the library's own key table.
inline agal_params params_from_parser(Parser &parser)
{
    agal_params p;
    agal_params_default(&p);
    char buf[64];
    auto set = [&](const std::string &k, const char *v) {
        const int rc = agal_params_set(&p, k.c_str(), v);
        if (rc != AGAL_OK && rc != AGAL_ERR_UNSUPPORTED)
            throw std::runtime_error("agal_b200: parameter " + k + " = " + v + " rejected");
    };
    for (const auto &kv : parser.params_int) {
        std::snprintf(buf, sizeof buf, "%d", kv.second);
        set(kv.first, buf);
    }
    for (const auto &kv : parser.params_dbl) {
        std::snprintf(buf, sizeof buf, "%.17g", kv.second);
        set(kv.first, buf);
    }
    for (const auto &kv : parser.params_str) set(kv.first, kv.second.c_str());
    return p;
}

// Implemented by Solver_B200; the mesh adaptor finds the context through it.
class ContextOwner {
  public:
    virtual ~ContextOwner() = default;
    agal_ctx *context() const { return ctx_; }
    // Called by M_RetrieveFromGPU: host copies of device data are out of date.
    virtual void host_copies_stale() {}

  protected:
    agal_ctx *ctx_ = nullptr;
};

// Host mirrors of the mesh counts (n_ids, id_max, n_gaps, capacity), which
// the reference's loop prints and its force report reads.
template <class MeshT>
void mirror_counts(MeshT &m, agal_ctx *ctx)
{
    int64_t nmb = 0;
    int ml = 0;
    check(ctx, agal_get_counts(ctx, m.n_ids[0], m.id_max[0], &m.n_gaps[0], &nmb, &ml), "agal_get_counts");
    m.n_maxcblocks = (long int)nmb;
    m.n_maxcells = (long int)nmb * m.M_CBLOCK;
}

template <class MeshT>
struct MeshAdaptor {
    static agal_ctx *ctx(MeshT &m)
    {
        ContextOwner *o = m.solver ? dynamic_cast<ContextOwner *>(m.solver) : nullptr;
        if (!o || !o->context())
            throw std::runtime_error("agal_b200: a mesh of the B200 argument packs needs a Solver_B200");
        return o->context();
    }

    // Mesh::M_Init (mesh_init.cu:11-567) without the block pool: the
    // parameters the loop reads, the level spacings, the count mirrors and
    // the output directory.  The context (created by the solver) holds the
    // mesh itself.
    static int init(MeshT &m)
    {
        m.solver = nullptr;
        m.geometry = nullptr;
        const agal_params p = params_from_parser(*m.parser);
        m.Lx = (float)p.L_c;
        m.Ly = (float)(p.L_fy * p.L_c);
        m.Lz = (float)(p.L_fz * p.L_c);
        m.Nx = p.Nx;
        m.Ny = (int)(m.Nx * (m.Ly / m.Lx));
        m.Nz = m.N_DIM == 2 ? 1 : (int)(m.Nx * (m.Lz / m.Lx));
        m.Nxi = new int[3]{m.Nx, m.Ny, m.Nz};
        m.dx = m.Lx / m.Nx;
        m.dx_cblock = 4 * m.Nqx * m.dx;
        m.MAX_LEVELS_WALL = p.MAX_LEVELS_WALL;
        m.MAX_LEVELS_INTERIOR = p.MAX_LEVELS_INTERIOR;
        m.N_ITER_TOTAL = p.N_ITER_TOTAL;
        m.N_LEVEL_START = p.N_LEVEL_START;
        m.N_RESTART = p.N_RESTART;
        m.PERIODIC_X = p.PERIODIC_X;
        m.PERIODIC_Y = p.PERIODIC_Y;
        m.PERIODIC_Z = p.PERIODIC_Z;
        m.P_REFINE = p.P_REFINE;
        m.N_REFINE_START = p.N_REFINE_START;
        m.N_REFINE_INC = p.N_REFINE_INC;
        m.N_REFINE_MAX = p.N_REFINE_MAX;
        m.N_PROBE = p.N_PROBE;
        m.N_PROBE_DENSITY = p.N_PROBE_DENSITY;
        m.N_PROBE_FREQUENCY = p.N_PROBE_FREQUENCY;
        m.V_PROBE_TOL = p.V_PROBE_TOL;
        m.N_PROBE_FORCE = p.N_PROBE_FORCE;
        m.N_PROBE_F_FREQUENCY = p.N_PROBE_F_FREQUENCY;
        m.N_PROBE_F_START = p.N_PROBE_F_START;
        m.N_PROBE_AVE = p.N_PROBE_AVE;
        m.N_PROBE_AVE_FREQUENCY = p.N_PROBE_AVE_FREQUENCY;
        m.N_PROBE_AVE_START = p.N_PROBE_AVE_START;
        m.N_PRINT_LEVELS = p.N_PRINT_LEVELS;
        m.N_PRINT_LEVELS_VTHB = p.N_PRINT_LEVELS_VTHB;
        m.N_PRINT_LEVELS_PATCH = p.N_PRINT_LEVELS_PATCH;
        m.N_PRINT_LEVELS_IMAGE = p.N_PRINT_LEVELS_IMAGE;
        m.P_OUTPUT = p.P_OUTPUT;
        m.N_OUTPUT_START = p.N_OUTPUT_START;
        const int bw = 4 * m.Nqx;
        m.VOL_I_MIN = p.VOL_I_MIN / bw;
        m.VOL_I_MAX = p.VOL_I_MAX / bw;
        m.VOL_J_MIN = p.VOL_J_MIN / bw;
        m.VOL_J_MAX = p.VOL_J_MAX / bw;
        m.VOL_K_MIN = p.VOL_K_MIN / bw;
        m.VOL_K_MAX = p.VOL_K_MAX / bw;
        m.input_dir = p.I_DIR_NAME;
        m.output_dir = p.P_DIR_NAME;
        m.use_cpu = p.USE_CPU;
        if (std::is_same<typename std::remove_reference<decltype(m.dx)>::type, double>::value) m.N_PRECISION = 1;

        // Level count and clamps (mesh_init.cu:73-95).
        m.MAX_LEVELS = m.MAX_LEVELS_WALL > m.MAX_LEVELS_INTERIOR ? m.MAX_LEVELS_WALL : m.MAX_LEVELS_INTERIOR;
        if (m.MAX_LEVELS == 1) m.N_LEVEL_START = 0;
        if (m.N_LEVEL_START > m.MAX_LEVELS - 1) m.N_LEVEL_START = m.MAX_LEVELS - 1;
        auto clamp = [&](int &v) { if (v > m.MAX_LEVELS) v = m.MAX_LEVELS; };
        clamp(m.N_PRINT_LEVELS);
        clamp(m.N_PRINT_LEVELS_VTHB);
        clamp(m.N_PRINT_LEVELS_PATCH);
        clamp(m.N_PRINT_LEVELS_IMAGE);
        if (m.MAX_LEVELS == 1) {
            m.N_PRINT_LEVELS_IMAGE = 1;
            m.N_PRINT_LEVELS = m.N_PRINT_LEVELS_VTHB = m.N_PRINT_LEVELS_PATCH = 0;
        }

        // Output directory with its img/ and input/ folders (mesh_init.cu:98-104).
        if (m.output_dir.empty() || m.output_dir.back() != '/') m.output_dir += "/";
        ::mkdir(m.output_dir.c_str(), 0755);
        ::mkdir((m.output_dir + "img").c_str(), 0755);
        ::mkdir((m.output_dir + "input").c_str(), 0755);
        m.output_file_direct = nullptr;   // the solver writes out_direct.dat through the library

        m.dxf_vec = new typename std::remove_reference<decltype(m.dxf_vec[0])>::type[m.MAX_LEVELS];
        for (int L = 0; L < m.MAX_LEVELS; L++) m.dxf_vec[L] = m.dx / (1 << L);
        for (int i = 0; i < m.N_DEV; i++) {
            m.n_ids[i] = new int[m.MAX_LEVELS + 1]();
            m.id_max[i] = new int[m.MAX_LEVELS + 1]();
            m.n_gaps[i] = 0;
        }
        m.mesh_init = 1;
        return 0;
    }

    static int dest(MeshT &m)
    {
        if (!m.mesh_init) return 0;
        delete[] m.Nxi;
        delete[] m.dxf_vec;
        for (int i = 0; i < m.N_DEV; i++) {
            delete[] m.n_ids[i];
            delete[] m.id_max[i];
        }
        m.mesh_init = 0;
        return 0;
    }

    static int ref_criteria(MeshT &m, int L, int var)
    {
        if (var == V_MESH_REF_SOLUTION) {
            // mesh_criterion.cu:112-116: the solver's criterion
            if (m.n_ids[0][L] > 0) m.solver->S_ComputeRefCriteria(0, L, var);
            return 0;
        }
        if (var != V_MESH_REF_NW_CASES && var != V_MESH_REF_UNIFORM) return 0;
        agal_ctx *c = ctx(m);
        check(c, agal_mesh_ref_criteria(c, L, var == V_MESH_REF_UNIFORM ? AGAL_MESH_REF_UNIFORM : AGAL_MESH_REF_NW_CASES),
              "agal_mesh_ref_criteria");
        return 0;
    }

    static int refine_coarsen(MeshT &m)
    {
        agal_ctx *c = ctx(m);
        check(c, agal_refine_coarsen(c), "agal_refine_coarsen");
        mirror_counts(m, c);
#if defined(P_SHOW_REFINE) && (P_SHOW_REFINE == 1)
        // completes the row M_Advance_RefineWithSolution started in
        // refine_counter.txt: blocks refined and coarsened by this pass
        if (m.to.init) {
            int nr = 0, nc = 0;
            check(c, agal_refine_stats(c, nullptr, &nr, &nc), "agal_refine_stats");
            m.to.ref_printer << nr << " " << nc << std::endl;
        }
#endif
        return 0;
    }

    static int freeze(MeshT &m, int var)
    {
        agal_ctx *c = ctx(m);
        check(c, agal_freeze_refined_cells(c, var), "agal_freeze_refined_cells");
        return 0;
    }

    template <class F>
    static int geometry_pass(MeshT &m, F f, const char *what)
    {
        agal_ctx *c = ctx(m);
        check(c, f(c), what);
        return 0;
    }

    // Mesh::M_Restart (mesh_restart.cu:45-225) on <P_DIR_NAME>restart.bin.
    // A missing or unreadable file returns 1, which M_Advance_LoadRestartFile
    // reports before starting from step 0.
    static int restart(MeshT &m, int var, int *iter)
    {
        agal_ctx *c = ctx(m);
        const std::string path = m.output_dir + "restart.bin";
        if (var == V_MESH_RESTART_SAVE) {
            check(c, agal_restart_save(c, path.c_str(), iter ? *iter : 0), "agal_restart_save");
            return 0;
        }
        int it = 0;
        const int rc = agal_restart_load(c, path.c_str(), &it);
        if (rc == AGAL_ERR_IO) {
            std::cout << "[-] Restart file " << path << " not loaded: " << agal_last_error(c) << std::endl;
            return 1;
        }
        check(c, rc, "agal_restart_load");
        if (iter) *iter = it;
        mirror_counts(m, c);
        return 0;
    }

    // Mesh::M_RetrieveFromGPU: the context keeps the data on the device;
    // host copies the solver made for output are refreshed on next use.
    static int retrieve(MeshT &m)
    {
        ContextOwner *o = m.solver ? dynamic_cast<ContextOwner *>(m.solver) : nullptr;
        if (o) o->host_copies_stale();
        return 0;
    }

    // Mesh::M_RenderAndPrint_Uniform (mesh_print_uniform.cu:96-188): one
    // frame of the current macros appended to out_direct.dat.
    static int print_uniform(MeshT &m, int iter)
    {
        agal_ctx *c = ctx(m);
        check(c, agal_uniform_append(c, (m.output_dir + "out_direct.dat").c_str(), iter), "agal_uniform_append");
        return 0;
    }

    static int vtk_not_built(const char *what)
    {
        static bool told = false;
        if (!told) std::cout << "[-] " << what << ": VTK output is not part of the B200 library" << std::endl;
        told = true;
        return 0;
    }
};

}  // namespace agal_b200

// Explicit specialisations of the Mesh members that touch device data, for
// one (ufloat_t, ufloat_g_t, ArgsPack) instantiation.  Declared before the
// first use of that instantiation, they replace the reference's definitions
// while the rest of the class (the M_Advance_* loop) stays the reference's.
#define AGAL_B200_MESH_ADAPTOR(UF, UG, APP)                                                                        \
    template <> inline int Mesh<UF, UG, APP>::M_Init()                                                              \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::init(*this); }                                              \
    template <> inline int Mesh<UF, UG, APP>::M_Dest()                                                              \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::dest(*this); }                                              \
    template <> inline int Mesh<UF, UG, APP>::M_ComputeRefCriteria(int, int L, int var)                             \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::ref_criteria(*this, L, var); }                              \
    template <> inline int Mesh<UF, UG, APP>::M_RefineAndCoarsenBlocks(int)                                         \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::refine_coarsen(*this); }                                    \
    template <> inline int Mesh<UF, UG, APP>::M_FreezeRefinedCells(int var)                                         \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::freeze(*this, var); }                                       \
    template <> inline int Mesh<UF, UG, APP>::M_Geometry_Voxelize_S1(int, int L)                                    \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::geometry_pass(                                              \
          *this, [L](agal_ctx *c) { return agal_voxelize_s1(c, L); }, "agal_voxelize_s1"); }                        \
    template <> inline int Mesh<UF, UG, APP>::M_Geometry_Voxelize_S2(int, int L)                                    \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::geometry_pass(                                              \
          *this, [L](agal_ctx *c) { return agal_voxelize_s2(c, L); }, "agal_voxelize_s2"); }                        \
    template <> inline int Mesh<UF, UG, APP>::M_Geometry_Voxelize_S3(int)                                           \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::geometry_pass(                                              \
          *this, [](agal_ctx *c) { return agal_voxelize_s3(c); }, "agal_voxelize_s3"); }                            \
    template <> inline int Mesh<UF, UG, APP>::M_UpdateSolidChildren(int, int L)                                     \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::geometry_pass(                                              \
          *this, [L](agal_ctx *c) { return agal_update_solid_children(c, L); }, "agal_update_solid_children"); }    \
    template <> inline int Mesh<UF, UG, APP>::M_LinkLengthComputation(int, int L)                                   \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::geometry_pass(                                              \
          *this, [L](agal_ctx *c) { return agal_link_lengths(c, L); }, "agal_link_lengths"); }                      \
    template <> inline int Mesh<UF, UG, APP>::M_Restart(int, int var, int *iter)                                    \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::restart(*this, var, iter); }                                \
    template <> inline int Mesh<UF, UG, APP>::M_LoadToGPU() { return 0; }                                           \
    template <> inline int Mesh<UF, UG, APP>::M_RetrieveFromGPU()                                                   \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::retrieve(*this); }                                          \
    template <> inline int Mesh<UF, UG, APP>::M_RenderAndPrint_Uniform(int, int iter)                               \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::print_uniform(*this, iter); }                               \
    template <> inline int Mesh<UF, UG, APP>::M_Print_VTHB(int, int)                                                \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::vtk_not_built("M_Print_VTHB"); }                            \
    template <> inline int Mesh<UF, UG, APP>::M_Print_VTHB_Patch(int, int)                                          \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::vtk_not_built("M_Print_VTHB_Patch"); }                      \
    template <> inline int Mesh<UF, UG, APP>::M_Print_ImageData(int, int)                                           \
    { return agal_b200::MeshAdaptor<Mesh<UF, UG, APP>>::vtk_not_built("M_Print_ImageData"); }

AGAL_B200_MESH_ADAPTOR(float, float, &agal_b200::AP2D)
AGAL_B200_MESH_ADAPTOR(float, float, &agal_b200::AP3D)
AGAL_B200_MESH_ADAPTOR(double, double, &agal_b200::AP2D)
AGAL_B200_MESH_ADAPTOR(double, double, &agal_b200::AP3D)

// The reference's Solver interface (inc/solver.h:62-71) on a library context.
template <typename ufloat_t, typename ufloat_g_t, const ArgsPack *AP, const LBMPack *LP>
class Solver_B200 : public Solver<ufloat_t, ufloat_g_t, AP>, public agal_b200::ContextOwner {
    using Base = Solver<ufloat_t, ufloat_g_t, AP>;

  public:
    Solver_B200(Mesh<ufloat_t, ufloat_g_t, AP> *mesh_, const agal_b200::Options &opt = agal_b200::Options())
        : Base(mesh_), opt_(opt)
    {
        S_Init();
    }
    ~Solver_B200() override
    {
        if (ctx_) agal_ctx_destroy(ctx_);
        ctx_ = nullptr;
    }
    Solver_B200(const Solver_B200 &) = delete;
    Solver_B200 &operator=(const Solver_B200 &) = delete;

    // S_SetIC (solver_lbm_kernels.cu:79-98).
    int S_SetIC(int, int L) override { return run(agal_set_ic(ctx_, L), "agal_set_ic"); }
    // S_Interpolate (solver_lbm_kernels_comm.cu:141-155, 642-658).
    int S_Interpolate(int, int L, int var) override { return run(agal_interpolate(ctx_, L, var), "agal_interpolate"); }
    // S_Average (solver_lbm_kernels_comm.cu:351-370).
    int S_Average(int, int L, int var) override { return run(agal_average(ctx_, L, var), "agal_average"); }

    // S_Advance (solver_lbm_advance.cu:31-174): one step of level L and the
    // finer levels.  With tmp (builds with P_SHOW_ADVANCE=1) the step is
    // timed and a row of time_counter.txt written as the reference does;
    // collide, boundary and stream are one fused kernel here, so the whole
    // step's time goes to the level's collide column.
    int S_Advance(int, int L, double *tmp) override
    {
        if (!tmp) return run(agal_advance(ctx_, L), "agal_advance");
        auto &m = *this->mesh;
        check_sync();
        const auto t0 = std::chrono::steady_clock::now();
        run(agal_advance(ctx_, L), "agal_advance");
        check_sync();
        const double us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
        tmp[1 + 6 * L] += us;
        if (L == m.N_LEVEL_START) {
            double tot = 0.0;
            for (int k = m.N_LEVEL_START; k < 6 * m.MAX_LEVELS; k++) {
                tot += tmp[k];
                m.to.adv_printer << tmp[k] << " ";
            }
            m.to.adv_printer << cell_updates() / tot << std::endl;
        }
        return 0;
    }

    // S_ComputeProperties (solver_lbm_compute.cu:5-26): rho, u, v, w of the
    // cells of block i_kap from the macros as of the last M_RetrieveFromGPU.
    int S_ComputeProperties(int, int, int i_kap, ufloat_t, double *out) override
    {
        fetch_macros();
        const int dim = this->N_DIM, MT = this->M_TBLOCK, MC = this->M_CBLOCK;
        const size_t nmc = (size_t)this->n_maxcells;
        for (int k = 0; k < MT; k++) {
            const size_t cell = (size_t)i_kap * MC + k;
            for (int r = 0; r < 4; r++) out[k + r * MT] = r <= dim ? macros_[r * nmc + cell] : 0.0;
        }
        return 0;
    }

    // S_ComputeOutputProperties (solver_lbm_compute.cu:29-160) feeds the VTK
    // writers, which are not part of the library: rho, u, v, w are filled,
    // the derived rows are not.
    int S_ComputeOutputProperties(int i_dev, int i_Q, int i_kap, ufloat_t dx_L, double *out) override
    {
        S_ComputeProperties(i_dev, i_Q, i_kap, dx_L, out);
        return AGAL_ERR_UNSUPPORTED;
    }

    // S_ReportForces (solver_lbm_compute.cu:166-215): FP64 sums of the MEA
    // partials, force coefficients printed and appended to forces.txt with
    // the reference's reference length 1/64 and velocity 0.05; the partials
    // are reset.  The last force (Fx, Fy, Fz) is kept for last_force().
    int S_ReportForces(int, int L, int iter, double t, int START) override
    {
        if (!(START == 1 && L == -1)) return 0;
        auto &m = *this->mesh;
        double F[6];
        run(agal_forces(ctx_, F), "agal_forces");
        const int lf = S_FORCE_TYPE_ == 1 ? m.N_LEVEL_START : m.MAX_LEVELS - 1;
        const double factor = 1.0 / (double)m.dxf_vec[lf];
        force_[0] = factor * (F[0] - F[1]);
        force_[1] = factor * (F[2] - F[3]);
        force_[2] = this->N_DIM == 3 ? factor * (F[4] - F[5]) : 0.0;
        const double Dp = 1.0 / 64.0, uin = 0.05, pi = 3.14159265358979323846;
        const double cd = 2.0 * force_[0] / (uin * uin * Dp), cl = 2.0 * force_[1] / (uin * uin * Dp);
        const double cd3 = 8.0 * force_[0] / (uin * uin * (pi * Dp * Dp)), cl3 = 8.0 * force_[1] / (uin * uin * (pi * Dp * Dp));
        std::cout << "Report:" << std::endl;
        std::cout << "CD: " << cd << "   " << cd3 << std::endl;
        std::cout << "CL: " << cl << std::endl;
        m.to.force_printer << iter << " " << t << " " << cd << " " << cl << " " << cd3 << " " << cl3 << std::endl;
        return 0;
    }

    // S_ComputeRefCriteria (solver_lbm_criterion.cu:595-613).
    int S_ComputeRefCriteria(int, int, int) override { return run(agal_ref_criteria(ctx_), "agal_ref_criteria"); }
    // S_RefreshVariables (solver_lbm_kernels.cu:161-175).
    int S_RefreshVariables(int, int L, int = 0) override { return run(agal_refresh(ctx_, L), "agal_refresh"); }
    // S_Debug (solver_lbm_kernels_debug.cu): geometry drawing for debugging,
    // not part of the library.
    int S_Debug(int, int, int) override { return 0; }

    void host_copies_stale() override { macros_valid_ = false; }

    // The force of the last S_ReportForces: (Fx, Fy, Fz) = (Fp - Fm) / dx.
    const double *last_force() const { return force_; }

  private:
    // S_Init (solver_lbm_init.cu:4-102): the context from the Parser's maps,
    // the LBMPack and the options; the geometry imported when the mesh has
    // one; the out_direct.dat header that M_Init writes in the reference.
    int S_Init() override
    {
        auto &m = *this->mesh;
        agal_params p = agal_b200::params_from_parser(*this->parser);
        p.velocity_set = LP->VS == VelocitySet::D2Q9 ? AGAL_D2Q9 : LP->VS == VelocitySet::D3Q19 ? AGAL_D3Q19 : AGAL_D3Q27;
        if (LP->CM == CollisionOperator::TRT) throw std::runtime_error("agal_b200: TRT collision is not built");
        p.collision = LP->CM == CollisionOperator::MRT ? AGAL_MRT : AGAL_BGK;
        if (LP->IM == InterpOrder::Quadratic) throw std::runtime_error("agal_b200: quadratic interpolation is not built");
        p.interp_order = LP->IM == InterpOrder::Cubic ? AGAL_INTERP_CUBIC : AGAL_INTERP_LINEAR;
        p.S_LES = LP->LM == LESModel::Smagorinsky ? 1 : LP->LM == LESModel::WALE ? 2 : LP->LM == LESModel::Vreman ? 3 : 0;
        p.storage = opt_.storage >= 0 ? opt_.storage
                                      : (std::is_same<ufloat_t, double>::value ? AGAL_STORE_FP64 : AGAL_STORE_FP32);
        p.half_rounding = opt_.half_rounding;
        p.bc_preset = opt_.bc_preset;
        p.ic_preset = opt_.ic_preset;
        p.region_preset = opt_.region_preset;
        p.u_ref = opt_.u_ref;
        p.n_maxcblocks = opt_.n_maxcblocks;
        p.mem_frac = opt_.mem_frac;
        p.device = opt_.device;
        S_FORCE_TYPE_ = p.S_FORCE_TYPE;
        const int rc = agal_ctx_create(&p, &ctx_);
        if (rc != AGAL_OK) {
            const char *e = agal_last_error(nullptr);
            ctx_ = nullptr;
            throw std::runtime_error(std::string("agal_b200: agal_ctx_create failed: ") + (e ? e : ""));
        }
        if (opt_.step_variant > 0) run(agal_set_tuning(ctx_, opt_.step_variant), "agal_set_tuning");
        if (m.geometry_init) run(agal_import_geometry(ctx_), "agal_import_geometry");

        int nids[64], idm[64], ng = 0, ml = 0;
        int64_t nmb = 0;
        run(agal_get_counts(ctx_, nids, idm, &ng, &nmb, &ml), "agal_get_counts");
        if (ml != m.MAX_LEVELS)
            throw std::runtime_error("agal_b200: the mesh and the context disagree on MAX_LEVELS");
        agal_b200::mirror_counts(m, ctx_);
        this->n_maxcblocks = (int)nmb;
        this->n_maxcells = (long int)nmb * this->M_CBLOCK;
        this->MAX_LEVELS = m.MAX_LEVELS;
        this->MAX_LEVELS_INTERIOR = m.MAX_LEVELS_INTERIOR;
        this->N_LEVEL_START = m.N_LEVEL_START;
        run(agal_uniform_header(ctx_, (m.output_dir + "out_direct.dat").c_str()), "agal_uniform_header");
        std::cout << "[-] Finished making solver (B200) object." << std::endl << std::endl;
        return 0;
    }

    int run(int rc, const char *what)
    {
        agal_b200::check(ctx_, rc, what);
        return 0;
    }
    void check_sync() { run(agal_sync(ctx_), "agal_sync"); }

    // Cell updates of one coarse step, counted as solver_lbm_advance.cu:74-89 does.
    double cell_updates() const
    {
        auto &m = *this->mesh;
        long long cells = 0, mult = 1;
        for (int L = m.N_LEVEL_START; L < m.MAX_LEVELS - 1; L++, mult *= 2)
            cells += mult * (m.n_ids[0][L] - m.n_ids[0][L + 1] / this->N_CHILDREN);
        cells += mult * m.n_ids[0][m.MAX_LEVELS - 1];
        return (double)cells * this->M_CBLOCK;
    }

    void fetch_macros()
    {
        if (macros_valid_) return;
        size_t bytes = 0;
        run(agal_array_bytes(ctx_, AGAL_ARR_MACROS, &bytes), "agal_array_bytes");
        macros_.resize(bytes / sizeof(double));
        run(agal_dump(ctx_, AGAL_ARR_MACROS, macros_.data(), bytes), "agal_dump");
        macros_valid_ = true;
    }

    agal_b200::Options opt_;
    int S_FORCE_TYPE_ = 0;
    double force_[3] = {0.0, 0.0, 0.0};
    std::vector<double> macros_;
    bool macros_valid_ = false;
};

#endif  // AGAL_SOLVER_B200_HPP
