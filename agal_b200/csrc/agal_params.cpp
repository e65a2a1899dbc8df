// input.txt parameters of the AGAL solver: defaults and parser.
//
// Keys, defaults and parsing rules follow inc/parser.h:58-183 of the
// reference: '#' starts a comment line, every line is "KEY VALUE", integer
// values may be written "A*Nx" (A times the Nx of the same file, Nx read in a
// first pass), unknown keys are reported and skipped.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "../../include/agal_b200.h"

namespace {

struct IntKey { const char *name; size_t off; int def; };
struct DblKey { const char *name; size_t off; double def; };
struct StrKey { const char *name; size_t off; const char *def; };

#define IK(n, d) {#n, offsetof(agal_params, n), d}
#define DK(n, d) {#n, offsetof(agal_params, n), d}
#define SK(n, d) {#n, offsetof(agal_params, n), d}

// Defaults of inc/parser.h:62-114.
const IntKey kInt[] = {
    IK(MAX_LEVELS_WALL, 5), IK(MAX_LEVELS_INTERIOR, 4), IK(N_ITER_TOTAL, 10 * 64), IK(N_LEVEL_START, 0),
    IK(Nx, 64), IK(N_RESTART, 1), IK(G_LOADTYPE, 0), IK(G_PRINT, 1), IK(G_VIS_TREE, 0),
    IK(G_BIN_DENSITY, 1), IK(G_BIN_APPROACH, 0), IK(G_BIN_LEVELS, 1), IK(G_BIN_SPEC, 1),
    IK(G_BIN_MAKE_LINKS, 0), IK(PERIODIC_X, 0), IK(PERIODIC_Y, 0), IK(PERIODIC_Z, 0),
    IK(S_COLLISION, 0), IK(S_INTERP, 1), IK(S_INTERP_HYBRID, 0), IK(S_AVERAGE, 0), IK(S_CRITERION, 0),
    IK(S_LES, 0), IK(S_FORCE_ORDER, 0), IK(S_FORCE_TYPE, 0), IK(S_BC_TYPE, 0), IK(P_REFINE, 32),
    IK(N_PROBE, 0), IK(N_PROBE_DENSITY, 4), IK(N_PROBE_FREQUENCY, 32), IK(N_PROBE_FORCE, 0),
    IK(N_PROBE_F_START, 0), IK(N_PROBE_F_FREQUENCY, 16), IK(N_PROBE_AVE, 0), IK(N_PROBE_AVE_FREQUENCY, 1),
    IK(N_PROBE_AVE_START, 100 * 64), IK(N_PRINT_LEVELS, 2), IK(N_PRINT_LEVELS_VTHB, 0),
    IK(N_PRINT_LEVELS_PATCH, 2), IK(N_PRINT_LEVELS_IMAGE, 2), IK(P_OUTPUT, 1 * 64), IK(N_OUTPUT, 10),
    IK(N_OUTPUT_START, 0), IK(VOL_I_MIN, 0), IK(VOL_I_MAX, 64), IK(VOL_J_MIN, 0), IK(VOL_J_MAX, 64),
    IK(VOL_K_MIN, 0), IK(VOL_K_MAX, 64), IK(USE_CPU, 1),
};
// Defaults of inc/parser.h:115-138.
const DblKey kDbl[] = {
    DK(L_c, 1.0), DK(L_fy, 1.0), DK(L_fz, 1.0), DK(v0, 1.5625e-5), DK(G_NEAR_WALL_DISTANCE, 0.05),
    DK(s1, 1.19), DK(s2, 1.40), DK(s3, 1.20), DK(s4, 1.20), DK(s5, 1.20), DK(s6, 1.98),
    DK(V_PROBE_TOL, 1e-4), DK(N_REFINE_START, -3.0), DK(N_REFINE_INC, 1.0), DK(N_REFINE_MAX, 1.0),
    DK(S_FORCEVOLUME_Xm, 0.0), DK(S_FORCEVOLUME_XM, 0.0), DK(S_FORCEVOLUME_Ym, 0.0),
    DK(S_FORCEVOLUME_YM, 0.0), DK(S_FORCEVOLUME_Zm, 0.0), DK(S_FORCEVOLUME_ZM, 0.0),
};
// Defaults of inc/parser.h:139-144.
const StrKey kStr[] = {
    SK(I_DIR_NAME, "../input/"), SK(P_DIR_NAME, "../out/TEST_UPLOAD/"), SK(G_FILENAME, "bunny_ascii.stl"),
};

int *int_field(agal_params *p, size_t off) { return reinterpret_cast<int *>(reinterpret_cast<char *>(p) + off); }
double *dbl_field(agal_params *p, size_t off) { return reinterpret_cast<double *>(reinterpret_cast<char *>(p) + off); }
char *str_field(agal_params *p, size_t off) { return reinterpret_cast<char *>(p) + off; }

// "A*Nx" -> A*Nx, "A" -> A  (parser.h:34-44).
bool parse_nx_factor(const std::string &s, int Nx, int *out)
{
    size_t pos = s.find('*');
    const std::string head = s.substr(0, pos);
    char *end = nullptr;
    long A = std::strtol(head.c_str(), &end, 10);
    if (end == head.c_str()) return false;
    *out = (pos != std::string::npos) ? static_cast<int>(A * Nx) : static_cast<int>(A);
    return true;
}

int set_key(agal_params *p, const std::string &key, const std::string &val, int Nx)
{
    for (const auto &k : kInt)
        if (key == k.name) {
            int v;
            if (!parse_nx_factor(val, Nx, &v)) return AGAL_ERR_PARAM;
            *int_field(p, k.off) = v;
            return AGAL_OK;
        }
    for (const auto &k : kDbl)
        if (key == k.name) {
            char *end = nullptr;
            double v = std::strtod(val.c_str(), &end);
            if (end == val.c_str()) return AGAL_ERR_PARAM;
            *dbl_field(p, k.off) = v;
            return AGAL_OK;
        }
    for (const auto &k : kStr)
        if (key == k.name) {
            if (val.size() >= 256) return AGAL_ERR_PARAM;
            std::strncpy(str_field(p, k.off), val.c_str(), 255);
            str_field(p, k.off)[255] = 0;
            return AGAL_OK;
        }
    return AGAL_ERR_UNSUPPORTED;
}

}  // namespace

extern "C" int agal_params_default(agal_params *p)
{
    if (!p) return AGAL_ERR_PARAM;
    std::memset(p, 0, sizeof(*p));
    for (const auto &k : kInt) *int_field(p, k.off) = k.def;
    for (const auto &k : kDbl) *dbl_field(p, k.off) = k.def;
    for (const auto &k : kStr) std::strncpy(str_field(p, k.off), k.def, 255);
    p->velocity_set = AGAL_D2Q9;
    p->collision = AGAL_BGK;
    p->interp_order = AGAL_INTERP_CUBIC;   // main.cu:55 (LP2D)
    p->storage = AGAL_STORE_FP32;
    p->bc_preset = AGAL_BC_NONE;
    p->ic_preset = AGAL_IC_REST;
    p->region_preset = AGAL_REGION_NONE;
    p->ref_pct_hi = 0.9;
    p->ref_pct_lo = 0.5;
    p->u_ref = 0.05;                       // custom.h literal
    p->ic_noise = 0.0;
    p->seed = 0;
    p->n_maxcblocks = 0;
    p->mem_frac = 0.975;                   // mesh.h:481 M_FRAC
    p->device = -1;
    p->half_rounding = AGAL_ROUND_STOCHASTIC;
    return AGAL_OK;
}

extern "C" size_t agal_params_size(void) { return sizeof(agal_params); }

extern "C" int agal_params_set(agal_params *p, const char *key, const char *value)
{
    if (!p || !key || !value) return AGAL_ERR_PARAM;
    return set_key(p, key, value, p->Nx);
}

extern "C" int agal_params_read(const char *input_dir, agal_params *p)
{
    if (!p || !input_dir) return AGAL_ERR_PARAM;
    std::string path = std::string(input_dir);
    if (!path.empty() && path.back() != '/') path += '/';
    path += "input.txt";
    std::ifstream in(path);
    if (!in) return AGAL_ERR_IO;
    // First pass: Nx (parser.h:146-160).
    int Nx = p->Nx;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ss(line);
        std::string k, v;
        ss >> k >> v;
        if (k == "Nx") {
            int t;
            if (!parse_nx_factor(v, Nx, &t)) return AGAL_ERR_PARAM;
            Nx = t;
        }
    }
    in.clear();
    in.seekg(0);
    int rc_all = AGAL_OK;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ss(line);
        std::string k, v;
        ss >> k >> v;
        if (k.empty()) continue;
        int rc = set_key(p, k, v, Nx);
        if (rc == AGAL_ERR_UNSUPPORTED) {
            std::fprintf(stderr, "Error: Invalid input (%s) skipped...\n", k.c_str());
        } else if (rc != AGAL_OK) {
            rc_all = rc;
        }
    }
    return rc_all;
}
