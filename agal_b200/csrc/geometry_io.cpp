// Geometry import on the host: ASCII STL (Geometry::G_ImportSTL_ASCII,
// geometry_import.cu:11-83), the primitives of geometry.txt
// (G_ImportBoundariesFromTextFile, geometry_add.cu:539-666, with
// G_Convert_IndexListsToCoordList, geometry_convert.cu:11-58), the splitting
// of long faces (G_RefineFaces_Length, geometry_refine.cu:8-225) and the
// import sequence of the reference's main (main.cu:94-101 and the refinement
// G_Init_Arrays_CoordsList_CPU runs first, geometry_init.cu:80-89).
//
// Faces are n x 9 floats (v1 x y z, v2 x y z, v3 x y z), in the reference's
// order: STL facets as read (degenerate ones dropped), primitives in the order
// of geometry.txt, the pieces of a split face replacing it (first piece) and
// appended after all faces (the others), faces visited from the last to the
// first.  All arithmetic is float as the reference's ufloat_g_t, with no
// contraction of multiply and add (plain x86-64 code).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ctx.h"

namespace {

struct Face {
    float v[9];
};

// Shapes built from a node list and index triples (G_Add*), converted to
// faces as G_Convert_IndexListsToCoordList does.
struct Shapes {
    std::vector<float> x, y, z;
    std::vector<int> f;   // triples
    int node(float a, float b, float c)
    {
        x.push_back(a);
        y.push_back(b);
        z.push_back(c);
        return (int)x.size() - 1;
    }
};

// Corners of an axis-aligned box in the reference's node order
// (x low: (ay,az) (by,az) (ay,bz) (by,bz); then x high, same order) and the
// two triangle tables: the domain box faces inwards (G_AddBoundingBox,
// geometry_add.cu:48-127), a prism outwards (G_AddPrism, :199-278).
const int kBoxFaces[12][3] = {{0, 1, 3}, {0, 3, 2}, {4, 6, 7}, {4, 7, 5}, {0, 2, 6}, {0, 6, 4},
                              {1, 5, 7}, {1, 7, 3}, {7, 6, 2}, {7, 2, 3}, {0, 4, 5}, {0, 5, 1}};
const int kPrismFaces[12][3] = {{0, 2, 3}, {0, 3, 1}, {4, 5, 7}, {4, 7, 6}, {0, 4, 6}, {0, 6, 2},
                                {1, 3, 7}, {1, 7, 5}, {7, 3, 2}, {7, 2, 6}, {0, 1, 5}, {0, 5, 4}};

void add_cuboid(Shapes &s, float ax, float bx, float ay, float by, float az, float bz, const int (*tab)[3])
{
    const int n0 = (int)s.x.size();
    const float X[2] = {ax, bx}, Y[2] = {ay, by}, Z[2] = {az, bz};
    for (int i = 0; i < 2; i++)
        for (int k = 0; k < 2; k++)
            for (int j = 0; j < 2; j++) s.node(X[i], Y[j], Z[k]);
    for (int t = 0; t < 12; t++)
        for (int q = 0; q < 3; q++) s.f.push_back(n0 + tab[t][q]);
}

// Latitude-longitude sphere (G_AddSphere, geometry_add.cu:281-317): N1 polar
// by N2 azimuthal nodes, two triangles per quad, the pole rows included.
void add_sphere(Shapes &s, int N1, int N2, float cx, float cy, float cz, float R)
{
    const int n0 = (int)s.x.size();
    const float pi = (float)M_PI;
    const float d1 = (float)N1 - 1.0f, d2 = (float)N2 - 1.0f;
    for (int j = 0; j < N1; j++)
        for (int k = 0; k < N2; k++) {
            const float t = (pi / d1) * (float)j, p = (2 * pi / d2) * (float)k;
            const float st = std::sin(t), ct = std::cos(t), sp = std::sin(p), cp = std::cos(p);
            s.node(R * st * cp + cx, R * st * sp + cy, R * ct + cz);
            if (j < N1 - 1 && k < N2 - 1) {
                // (ID1, ID2, ID3) = (k,j), (k+1,j+1), (k+1,j) and (k,j), (k,j+1), (k+1,j+1)
                const int a = n0 + k + N2 * j, b = n0 + (k + 1) + N2 * j, c = n0 + (k + 1) + N2 * (j + 1),
                          d = n0 + k + N2 * (j + 1);
                s.f.insert(s.f.end(), {a, c, b, a, d, c});
            }
        }
}

std::vector<Face> to_faces(const Shapes &s)
{
    std::vector<Face> out(s.f.size() / 3);
    for (size_t j = 0; j < out.size(); j++)
        for (int q = 0; q < 3; q++) {
            const int n = s.f[3 * j + q];
            out[j].v[3 * q + 0] = s.x[n];
            out[j].v[3 * q + 1] = s.y[n];
            out[j].v[3 * q + 2] = s.z[n];
        }
    return out;
}

int read_stl(const char *path, std::vector<Face> &out)
{
    std::ifstream in(path);
    if (!in) return AGAL_ERR_IO;
    std::string line, word;
    std::getline(in, line);   // solid ...
    std::getline(in, line);   // facet normal ... of the first facet
    std::stringstream ss(line);
    // Facet blocks until the line after a facet starts with "endsolid".
    while (word != "endsolid") {
        float v[9];
        std::getline(in, line);   // outer loop
        for (int q = 0; q < 3; q++) {
            std::getline(in, line);
            ss.clear();
            ss.str(line);
            ss >> word >> v[3 * q] >> v[3 * q + 1] >> v[3 * q + 2];
        }
        const bool d12 = v[0] == v[3] && v[1] == v[4] && v[2] == v[5];
        const bool d13 = v[0] == v[6] && v[1] == v[7] && v[2] == v[8];
        const bool d23 = v[6] == v[3] && v[7] == v[4] && v[8] == v[5];
        if (!d12 && !d13 && !d23) {
            Face f;
            std::copy(v, v + 9, f.v);
            out.push_back(f);
        }
        std::getline(in, line);   // endloop
        std::getline(in, line);   // endfacet
        if (!std::getline(in, line)) break;   // next facet normal, or endsolid
        ss = std::stringstream(line);
        ss >> word;
    }
    return AGAL_OK;
}

int read_text(const agal_params &P, const char *path, std::vector<Face> &out)
{
    std::ifstream in(path);
    if (!in) return AGAL_ERR_IO;
    const float Lx = (float)P.L_c, Ly = (float)(P.L_fy * P.L_c), Lz = (float)(P.L_fz * P.L_c);
    Shapes s;
    for (std::string line; std::getline(in, line);) {
        if (line == "END") break;
        std::stringstream ss(line);
        std::string w;
        if (!(ss >> w)) continue;
        if (w == "BOX") {
            add_cuboid(s, 0.0f, Lx, 0.0f, Ly, 0.0f, Lz, kBoxFaces);
        } else if (w == "PRISM") {
            std::string how;
            float ax, bx, ay, by, az, bz;
            ss >> how;
            if (how == "CORNER") {
                ss >> ax >> bx >> ay >> by >> az >> bz;
            } else {
                float cx, cy, cz, lx, ly, lz;
                ss >> cx >> cy >> cz >> lx >> ly >> lz;
                ax = (float)(cx - lx / 2.0);
                bx = (float)(cx + lx / 2.0);
                ay = (float)(cy - ly / 2.0);
                by = (float)(cy + ly / 2.0);
                az = (float)(cz - lz / 2.0);
                bz = (float)(cz + lz / 2.0);
            }
            add_cuboid(s, ax, bx, ay, by, az, bz, kPrismFaces);
        } else if (w == "SPHERE") {
            int N1, N2;
            float cx, cy, cz, R;
            ss >> N1 >> N2 >> cx >> cy >> cz >> R;
            add_sphere(s, N1, N2, cx, cy, cz, R);
        } else if (w == "RECTANGLE" || w == "CIRCLE" || w == "NACA002D" || w == "NACA003D") {
            // 2D segment shapes (the 3D solver path does not take them) and
            // the NACA airfoil generators are not built
            return AGAL_ERR_UNSUPPORTED;
        }
    }
    out = to_faces(s);
    return AGAL_OK;
}

float edge(const float *a, const float *b)
{
    const float dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}

// Midpoint subdivision until every edge is at most l_spec; the first leaf
// replaces the face, the others are appended (RecursiveRefineFace).
void refine(int depth, float l_spec, const float *v1, const float *v2, const float *v3, std::vector<Face> &fs,
            bool &replaced, size_t first)
{
    const float lm = std::max({edge(v1, v2), edge(v2, v3), edge(v3, v1)});
    if (lm > l_spec) {
        float m1[3], m2[3], m3[3];
        for (int d = 0; d < 3; d++) {
            m1[d] = 0.5f * (v1[d] + v2[d]);
            m2[d] = 0.5f * (v2[d] + v3[d]);
            m3[d] = 0.5f * (v3[d] + v1[d]);
        }
        refine(depth + 1, l_spec, v1, m1, m3, fs, replaced, first);
        refine(depth + 1, l_spec, m1, v2, m2, fs, replaced, first);
        refine(depth + 1, l_spec, m3, m2, v3, fs, replaced, first);
        refine(depth + 1, l_spec, m1, m2, m3, fs, replaced, first);
    }
    if (lm <= l_spec && depth > 0) {
        Face f;
        std::copy(v1, v1 + 3, f.v);
        std::copy(v2, v2 + 3, f.v + 3);
        std::copy(v3, v3 + 3, f.v + 6);
        if (!replaced) {
            fs[first] = f;
            replaced = true;
        } else {
            fs.push_back(f);
        }
    }
}

void refine_length(const agal_params &P, std::vector<Face> &fs)
{
    // l_spec = 0.95 G_BIN_SPEC min(Lx, Ly, Lz) / (2^(G_BIN_LEVELS-1) G_BIN_DENSITY)
    const float mult = 0.95f * (float)P.G_BIN_SPEC;
    const float Lx = (float)P.L_c, Ly = (float)(P.L_fy * P.L_c), Lz = (float)(P.L_fz * P.L_c);
    const float Lmin = std::min({Lx, Ly, Lz});
    const float finest = std::pow(2.0f, (float)(P.G_BIN_LEVELS - 1)) * (float)P.G_BIN_DENSITY;
    const float l_spec = mult * Lmin / finest;
    for (long long p = (long long)fs.size() - 1; p >= 0; p--) {
        const Face f = fs[p];
        bool replaced = false;
        refine(0, l_spec, f.v, f.v + 3, f.v + 6, fs, replaced, (size_t)p);
    }
}

int emit(const std::vector<Face> &fs, float *faces, long long cap, long long *n)
{
    if (n) *n = (long long)fs.size();
    if (!faces) return AGAL_OK;
    if (cap < (long long)fs.size()) return AGAL_ERR_PARAM;
    for (size_t j = 0; j < fs.size(); j++) std::copy(fs[j].v, fs[j].v + 9, faces + 9 * j);
    return AGAL_OK;
}

}  // namespace

extern "C" int agal_geometry_read_stl(const char *path, float *faces, long long cap, long long *n)
{
    if (!path) return AGAL_ERR_PARAM;
    std::vector<Face> fs;
    const int rc = read_stl(path, fs);
    return rc ? rc : emit(fs, faces, cap, n);
}

extern "C" int agal_geometry_read_text(const agal_params *p, const char *path, float *faces, long long cap,
                                       long long *n)
{
    if (!p || !path) return AGAL_ERR_PARAM;
    std::vector<Face> fs;
    const int rc = read_text(*p, path, fs);
    return rc ? rc : emit(fs, faces, cap, n);
}

extern "C" int agal_geometry_refine_length(const agal_params *p, float *faces, long long cap, long long *n)
{
    if (!p || !n || *n < 0 || (*n > 0 && !faces)) return AGAL_ERR_PARAM;
    std::vector<Face> fs((size_t)*n);
    for (long long j = 0; j < *n; j++) std::copy(faces + 9 * j, faces + 9 * j + 9, fs[j].v);
    refine_length(*p, fs);
    *n = (long long)fs.size();
    if (cap < *n) return AGAL_ERR_PARAM;   // *n tells the size needed
    for (size_t j = 0; j < fs.size(); j++) std::copy(fs[j].v, fs[j].v + 9, faces + 9 * j);
    return AGAL_OK;
}

extern "C" int agal_import_geometry(agal_ctx *c)
{
    if (!c) return AGAL_ERR_PARAM;
    const agal_params &P = c->P;
    std::string dir = P.I_DIR_NAME;
    if (!dir.empty() && dir.back() != '/') dir += "/";
    std::vector<Face> fs;
    int rc;
    if (P.G_LOADTYPE == 0) {
        const std::string path = dir + "geometry/" + P.G_FILENAME;
        if ((rc = read_stl(path.c_str(), fs))) return agal_set_err(c, rc, "geometry: cannot read " + path);
    } else {
        const std::string path = dir + "geometry.txt";
        if ((rc = read_text(P, path.c_str(), fs)))
            return agal_set_err(c, rc, rc == AGAL_ERR_UNSUPPORTED ? "geometry: 2D shapes and NACA profiles are not supported"
                                                                  : "geometry: cannot read " + path);
    }
    if (fs.empty()) return agal_set_err(c, AGAL_ERR_PARAM, "geometry: no faces");
    refine_length(P, fs);
    std::vector<float> flat(fs.size() * 9);
    for (size_t j = 0; j < fs.size(); j++) std::copy(fs[j].v, fs[j].v + 9, flat.data() + 9 * j);
    return agal_set_geometry(c, flat.data(), (long long)fs.size());
}
