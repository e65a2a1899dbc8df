// Headless field output on a uniform grid in the reference's out_direct.dat
// format (the header of mesh_init.cu:114-150, the frames of
// Mesh::M_RenderAndPrint_Uniform, mesh_print_uniform.cu:96-188).
//
// The output box is [VOL_I_MIN, VOL_I_MAX) x [VOL_J_MIN, VOL_J_MAX) x
// [VOL_K_MIN, VOL_K_MAX) of the input (cells, rounded down to root blocks) at
// the resolution of level N_PRINT_LEVELS - 1: each output cell takes rho, u,
// v, w from the macros of the cell of the deepest block (at most level
// N_PRINT_LEVELS - 1) covering it, piecewise constant, with that block's
// level and ID; cells outside every root block keep rho 1, u 0, level and ID
// -1.  The reference walks the tree from each root block on the host; here
// one thread per output cell descends from its root block through the child
// lists on the device.  A frame is written after the reference's
// M_Advance_PrintData preparation (grid average, interface interpolation,
// macro refresh on every level).
//
// File: int[100] {n_frames = (N_ITER_TOTAL - N_OUTPUT_START) / P_OUTPUT,
// P_OUTPUT, N_OUTPUT_START, Nx, Ny, Nz, N_LEVEL_START, N_PRINT_LEVELS,
// N_PRECISION, VOL_I_MIN/4, VOL_I_MAX/4, VOL_J_MIN/4, VOL_J_MAX/4,
// VOL_K_MIN/4, VOL_K_MAX/4, 0 ...} (the volume bounds in root blocks), then
// double[100] {Lx, Ly, Lz, 0 ...}; per frame double t = iter / Nx, then six
// fields of nx*ny*nz doubles (x fastest): rho, u, v, w, level, block ID.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "ctx.h"
#include "lattice.cuh"

namespace agal {
namespace {

struct UniformArgs {
    int dim, MC, print_levels, mult;   // mult = 2^(print_levels - 1)
    int nx, ny, nz;                    // output cells
    int i0, j0, k0;                    // volume origin in root blocks
    int rbx, rby, rbz;                 // root grid size in blocks
    const int *root;                   // [rbz][rby][rbx] level-0 block ID, -1 none
    const int *nbr_child;
    long long nmc;
    const void *macro;                 // [dim+1][n_maxcells] of the compute type
    bool f64;
    double *out;                       // [6][nx*ny*nz]
};

__global__ void k_render_uniform(const UniformArgs a)
{
    const long long vol = (long long)a.nx * a.ny * a.nz;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= vol) return;
    const int X = (int)(g % a.nx), Y = (int)((g / a.nx) % a.ny), Z = (int)(g / ((long long)a.nx * a.ny));
    // root block and the fine position inside it (units of the output grid)
    const int span = 4 * a.mult;
    const int bi = X / span + a.i0, bj = Y / span + a.j0, bk = (a.dim == 3 ? Z / span : 0) + a.k0;
    double rho = 1.0, u = 0.0, v = 0.0, w = 0.0, lev = -1.0, id = -1.0;
    if (bi >= 0 && bi < a.rbx && bj >= 0 && bj < a.rby && bk >= 0 && bk < a.rbz) {
        int b = a.root[((long long)bk * a.rby + bj) * a.rbx + bi];
        if (b >= 0) {
            int px = X % span, py = Y % span, pz = a.dim == 3 ? Z % span : 0;
            int L = 0, s = span;   // s: output cells per block side at level L
            while (L + 1 < a.print_levels) {
                const int c0 = a.nbr_child[b];
                if (c0 < 0) break;
                const int h = s / 2;
                const int xi = px >= h, xj = py >= h, xk = (a.dim == 3 && pz >= h);
                b = c0 + xi + 2 * xj + 4 * xk;
                px -= xi * h;
                py -= xj * h;
                pz -= xk * h;
                s = h;
                L++;
            }
            const int m = s / 4;   // output cells per cell of this block
            const int cell = px / m + 4 * (py / m) + (a.dim == 3 ? 16 * (pz / m) : 0);
            const long long ci = (long long)b * a.MC + cell;
            auto mac = [&](int r) {
                return a.f64 ? static_cast<const double *>(a.macro)[r * a.nmc + ci]
                             : (double)static_cast<const float *>(a.macro)[r * a.nmc + ci];
            };
            rho = mac(0);
            u = mac(1);
            v = mac(2);
            w = a.dim == 3 ? mac(3) : 0.0;
            lev = (double)L;
            id = (double)b;
        }
    }
    a.out[g] = rho;
    a.out[g + vol] = u;
    a.out[g + 2 * vol] = v;
    a.out[g + 3 * vol] = w;
    a.out[g + 4 * vol] = lev;
    a.out[g + 5 * vol] = id;
}

struct Box {
    int i0, i1, j0, j1, k0, k1, pl, mult, nx, ny, nz;
};

Box box_of(const agal_ctx *c)
{
    Box x{};
    const agal_params &P = c->P;
    x.i0 = P.VOL_I_MIN / 4;
    x.i1 = P.VOL_I_MAX / 4;
    x.j0 = P.VOL_J_MIN / 4;
    x.j1 = P.VOL_J_MAX / 4;
    x.k0 = c->dim == 3 ? P.VOL_K_MIN / 4 : 0;
    x.k1 = c->dim == 3 ? P.VOL_K_MAX / 4 : 1;
    x.pl = P.N_PRINT_LEVELS > 0 ? P.N_PRINT_LEVELS : 1;
    x.mult = 1 << (x.pl - 1);
    x.nx = std::max(0, x.i1 - x.i0) * 4 * x.mult;
    x.ny = std::max(0, x.j1 - x.j0) * 4 * x.mult;
    x.nz = c->dim == 3 ? std::max(0, x.k1 - x.k0) * 4 * x.mult : 1;
    return x;
}

}  // namespace
}  // namespace agal

using namespace agal;

extern "C" int agal_uniform_dims(const agal_ctx *c, int *dims)
{
    if (!c || !dims) return AGAL_ERR_PARAM;
    const Box x = box_of(c);
    dims[0] = x.nx;
    dims[1] = x.ny;
    dims[2] = x.nz;
    return AGAL_OK;
}

// Six fields [rho, u, v, w, level, block ID][nz][ny][nx] of the current
// macros (no preparation: call agal_refresh on every level first).
extern "C" int agal_uniform_render(agal_ctx *c, double *out, long long n)
{
    if (!c || !out) return AGAL_ERR_PARAM;
    const Box x = box_of(c);
    const long long vol = (long long)x.nx * x.ny * x.nz;
    if (n != 6 * vol) return agal_set_err(c, AGAL_ERR_PARAM, "uniform render: buffer size");
    if (vol == 0) return AGAL_OK;
    // root grid of level-0 blocks from their lower corners
    const int rbx = c->Nx / 4, rby = c->Ny / 4, rbz = c->dim == 3 ? c->Nz / 4 : 1;
    const int n0 = c->n_ids[0];
    std::vector<int> ids(std::max(n0, 1)), root((size_t)rbx * rby * rbz, -1);
    std::vector<float> fx((size_t)c->dim * c->nmb);
    AGAL_CUDA(c, cudaStreamSynchronize(c->stream));
    if (n0 > 0) AGAL_CUDA(c, cudaMemcpy(ids.data(), c->id_set, sizeof(int) * n0, cudaMemcpyDeviceToHost));
    AGAL_CUDA(c, cudaMemcpy(fx.data(), c->cblock_f_X, sizeof(float) * fx.size(), cudaMemcpyDeviceToHost));
    for (int q = 0; q < n0; q++) {
        const int b = ids[q];
        const int i = (int)std::floor(fx[b] / c->dx_cblock + 0.5f);
        const int j = (int)std::floor(fx[(size_t)c->nmb + b] / c->dx_cblock + 0.5f);
        const int k = c->dim == 3 ? (int)std::floor(fx[2 * (size_t)c->nmb + b] / c->dx_cblock + 0.5f) : 0;
        if (i >= 0 && i < rbx && j >= 0 && j < rby && k >= 0 && k < rbz) root[((size_t)k * rby + j) * rbx + i] = b;
    }
    int *d_root = nullptr;
    double *d_out = nullptr;
    AGAL_CUDA(c, cudaMalloc(&d_root, sizeof(int) * root.size()));
    if (cudaMalloc(&d_out, sizeof(double) * 6 * vol) != cudaSuccess) {
        cudaFree(d_root);
        return agal_set_err(c, AGAL_ERR_OOM, "uniform render: output buffer");
    }
    int rc = AGAL_OK;
    UniformArgs a{};
    a.dim = c->dim;
    a.MC = c->MC;
    a.print_levels = x.pl;
    a.mult = x.mult;
    a.nx = x.nx;
    a.ny = x.ny;
    a.nz = x.nz;
    a.i0 = x.i0;
    a.j0 = x.j0;
    a.k0 = x.k0;
    a.rbx = rbx;
    a.rby = rby;
    a.rbz = rbz;
    a.root = d_root;
    a.nbr_child = c->cblock_ID_nbr_child;
    a.nmc = c->nmc;
    a.macro = c->macro;
    a.f64 = c->storage == AGAL_STORE_FP64;
    a.out = d_out;
    if (cudaMemcpyAsync(d_root, root.data(), sizeof(int) * root.size(), cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess) {
        rc = agal_set_err(c, AGAL_ERR_CUDA, "uniform render: root grid copy");
    } else {
        k_render_uniform<<<(unsigned)((vol + 255) / 256), 256, 0, c->stream>>>(a);
        if (cudaGetLastError() != cudaSuccess || cudaMemcpyAsync(out, d_out, sizeof(double) * 6 * vol,
                                                                 cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
            cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = agal_set_err(c, AGAL_ERR_CUDA, "uniform render failed");
    }
    cudaFree(d_root);
    cudaFree(d_out);
    return rc;
}

// The file header (M_Init, mesh_init.cu:114-150): creates or truncates `path`.
extern "C" int agal_uniform_header(agal_ctx *c, const char *path)
{
    if (!c || !path) return AGAL_ERR_PARAM;
    const agal_params &P = c->P;
    int ip[100] = {0};
    double dp[100] = {0.0};
    ip[0] = P.P_OUTPUT > 0 ? (P.N_ITER_TOTAL - P.N_OUTPUT_START) / P.P_OUTPUT : 0;
    ip[1] = P.P_OUTPUT;
    ip[2] = P.N_OUTPUT_START;
    ip[3] = c->Nx;
    ip[4] = c->Ny;
    ip[5] = c->Nz;   // 1 in 2D
    ip[6] = P.N_LEVEL_START;
    ip[7] = P.N_PRINT_LEVELS;
    ip[8] = c->storage == AGAL_STORE_FP64 ? 1 : 0;   // N_PRECISION
    // the reference stores these in root blocks, the maxima (and J/K minima)
    // multiplied by its sub-block count Nqx = 1
    ip[9] = P.VOL_I_MIN / 4;
    ip[10] = P.VOL_I_MAX / 4;
    ip[11] = P.VOL_J_MIN / 4;
    ip[12] = P.VOL_J_MAX / 4;
    ip[13] = P.VOL_K_MIN / 4;
    ip[14] = P.VOL_K_MAX / 4;
    dp[0] = P.L_c;
    dp[1] = P.L_fy * P.L_c;
    dp[2] = P.L_fz * P.L_c;
    FILE *f = fopen(path, "wb");
    if (!f) return agal_set_err(c, AGAL_ERR_IO, std::string("uniform output: cannot open ") + path);
    const bool ok = fwrite(ip, sizeof(int), 100, f) == 100 && fwrite(dp, sizeof(double), 100, f) == 100;
    fclose(f);
    return ok ? AGAL_OK : agal_set_err(c, AGAL_ERR_IO, "uniform output: write failed");
}

// One frame of the current macros (M_RenderAndPrint_Uniform): t = iter / Nx
// and the six fields appended to `path`.
extern "C" int agal_uniform_append(agal_ctx *c, const char *path, int iter)
{
    if (!c || !path) return AGAL_ERR_PARAM;
    int rc;
    int d[3];
    agal_uniform_dims(c, d);
    const long long vol = (long long)d[0] * d[1] * d[2];
    std::vector<double> buf((size_t)std::max<long long>(6 * vol, 1));
    if ((rc = agal_uniform_render(c, buf.data(), 6 * vol))) return rc;
    FILE *f = fopen(path, "ab");
    if (!f) return agal_set_err(c, AGAL_ERR_IO, std::string("uniform output: cannot open ") + path);
    const double t = (double)iter / (double)c->Nx;
    const bool ok = fwrite(&t, sizeof(double), 1, f) == 1 &&
                    (vol == 0 || fwrite(buf.data(), sizeof(double), (size_t)(6 * vol), f) == (size_t)(6 * vol));
    fclose(f);
    return ok ? AGAL_OK : agal_set_err(c, AGAL_ERR_IO, "uniform output: write failed");
}

// One frame as M_Advance_PrintData makes it: grid average and interface
// interpolation on a multi-level mesh, macros refreshed on every level, then
// the frame appended.
extern "C" int agal_uniform_frame(agal_ctx *c, const char *path, int iter)
{
    if (!c || !path) return AGAL_ERR_PARAM;
    const int ML = c->max_levels;
    int rc;
    if (ML > 1) {
        for (int L = ML - 2; L >= 0; L--)
            if ((rc = agal_average(c, L, AGAL_AVERAGE_GRID))) return rc;
        for (int L = 0; L < ML - 1; L++)
            if ((rc = agal_interpolate(c, L, AGAL_INTERP_INTERFACE))) return rc;
    }
    for (int L = 0; L < ML; L++)
        if ((rc = agal_refresh(c, L))) return rc;
    return agal_uniform_append(c, path, iter);
}
