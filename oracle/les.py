"""CPU restatement of the reference's LES eddy viscosity (test infrastructure
only: the product path is the CUDA kernel k_eddy).

Cu_ComputeEddyViscosity (src/solver_lbm/solver_lbm_kernels_les.cu:460-600):
per cell-block of 4^dim cells, the stored velocity is copied into a block
with a one-cell halo, the halo is extrapolated from the block itself
(ExtrapolateToHalo, inc/util_math.h:55-110: d_-1 = 4 d0 - 6 d1 + 4 d2 - d3
and mirrored at the far side), the velocity gradient is taken by central
differences (FinDiff_D1_Central, inc/util_math.h:116-120), and one of the
models gives nu_SGS (solver_lbm_kernels_les.cu:13-250):

- Smagorinsky: C_s^2 dx^2 sqrt(2 S:S), C_s = 0.1;
- WALE: C_w^2 dx^2 (Sd:Sd)^(3/2) / ((S:S)^(5/2) + (Sd:Sd)^(5/4)), C_w = 0.325,
  Sd the traceless symmetric part of grad(u) . grad(u);
- Vreman: c dx^2 sqrt(B_beta / (grad u : grad u)), c = 2.5 * 0.17^2,
  B = grad(u)^T grad(u) and B_beta its sum of principal 2x2 minors.

Evaluated in float64; the reference computes in FP32.
"""
import numpy as np

MODELS = {1: "smagorinsky", 2: "wale", 3: "vreman"}


def _halo_block(u: np.ndarray, dim: int) -> np.ndarray:
    """u: (n, 4, 4[, 4]) indexed [n, (K,) J, I] -> (n, 6, 6[, 6]) with the
    extrapolated faces (edges and corners are never read)."""
    n = u.shape[0]
    shape = (n,) + (6,) * dim
    h = np.zeros(shape)
    inner = (slice(None),) + (slice(1, 5),) * dim
    h[inner] = u

    def ext(d1, d2, d3, d4):
        return 4.0 * d1 - 6.0 * d2 + 4.0 * d3 - d4

    for ax in range(1, dim + 1):            # array axis: 1..dim
        def sl(i):
            idx = [slice(None)] + [slice(1, 5)] * dim
            idx[ax] = i
            return tuple(idx)
        h[sl(0)] = ext(h[sl(1)], h[sl(2)], h[sl(3)], h[sl(4)])
        h[sl(5)] = ext(h[sl(4)], h[sl(3)], h[sl(2)], h[sl(1)])
    return h


def velocity_gradient(U: np.ndarray, dx: float, dim: int) -> np.ndarray:
    """U: (n, dim, MC) velocity per block and cell (cell t = I + 4 J + 16 K).
    Returns G (n, 3, 3, MC): G[:, c, a] = d u_c / d x_a (zero beyond dim)."""
    n, MC = U.shape[0], U.shape[2]
    G = np.zeros((n, 3, 3, MC))
    for c in range(dim):
        u = U[:, c, :].reshape((n,) + (4,) * dim)     # [n, (K,) J, I]
        h = _halo_block(u, dim)
        for a in range(dim):
            ax = dim - a                              # x is the last array axis
            lo = [slice(None)] + [slice(1, 5)] * dim
            hi = list(lo)
            lo[ax] = slice(0, 4)
            hi[ax] = slice(2, 6)
            d = (h[tuple(hi)] - h[tuple(lo)]) / (2.0 * dx)
            G[:, c, a, :] = d.reshape(n, MC)
    return G


def eddy_viscosity(U: np.ndarray, dx: float, model: int, dim: int) -> np.ndarray:
    """nu_SGS (n, MC) of the reference's model 1 (Smagorinsky), 2 (WALE) or
    3 (Vreman) from the velocity U (n, dim, MC)."""
    G = velocity_gradient(U, dx, dim)
    S = 0.5 * (G + np.transpose(G, (0, 2, 1, 3)))
    F2 = np.einsum("nabt,nabt->nt", S, S)
    if model == 1:
        return np.where(F2 > 0, 0.1 ** 2 * dx * dx * np.sqrt(2.0 * np.maximum(F2, 0)), 0.0)
    if model == 2:
        g = np.einsum("nikt,nkjt->nijt", G, G)
        tr = np.einsum("niit->nt", g)
        D = 0.5 * (g + np.transpose(g, (0, 2, 1, 3)))
        for i in range(3):
            D[:, i, i, :] -= tr / 3.0
        if dim == 2:
            D[:, 2, 2, :] = 0.0                      # the 2D model sums the xy block only
        F1 = np.einsum("nabt,nabt->nt", D, D)
        ok = (F1 > 0) & (F2 > 0)
        F1c, F2c = np.where(ok, F1, 1.0), np.where(ok, F2, 1.0)
        v = 0.325 ** 2 * dx * dx * F1c ** 1.5 / (F2c ** 2.5 + F1c ** 1.25)
        return np.where(ok, v, 0.0)
    if model == 3:
        B = np.einsum("nikt,njkt->nijt", G, G)     # B_xy = ux vx + uy vy + uz vz
        Bb = (B[:, 0, 0] * B[:, 1, 1] - B[:, 0, 1] ** 2 + B[:, 0, 0] * B[:, 2, 2] - B[:, 0, 2] ** 2
              + B[:, 1, 1] * B[:, 2, 2] - B[:, 1, 2] ** 2)
        aa = np.einsum("nabt,nabt->nt", G, G)
        ok = aa > 0
        Bb = np.where(ok, Bb / np.where(ok, aa, 1.0), 0.0)
        return np.where(ok & (Bb > 0), 2.5 * 0.17 ** 2 * dx * dx * np.sqrt(np.maximum(Bb, 0)), 0.0)
    raise ValueError(model)
