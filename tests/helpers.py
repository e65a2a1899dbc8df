"""Shared helpers of the parity tests."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def tables():
    return json.loads((GOLDEN / "lattice_tables.json").read_text())


def brute_root_grid(dim, Nx, Ny, Nz, periodic=(0, 0, 0)):
    """Root-grid block neighbours by the literal padded-grid procedure of
    mesh_init.cu:354-500 (IDs x-fastest; z faces, then y faces, then x faces
    written last; periodic faces copy the opposite interior layer), using the
    golden direction table inc/mesh.h:468-472."""
    t = tables()
    bx, by = Nx // 4, Ny // 4
    bz = Nz // 4 if dim == 3 else 1
    Qmax = 9 if dim == 2 else 27
    c = np.array(t["MESH_C_2D"] + [0] * 9 if dim == 2 else t["MESH_C_3D"]).reshape(3, Qmax)
    gh = bz
    G = np.full((bx + 2, by + 2, gh + 2), -12345, dtype=np.int64)
    ctr = 0
    krange = range(1, bz + 1) if dim == 3 else [0]
    for k in krange:
        for j in range(1, by + 1):
            for i in range(1, bx + 1):
                G[i, j, k] = ctr
                ctr += 1
    if dim == 3:
        for j in range(by + 2):
            for i in range(bx + 2):
                if periodic[2]:
                    G[i, j, 0] = G[i, j, gh]
                    G[i, j, gh + 1] = G[i, j, 1]
                else:
                    G[i, j, 0] = -5
                    G[i, j, gh + 1] = -6
    kr = range(gh + 2) if dim == 3 else [0]
    for k in kr:
        for i in range(bx + 2):
            if periodic[1]:
                G[i, 0, k] = G[i, by, k]
                G[i, by + 1, k] = G[i, 1, k]
            else:
                G[i, 0, k] = -3
                G[i, by + 1, k] = -4
    for k in kr:
        for j in range(by + 2):
            if periodic[0]:
                G[0, j, k] = G[bx, j, k]
                G[bx + 1, j, k] = G[1, j, k]
            else:
                G[0, j, k] = -1
                G[bx + 1, j, k] = -2
    n = ctr
    nbr = np.zeros((Qmax, n), dtype=np.int64)
    onb = np.zeros(n, dtype=np.int64)
    for k in krange:
        for j in range(1, by + 1):
            for i in range(1, bx + 1):
                b = G[i, j, k]
                for p in range(Qmax):
                    kk = (k + c[2, p]) if dim == 3 else 0
                    nbr[p, b] = G[i + c[0, p], j + c[1, p], kk]
                onb[b] = int((nbr[:, b] < 0).any())
    return nbr, onb


def macros_from_F(F: np.ndarray, dim: int, Q: int, pb, cvec):
    """rho, u from populations in the reference slot layout F[slot, cell]
    (slot pb(p) holds f_p)."""
    f = F[np.asarray(pb)[:Q]]  # f[p] = F[pb(p)]
    rho = f.sum(axis=0)
    u = [(np.asarray(cvec[a][:Q])[:, None] * f).sum(axis=0) / rho for a in range(dim)]
    return rho, u


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt((b * b).sum())
    return float(np.sqrt(((a - b) ** 2).sum()) / (den if den > 0 else 1.0))


def lattice(Q: int):
    """(pb, c[3][Q], dim) from the golden tables."""
    t = tables()
    if Q == 9:
        c = np.array(t["V_CONN_ID_2D"]).reshape(3, 27)[:, :9]
        return t["LBMpb_D2Q9"], c, 2
    c = np.array(t["V_CONN_ID_3D"]).reshape(3, 27)[:, :Q]
    return (t["LBMpb_D3Q19"] if Q == 19 else t["LBMpb_D3Q27"]), c, 3
