"""Triangle surfaces for the voxelizer: a seeded icosphere and ASCII STL I/O.

Faces are float32 arrays of shape (n_faces, 3, 3): face j has vertices
faces[j, 0], faces[j, 1], faces[j, 2] with (x, y, z) in the unit-length
domain coordinates of the solver (L_c = 1).  The winding is outward for the
icosphere; the voxelizer classifies cells by the sign of the unit normal
(v2 - v1) x (v3 - v1), as Cu_Voxelize_V1 does (mesh_voxelizer_voxelize.cu:203).

The STL reader follows Geometry::G_ImportSTL_ASCII (geometry_import.cu:11-83):
one facet per seven lines, vertices parsed as float, and triangles with two
equal vertices dropped.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

__all__ = ["icosphere", "write_stl_ascii", "read_stl_ascii", "face_soa"]


def _icosahedron() -> tuple[np.ndarray, list[tuple[int, int, int]]]:
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
         (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
         (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
         (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    return v, f


def icosphere(subdivisions: int, radius: float, centre, seed: int = 0) -> np.ndarray:
    """Unit icosahedron refined `subdivisions` times (20 * 4^k faces, new
    vertices projected to the sphere), turned by a seeded random rotation so
    that no face is aligned with the lattice, scaled to `radius` and moved to
    `centre`.  Returns float32 faces (n, 3, 3) with outward winding."""
    verts, faces = _icosahedron()
    verts = [tuple(p) for p in verts]
    for _ in range(int(subdivisions)):
        cache: dict[tuple[int, int], int] = {}

        def mid(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            if key not in cache:
                m = (np.asarray(verts[a]) + np.asarray(verts[b])) / 2.0
                m /= np.linalg.norm(m)
                verts.append(tuple(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.asarray(verts, dtype=np.float64)
    rng = np.random.default_rng(seed)
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q *= np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    V = V @ q.T
    tri = V[np.asarray(faces)]                                   # (n, 3, 3)
    # Outward winding: the normal must point away from the centre.
    nrm = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    flip = np.einsum("ij,ij->i", nrm, tri.mean(axis=1)) < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    tri = tri * float(radius) + np.asarray(centre, dtype=np.float64)[None, None, :]
    return tri.astype(np.float32)


def write_stl_ascii(path, faces: np.ndarray, name: str = "agal") -> None:
    """ASCII STL with every coordinate printed exactly (9 significant digits
    round-trip a float32)."""
    faces = np.asarray(faces, dtype=np.float32)
    lines = [f"solid {name}"]
    for tri in faces:
        n = np.cross(tri[1].astype(np.float64) - tri[0], tri[2].astype(np.float64) - tri[0])
        nn = np.linalg.norm(n)
        n = n / nn if nn > 0 else n
        lines.append(f"  facet normal {n[0]:.9e} {n[1]:.9e} {n[2]:.9e}")
        lines.append("    outer loop")
        for v in tri:
            lines.append(f"      vertex {float(v[0]):.9e} {float(v[1]):.9e} {float(v[2]):.9e}")
        lines.append("    endloop")
        lines.append("  endfacet")
    lines.append(f"endsolid {name}")
    Path(path).write_text("\n".join(lines) + "\n")


def read_stl_ascii(path) -> np.ndarray:
    """Faces of an ASCII STL, degenerate triangles (two equal vertices)
    dropped, as geometry_import.cu:51-68 does."""
    out = []
    cur: list[list[float]] = []
    for ln in Path(path).read_text().splitlines():
        w = ln.split()
        if w and w[0] == "vertex":
            cur.append([np.float32(w[1]), np.float32(w[2]), np.float32(w[3])])
            if len(cur) == 3:
                a, b, c = (tuple(x) for x in cur)
                if a != b and a != c and b != c:
                    out.append(cur)
                cur = []
    return np.asarray(out, dtype=np.float32).reshape(-1, 3, 3)


def face_soa(faces: np.ndarray) -> np.ndarray:
    """Rows v1x, v1y, v1z, v2x, ..., v3z of shape (9, n_faces), the first nine
    rows of the reference's geom_f_face_X (geometry_init.cu:139-149)."""
    f = np.asarray(faces, dtype=np.float32).reshape(-1, 9)
    return np.ascontiguousarray(f.T)


# ---- the library's host-side import (the reference's import rules) --------
def _call_faces(fn, *args):
    import ctypes as C
    from . import _lib
    n = C.c_longlong()
    rc = fn(*args, None, 0, C.byref(n))
    if rc != _lib.OK:
        raise _lib.AgalError(rc, fn.__name__)
    out = np.zeros((n.value, 9), np.float32)
    rc = fn(*args, out.ctypes.data_as(C.c_void_p), n.value, C.byref(n))
    if rc != _lib.OK:
        raise _lib.AgalError(rc, fn.__name__)
    return out


def import_stl(path) -> np.ndarray:
    """ASCII STL read as the reference reads it (agal_geometry_read_stl): (n, 9) float32."""
    from . import _lib
    return _call_faces(_lib.lib().agal_geometry_read_stl, str(path).encode())


def import_text(params, path) -> np.ndarray:
    """The primitives of a geometry.txt (agal_geometry_read_text): (n, 9) float32."""
    import ctypes as C
    from . import _lib
    return _call_faces(_lib.lib().agal_geometry_read_text, C.byref(params), str(path).encode())


def refine_length(params, faces) -> np.ndarray:
    """Faces split as G_RefineFaces_Length splits them (agal_geometry_refine_length)."""
    import ctypes as C
    from . import _lib
    f = np.ascontiguousarray(faces, np.float32).reshape(-1, 9)
    n = C.c_longlong(len(f))
    L = _lib.lib()
    buf = f.copy()
    rc = L.agal_geometry_refine_length(C.byref(params), buf.ctypes.data_as(C.c_void_p), len(buf), C.byref(n))
    if rc == _lib.ERR_PARAM and n.value > len(buf):
        buf = np.zeros((n.value, 9), np.float32)
        buf[: len(f)] = f
        n = C.c_longlong(len(f))
        rc = L.agal_geometry_refine_length(C.byref(params), buf.ctypes.data_as(C.c_void_p), len(buf), C.byref(n))
    if rc != _lib.OK:
        raise _lib.AgalError(rc, "agal_geometry_refine_length")
    return buf[: n.value]
