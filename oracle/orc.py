"""ORACLE (test infrastructure only): ctypes binding of oracle/liborc.so.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU baseline; never
by the agal_b200 package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liborc.so"


def build(force: bool = False) -> Path:
    srcs = list(HERE.glob("*.c")) + list(HERE.glob("*.h")) + [HERE.parent / "include" / "agal_b200.h"]
    if force or not LIB_PATH.exists() or any(s.stat().st_mtime > LIB_PATH.stat().st_mtime for s in srcs):
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "all"], check=True, env=env)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        from agal_b200._lib import AgalParams
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER(AgalParams)
        protos = [
            ("orc_create", C.c_void_p, [P, C.c_int64, C.c_int]),
            ("orc_destroy", None, [C.c_void_p]),
            ("orc_set_threads", None, [C.c_int]),
            ("orc_get_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
            ("orc_set_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]),
            ("orc_set_ic", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_refresh", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_collide", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_impose_bc", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_stream", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_advance", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_interpolate", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
            ("orc_average", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
            ("orc_ref_criteria", C.c_int, [C.c_void_p]),
            ("orc_refine_coarsen", C.c_int, [C.c_void_p]),
            ("orc_refine_with_solution", C.c_int, [C.c_void_p]),
            ("orc_refine_near_wall", C.c_int, [C.c_void_p]),
            ("orc_advance_n", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_array_bytes", C.c_size_t, [C.c_void_p, C.c_int]),
            ("orc_dump", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
            ("orc_load", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
            ("orc_mass_momentum", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
            ("orc_set_geometry", C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
            ("orc_bins_info", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                        C.POINTER(C.c_int64)]),
            ("orc_bins_copy", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
            ("orc_voxelize_s1", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_update_solid_children", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_voxelize_s2", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_voxelize_s3", C.c_int, [C.c_void_p]),
            ("orc_link_lengths", C.c_int, [C.c_void_p, C.c_int]),
            ("orc_geometry_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
            ("orc_forces", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
        ]
        for name, res, args in protos:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


# input.txt defaults of the reference's Parser (inc/parser.h:62-144),
# restated so that the oracle can be configured without the CUDA library
# (bench.py's reference arm loads nothing of agal_b200's native code).
_PARSER_INT_DEFAULTS = dict(
    MAX_LEVELS_WALL=5, MAX_LEVELS_INTERIOR=4, N_ITER_TOTAL=10 * 64, N_LEVEL_START=0, Nx=64, N_RESTART=1,
    G_LOADTYPE=0, G_PRINT=1, G_VIS_TREE=0, G_BIN_DENSITY=1, G_BIN_APPROACH=0, G_BIN_LEVELS=1, G_BIN_SPEC=1,
    G_BIN_MAKE_LINKS=0, PERIODIC_X=0, PERIODIC_Y=0, PERIODIC_Z=0, S_COLLISION=0, S_INTERP=1,
    S_INTERP_HYBRID=0, S_AVERAGE=0, S_CRITERION=0, S_LES=0, S_FORCE_ORDER=0, S_FORCE_TYPE=0, S_BC_TYPE=0,
    P_REFINE=32, N_PROBE=0, N_PROBE_DENSITY=4, N_PROBE_FREQUENCY=32, N_PROBE_FORCE=0, N_PROBE_F_START=0,
    N_PROBE_F_FREQUENCY=16, N_PROBE_AVE=0, N_PROBE_AVE_FREQUENCY=1, N_PROBE_AVE_START=100 * 64,
    N_PRINT_LEVELS=2, N_PRINT_LEVELS_VTHB=0, N_PRINT_LEVELS_PATCH=2, N_PRINT_LEVELS_IMAGE=2, P_OUTPUT=1 * 64,
    N_OUTPUT=10, N_OUTPUT_START=0, VOL_I_MIN=0, VOL_I_MAX=64, VOL_J_MIN=0, VOL_J_MAX=64, VOL_K_MIN=0,
    VOL_K_MAX=64, USE_CPU=1)
_PARSER_DBL_DEFAULTS = dict(
    L_c=1.0, L_fy=1.0, L_fz=1.0, v0=1.5625e-5, G_NEAR_WALL_DISTANCE=0.05, s1=1.19, s2=1.40, s3=1.20, s4=1.20,
    s5=1.20, s6=1.98, V_PROBE_TOL=1e-4, N_REFINE_START=-3.0, N_REFINE_INC=1.0, N_REFINE_MAX=1.0,
    S_FORCEVOLUME_Xm=0.0, S_FORCEVOLUME_XM=0.0, S_FORCEVOLUME_Ym=0.0, S_FORCEVOLUME_YM=0.0,
    S_FORCEVOLUME_Zm=0.0, S_FORCEVOLUME_ZM=0.0)
_PARSER_STR_DEFAULTS = dict(I_DIR_NAME="../input/", P_DIR_NAME="../out/TEST_UPLOAD/",
                            G_FILENAME="bunny_ascii.stl")


def default_params(**kw):
    """agal_params with the reference's input.txt defaults and the solver
    selections of its shipped build (D2Q9 BGK, cubic interpolation, main.cu:55;
    FP32; no hook preset; u_ref = the custom.h literal 0.05), then ``kw``.
    Field for field what agal_params_default gives (tests/test_abi.py)."""
    from agal_b200._lib import AgalParams   # the Python structure only
    p = AgalParams()
    for k, v in _PARSER_INT_DEFAULTS.items():
        setattr(p, k, v)
    for k, v in _PARSER_DBL_DEFAULTS.items():
        setattr(p, k, v)
    for k, v in _PARSER_STR_DEFAULTS.items():
        setattr(p, k, v.encode())
    p.velocity_set, p.collision, p.interp_order, p.storage = 0, 0, 2, 0
    p.bc_preset = p.ic_preset = p.region_preset = 0
    p.ref_pct_hi, p.ref_pct_lo, p.u_ref, p.ic_noise, p.seed = 0.9, 0.5, 0.05, 0.0, 0
    p.n_maxcblocks, p.mem_frac, p.device = 0, 0.975, -1
    p.half_rounding = 0   # stochastic
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v.encode() if isinstance(v, str) else v)
    return p


class OracleCase:
    """CPU oracle case with the same array selectors as agal_b200.Case."""

    def __init__(self, params, n_maxcblocks: int, fp64: bool = False, threads: int = 0):
        self._lib = lib()
        if threads:
            self._lib.orc_set_threads(threads)
        self._h = self._lib.orc_create(C.byref(params), n_maxcblocks, 1 if fp64 else 0)
        if not self._h:
            raise RuntimeError("orc_create failed")
        self.params = params
        self.dim = 2 if params.velocity_set == 0 else 3
        self.Q = {0: 9, 1: 19, 2: 27}[params.velocity_set]

    def close(self):
        if getattr(self, "_h", None):
            self._lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        if rc != 0:
            raise RuntimeError(f"oracle call failed: {rc}")

    def counts(self):
        n_ids = (C.c_int * 17)()
        id_max = (C.c_int * 17)()
        n_gaps = C.c_int()
        nmb = C.c_int64()
        ml = C.c_int()
        self._c(self._lib.orc_get_counts(self._h, n_ids, id_max, C.byref(n_gaps), C.byref(nmb), C.byref(ml)))
        L = ml.value
        return {"n_ids": list(n_ids[: L + 1]), "id_max": list(id_max[: L + 1]), "n_gaps": n_gaps.value,
                "n_maxcblocks": nmb.value, "max_levels": L}

    def set_counts(self, n_ids, id_max, n_gaps):
        ml = self.counts()["max_levels"]
        a = (C.c_int * (ml + 1))(*[int(v) for v in n_ids[: ml + 1]])
        b = (C.c_int * (ml + 1))(*[int(v) for v in id_max[: ml + 1]])
        self._c(self._lib.orc_set_counts(self._h, a, b, int(n_gaps)))

    def set_ic(self, L=0):
        self._c(self._lib.orc_set_ic(self._h, L))

    def refresh(self, L=0):
        self._c(self._lib.orc_refresh(self._h, L))

    def advance(self, L=None):
        self._c(self._lib.orc_advance(self._h, self.params.N_LEVEL_START if L is None else L))

    def advance_n(self, n):
        self._c(self._lib.orc_advance_n(self._h, n))

    def interpolate(self, L, var):
        self._c(self._lib.orc_interpolate(self._h, L, var))

    def average(self, L, var):
        self._c(self._lib.orc_average(self._h, L, var))

    def ref_criteria(self):
        self._c(self._lib.orc_ref_criteria(self._h))

    def refine_coarsen(self):
        self._c(self._lib.orc_refine_coarsen(self._h))

    def refine_with_solution(self):
        self._c(self._lib.orc_refine_with_solution(self._h))

    def refine_near_wall(self):
        self._c(self._lib.orc_refine_near_wall(self._h))

    def mass_momentum(self):
        out = (C.c_double * 4)()
        self._c(self._lib.orc_mass_momentum(self._h, out))
        return np.array(out[: self.dim + 1])

    def set_geometry(self, faces):
        """faces: (n, 3, 3) or (n, 9) float32, vertex coordinates per face."""
        f = np.ascontiguousarray(np.asarray(faces, dtype=np.float32).reshape(-1, 9))
        self._c(self._lib.orc_set_geometry(self._h, f.ctypes.data_as(C.c_void_p), int(f.shape[0])))

    def bins(self, level):
        """CSR bins (n, N, ids) of a voxelizer bin level, or of the link bins for level=-1."""
        dens, nb, ne = C.c_int(), C.c_int(), C.c_int64()
        self._c(self._lib.orc_bins_info(self._h, level, C.byref(dens), C.byref(nb), C.byref(ne)))
        n = np.empty(nb.value, np.int32)
        N = np.empty(nb.value, np.int32)
        ids = np.empty(max(ne.value, 1), np.int32)
        self._c(self._lib.orc_bins_copy(self._h, level, n.ctypes.data_as(C.c_void_p), N.ctypes.data_as(C.c_void_p),
                                        ids.ctypes.data_as(C.c_void_p)))
        return dens.value, n, N, ids[: ne.value]

    def voxelize_s1(self, L):
        self._c(self._lib.orc_voxelize_s1(self._h, L))

    def update_solid_children(self, L):
        self._c(self._lib.orc_update_solid_children(self._h, L))

    def voxelize_s2(self, L):
        self._c(self._lib.orc_voxelize_s2(self._h, L))

    def voxelize_s3(self):
        self._c(self._lib.orc_voxelize_s3(self._h))

    def link_lengths(self, L):
        self._c(self._lib.orc_link_lengths(self._h, L))

    def geometry_counts(self):
        out = (C.c_int64 * 4)()
        self._c(self._lib.orc_geometry_counts(self._h, out))
        return dict(n_faces=out[0], n_solida=out[1], n_solidb=out[2], n_maxcells_b=out[3])

    def forces(self):
        out = (C.c_double * 6)()
        self._c(self._lib.orc_forces(self._h, out))
        return np.array(out[:])

    def dump(self, which):
        dt = np.float64 if which in (0, 1, 14) else (np.float32 if which in (3, 13) else np.int32)
        n = self._lib.orc_array_bytes(self._h, which)
        out = np.empty(n // np.dtype(dt).itemsize, dtype=dt)
        self._c(self._lib.orc_dump(self._h, which, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def load(self, which, arr):
        dt = np.float64 if which in (0, 1) else (np.float32 if which == 3 else np.int32)
        a = np.ascontiguousarray(arr, dtype=dt)
        self._c(self._lib.orc_load(self._h, which, a.ctypes.data_as(C.c_void_p), a.nbytes))
