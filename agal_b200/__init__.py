"""agal_b200 - B200-native octree-AMR lattice Boltzmann time step.

Python mirror of the reference's host interface (Parser, Mesh, Solver_LBM of
AGAL: inc/parser.h, inc/mesh.h, inc/solver_lbm.h) over the C ABI of
libagal_b200.so.  Every numerical operation runs in the CUDA library; this
module only marshals parameters and host buffers.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import AgalError, AgalParams

__all__ = ["Parser", "Case", "Batch", "Learner", "Mesh", "Solver_LBM", "AgalError", "AgalParams", "default_params"]


def _check(rc: int, ctx: Optional[C.c_void_p] = None) -> None:
    if rc != _lib.OK:
        msg = _lib.lib().agal_last_error(ctx)
        raise AgalError(rc, msg.decode() if msg else "")


def default_params(**kw) -> AgalParams:
    """agal_params with the reference defaults (parser.h:62-144), then ``kw``."""
    p = AgalParams()
    _check(_lib.lib().agal_params_default(C.byref(p)))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        if isinstance(v, str):
            v = v.encode()
        setattr(p, k, v)
    return p


class Parser:
    """input.txt reader with the reference's rules (inc/parser.h:58-183)."""

    def __init__(self, input_file_directory: Optional[str] = None, params: Optional[AgalParams] = None):
        self.params = params if params is not None else default_params()
        self.input_file_directory = input_file_directory
        if input_file_directory is not None:
            _check(_lib.lib().agal_params_read(input_file_directory.encode(), C.byref(self.params)))

    @property
    def params_int(self) -> dict:
        return {k: getattr(self.params, k) for k in _lib.INT_KEYS}

    @property
    def params_dbl(self) -> dict:
        return {k: getattr(self.params, k) for k in _lib.DBL_KEYS}

    @property
    def params_str(self) -> dict:
        return {k: getattr(self.params, k).decode() for k in _lib.STR_KEYS}

    def set(self, key: str, value) -> None:
        _check(_lib.lib().agal_params_set(C.byref(self.params), key.encode(), str(value).encode()))


class Case:
    """One simulation case: an agal_ctx and its device arrays."""

    def __init__(self, params: AgalParams):
        self._lib = _lib.lib()
        self.params = params
        h = C.c_void_p()
        rc = self._lib.agal_ctx_create(C.byref(params), C.byref(h))
        if rc != _lib.OK:
            raise AgalError(rc, self._lib.agal_last_error(None).decode())
        self._h = h
        self.dim = 2 if params.velocity_set == _lib.D2Q9 else 3
        self.Q = {_lib.D2Q9: 9, _lib.D3Q19: 19, _lib.D3Q27: 27}[params.velocity_set]
        self.M_CBLOCK = 16 if self.dim == 2 else 64
        self.N_Q_max = 9 if self.dim == 2 else 27

    # -- life cycle -----------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.agal_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc: int) -> None:
        _check(rc, self._h)

    # -- counts ---------------------------------------------------------
    def counts(self) -> dict:
        n_ids = (C.c_int * 17)()
        id_max = (C.c_int * 17)()
        n_gaps = C.c_int()
        nmb = C.c_int64()
        ml = C.c_int()
        self._c(self._lib.agal_get_counts(self._h, n_ids, id_max, C.byref(n_gaps), C.byref(nmb), C.byref(ml)))
        L = ml.value
        return {"n_ids": list(n_ids[: L + 1]), "id_max": list(id_max[: L + 1]), "n_gaps": n_gaps.value,
                "n_maxcblocks": nmb.value, "max_levels": L}

    def set_counts(self, n_ids, id_max, n_gaps: int) -> None:
        """Restore n_ids / id_max / n_gaps after agal_load (restart)."""
        ml = self.counts()["max_levels"]
        a = (C.c_int * (ml + 1))(*[int(v) for v in n_ids[: ml + 1]])
        b = (C.c_int * (ml + 1))(*[int(v) for v in id_max[: ml + 1]])
        self._c(self._lib.agal_set_counts(self._h, a, b, int(n_gaps)))

    # -- solver entry points -------------------------------------------
    def set_ic(self, L: int = 0) -> None:
        self._c(self._lib.agal_set_ic(self._h, L))

    def set_ic_all(self) -> None:
        for L in range(self.counts()["max_levels"]):
            self.set_ic(L)

    def refresh(self, L: int = 0) -> None:
        self._c(self._lib.agal_refresh(self._h, L))

    def advance(self, L: Optional[int] = None) -> None:
        if L is None:
            L = self.params.N_LEVEL_START
        self._c(self._lib.agal_advance(self._h, L))

    def advance_n(self, n: int, use_graph: bool = True) -> None:
        self._c(self._lib.agal_advance_n(self._h, n, 1 if use_graph else 0))

    def sync(self) -> None:
        self._c(self._lib.agal_sync(self._h))

    # -- multi-level mesh ------------------------------------------------
    def interpolate(self, L: int, var: int = _lib.INTERP_INTERFACE) -> None:
        self._c(self._lib.agal_interpolate(self._h, L, var))

    def average(self, L: int, var: int = _lib.AVERAGE_GRID) -> None:
        self._c(self._lib.agal_average(self._h, L, var))

    def ref_criteria(self) -> None:
        self._c(self._lib.agal_ref_criteria(self._h))

    def refine_coarsen(self) -> None:
        self._c(self._lib.agal_refine_coarsen(self._h))

    def refine_with_solution(self) -> None:
        self._c(self._lib.agal_refine_with_solution(self._h))

    def refine_near_wall(self) -> None:
        self._c(self._lib.agal_refine_near_wall(self._h))

    def mesh_ref_criteria(self, L: int, var: int = _lib.MESH_REF_NW_CASES) -> None:
        self._c(self._lib.agal_mesh_ref_criteria(self._h, int(L), int(var)))

    def freeze_refined_cells(self, var: int = 0) -> None:
        self._c(self._lib.agal_freeze_refined_cells(self._h, int(var)))

    def refine_stats(self) -> dict:
        it, nr, nc = C.c_longlong(), C.c_int(), C.c_int()
        self._c(self._lib.agal_refine_stats(self._h, C.byref(it), C.byref(nr), C.byref(nc)))
        return {"iter": it.value, "n_refined": nr.value, "n_coarsened": nc.value}

    def graph_stats(self) -> dict:
        b, u = C.c_longlong(), C.c_longlong()
        self._c(self._lib.agal_graph_stats(self._h, C.byref(b), C.byref(u)))
        return {"builds": b.value, "updates": u.value}

    STEP_VARIANTS = {1: "1 cell/thread", 2: "2 cells/thread", 3: "TMA-staged persistent pipeline",
                     4: "1 row of 4 cells/thread, vector loads and stores",
                     5: "root-level tile of 8x8 blocks per CTA, gathered whole-block stores (2D)",
                     6: "root-level push tile of 8x4 blocks per CTA, shared-memory pushes, 16-byte row stores (2D)"}

    def autotune(self, L: int = 0, reps: int = 5) -> dict:
        """Pick the step kernel variant by timing each one (state unchanged)."""
        n = len(self.STEP_VARIANTS)
        ms = (C.c_float * n)()
        v = C.c_int()
        self._c(self._lib.agal_autotune(self._h, L, reps, ms, C.byref(v)))
        return {"variant": v.value, "name": self.STEP_VARIANTS[v.value], "ms": [ms[i] for i in range(n)]}

    def set_tuning(self, variant: int) -> None:
        self._c(self._lib.agal_set_tuning(self._h, variant))

    def stream_ptr(self) -> int:
        """The library's cudaStream_t for this case, as an integer."""
        s = C.c_void_p()
        self._c(self._lib.agal_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def mass_momentum(self) -> np.ndarray:
        out = (C.c_double * 4)()
        self._c(self._lib.agal_mass_momentum(self._h, out))
        return np.array(out[: self.dim + 1])

    def mass_momentum_async(self, out: np.ndarray) -> None:
        """Enqueue mass_momentum into out[0:4] (float64, ideally pinned);
        valid after sync()."""
        if out.dtype != np.float64 or out.size < 4 or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of at least 4 values")
        self._c(self._lib.agal_mass_momentum_async(self._h, out.ctypes.data_as(C.c_void_p)))

    def render_prepared(self) -> dict:
        """The uniform-grid fields after M_Advance_PrintData's preparation
        (grid averages, interface interpolations, macros of every level), as
        agal_uniform_frame writes them."""
        ml = self.counts()["max_levels"]
        for L in range(ml - 2, -1, -1):
            self.average(L, _lib.AVERAGE_GRID)
        for L in range(ml - 1):
            self.interpolate(L, _lib.INTERP_INTERFACE)
        for L in range(ml):
            self.refresh(L)
        return self.render_uniform()

    def mass_momentum_noalloc(self) -> np.ndarray:
        """mass_momentum with a fixed static device scratch (allocates nothing)."""
        out = (C.c_double * 4)()
        self._c(self._lib.agal_mass_momentum_noalloc(self._h, out))
        return np.array(out[: self.dim + 1])

    # -- checkpoint / restart (the reference's restart.bin) -------------
    def restart_save(self, path: str, iter: Optional[int] = None) -> None:
        """Write restart.bin; iter = index of the last coarse step taken
        (default: the library's own count - 1)."""
        if iter is None:
            iter = self.refine_stats()["iter"] - 1
        self._c(self._lib.agal_restart_save(self._h, str(path).encode(), int(iter)))

    def restart_load(self, path: str) -> int:
        """Load a restart.bin; returns the coarse-step counter stored in it."""
        it = C.c_int()
        self._c(self._lib.agal_restart_load(self._h, str(path).encode(), C.byref(it)))
        return it.value

    # -- headless uniform-grid output (out_direct.dat) -------------------
    def uniform_dims(self) -> tuple:
        d = (C.c_int * 3)()
        self._c(self._lib.agal_uniform_dims(self._h, d))
        return d[0], d[1], d[2]

    def render_uniform(self) -> dict:
        """rho, u, v, w, level, block ID on the output grid ([nz][ny][nx]) from
        the current macros (refresh every level first)."""
        nx, ny, nz = self.uniform_dims()
        out = np.empty(6 * nx * ny * nz, np.float64)
        self._c(self._lib.agal_uniform_render(self._h, out.ctypes.data_as(C.c_void_p), out.size))
        f = out.reshape(6, nz, ny, nx)
        return dict(zip(("rho", "u", "v", "w", "level", "block"), f))

    def uniform_header(self, path: str) -> None:
        self._c(self._lib.agal_uniform_header(self._h, str(path).encode()))

    def uniform_frame(self, path: str, iter: int) -> None:
        self._c(self._lib.agal_uniform_frame(self._h, str(path).encode(), int(iter)))

    def uniform_append(self, path: str, iter: int) -> None:
        self._c(self._lib.agal_uniform_append(self._h, str(path).encode(), int(iter)))

    # -- geometry -------------------------------------------------------
    def set_geometry(self, faces) -> None:
        """Attach a triangle surface: faces (n, 3, 3) or (n, 9) float32 in
        unit-length coordinates; builds the face bins on the device."""
        f = np.ascontiguousarray(np.asarray(faces, dtype=np.float32).reshape(-1, 9))
        self._c(self._lib.agal_set_geometry(self._h, f.ctypes.data_as(C.c_void_p), int(f.shape[0])))

    def bins(self, level: int):
        """(density, n, N, ids) of voxelizer bin level `level`, or of the link bins for level -1."""
        dens, nb, ne = C.c_int(), C.c_int(), C.c_longlong()
        self._c(self._lib.agal_bins_get(self._h, level, C.byref(dens), C.byref(nb), C.byref(ne), None, None, None))
        n = np.empty(nb.value, np.int32)
        N = np.empty(nb.value, np.int32)
        ids = np.empty(max(ne.value, 1), np.int32)
        self._c(self._lib.agal_bins_get(self._h, level, None, None, None, n.ctypes.data_as(C.c_void_p),
                                        N.ctypes.data_as(C.c_void_p), ids.ctypes.data_as(C.c_void_p)))
        return dens.value, n, N, ids[: ne.value]

    def voxelize_s1(self, L: int) -> None:
        self._c(self._lib.agal_voxelize_s1(self._h, L))

    def update_solid_children(self, L: int) -> None:
        self._c(self._lib.agal_update_solid_children(self._h, L))

    def voxelize_s2(self, L: int) -> None:
        self._c(self._lib.agal_voxelize_s2(self._h, L))

    def voxelize_s3(self) -> None:
        self._c(self._lib.agal_voxelize_s3(self._h))

    def link_lengths(self, L: int) -> None:
        self._c(self._lib.agal_link_lengths(self._h, L))

    def geometry_counts(self) -> dict:
        out = (C.c_longlong * 4)()
        self._c(self._lib.agal_geometry_counts(self._h, out))
        return dict(n_faces=out[0], n_solida=out[1], n_solidb=out[2], n_maxcells_b=out[3])

    def forces(self) -> np.ndarray:
        """MEA force sums {Fpx, Fmx, Fpy, Fmy, Fpz, Fmz} (FP64); resets the partials."""
        out = (C.c_double * 6)()
        self._c(self._lib.agal_forces(self._h, out))
        return np.array(out[:])

    # -- arrays ---------------------------------------------------------
    _DTYPES = {_lib.ARR_F: np.float64, _lib.ARR_MACROS: np.float64, _lib.ARR_CBLOCK_F_X: np.float32,
               _lib.ARR_CELLS_F_X_B: np.float32, _lib.ARR_CBLOCK_F_FF: np.float64, _lib.ARR_NU_SGS: np.float64}

    def array_bytes(self, which: int) -> int:
        n = C.c_size_t()
        self._c(self._lib.agal_array_bytes(self._h, which, C.byref(n)))
        return n.value

    def dump(self, which: int) -> np.ndarray:
        dt = self._DTYPES.get(which, np.int32)
        out = np.empty(self.array_bytes(which) // np.dtype(dt).itemsize, dtype=dt)
        self._c(self._lib.agal_dump(self._h, which, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def load(self, which: int, arr: np.ndarray) -> None:
        dt = self._DTYPES.get(which, np.int32)
        a = np.ascontiguousarray(arr, dtype=dt)
        self._c(self._lib.agal_load(self._h, which, a.ctypes.data_as(C.c_void_p), a.nbytes))


class Batch:
    """Independent cases advanced together (agal_batch_*): one CUDA graph per
    coarse step; in work-list mode (the default where every case allows it)
    the fused steps of all cases run as one persistent kernel per phase over
    a global (case, chunk) list, otherwise each case is one graph branch.
    Each case ends where advancing it alone would have left it."""

    def __init__(self, cases):
        self._lib = _lib.lib()
        self.cases = list(cases)
        arr = (C.c_void_p * len(self.cases))(*[c._h for c in self.cases])
        h = C.c_void_p()
        rc = self._lib.agal_batch_create(arr, len(self.cases), C.byref(h))
        if rc != _lib.OK:
            raise AgalError(rc, "agal_batch_create")
        self._h = h

    def _c(self, rc: int) -> None:
        if rc != _lib.OK:
            raise AgalError(rc, self._lib.agal_batch_last_error(self._h).decode())

    def advance_n(self, n: int, use_graph: bool = True) -> None:
        self._c(self._lib.agal_batch_advance_n(self._h, n, 1 if use_graph else 0))

    def sync(self) -> None:
        self._c(self._lib.agal_batch_sync(self._h))

    def set_worklist(self, on: bool) -> None:
        self._c(self._lib.agal_batch_set_worklist(self._h, 1 if on else 0))

    def autotune(self, steps: int = 4) -> dict:
        """Time both launch modes (the cases advance) and keep the faster."""
        ms = (C.c_float * 2)()
        mode = C.c_int()
        self._c(self._lib.agal_batch_autotune(self._h, int(steps), ms, C.byref(mode)))
        return {"worklist": bool(mode.value), "ms_branches": ms[0], "ms_worklist": ms[1]}

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(self._lib.agal_batch_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.agal_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Learner:
    """Learned refinement predictor (agal_learn_*): a 3-layer convolutional
    network over each block's cells, trained on the GPU on snapshots that the
    plain percentile criterion labels, and coupled with a case's
    solution-based refinement."""

    N_OUT = 2

    def __init__(self, dim: int, seed: int = 0):
        self._lib = _lib.lib()
        h = C.c_void_p()
        rc = self._lib.agal_learn_create(dim, seed, C.byref(h))
        if rc != _lib.OK:
            raise AgalError(rc, "agal_learn_create")
        self._h = h
        self.dim = dim
        self.cells = 16 if dim == 2 else 64
        self.taps = 9 if dim == 2 else 27
        n = C.c_longlong()
        self._c(self._lib.agal_learn_num_params(self._h, C.byref(n)))
        self.num_params = n.value

    def _c(self, rc: int) -> None:
        if rc != _lib.OK:
            raise AgalError(rc, self._lib.agal_learn_last_error(self._h).decode())

    def shapes(self) -> dict:
        """Parameter blocks in storage order: name -> (rows, columns)."""
        T = self.taps
        k1p = (8 * T + 15) // 16 * 16
        return {"W1": (32, k1p), "b1": (32,), "W2": (32, 32 * T), "b2": (32,), "W3": (2, 32 * T), "b3": (2,)}

    def get_params(self) -> np.ndarray:
        out = np.empty(self.num_params, np.float32)
        self._c(self._lib.agal_learn_get_params(self._h, out.ctypes.data_as(C.c_void_p), out.size))
        return out

    def set_params(self, w) -> None:
        a = np.ascontiguousarray(w, dtype=np.float32)
        self._c(self._lib.agal_learn_set_params(self._h, a.ctypes.data_as(C.c_void_p), a.size))

    def record(self, case: Case) -> None:
        self._c(self._lib.agal_learn_record(self._h, case._h))

    def label(self, case: Case) -> None:
        self._c(self._lib.agal_learn_label(self._h, case._h))

    def counts(self) -> dict:
        out = (C.c_longlong * 6)()
        self._c(self._lib.agal_learn_counts(self._h, out))
        keys = ("snapshots", "labelled", "regrids", "judged", "plain_refine", "missed")
        return dict(zip(keys, list(out)))

    def snapshot(self, k: int):
        """(X [n*cells][8], labels [n][2], weights [n]) of snapshot k."""
        n = C.c_int()
        self._c(self._lib.agal_learn_snapshot(self._h, k, C.byref(n), None, None, None))
        X = np.empty((n.value * self.cells, 8), np.float32)
        Y = np.empty((n.value, 2), np.float32)
        W = np.empty(n.value, np.float32)
        self._c(self._lib.agal_learn_snapshot(self._h, k, C.byref(n), X.ctypes.data_as(C.c_void_p),
                                              Y.ctypes.data_as(C.c_void_p), W.ctypes.data_as(C.c_void_p)))
        return X, Y, W

    def decisions(self, k: int) -> np.ndarray:
        """The percentile rule's decisions [n][2] on snapshot k's own state."""
        n = C.c_int()
        self._c(self._lib.agal_learn_snapshot(self._h, k, C.byref(n), None, None, None))
        out = np.zeros((n.value, 2), np.float32)
        self._c(self._lib.agal_learn_snapshot_decisions(self._h, k, out.ctypes.data_as(C.c_void_p)))
        return out

    def set_class_weights(self, refine: float, coarsen: float) -> None:
        """Weights of the positive class (a mark) of the two outputs in the loss."""
        self._c(self._lib.agal_learn_set_class_weights(self._h, refine, coarsen))

    def balance_classes(self, first: int, last: int, cap: float = 50.0) -> tuple:
        """Set the class weights to the ratio of unmarked to marked blocks over
        the labelled snapshots [first, last), capped; returns them."""
        pos = np.zeros(2)
        tot = 0.0
        for k in range(first, last):
            _, Y, W = self.snapshot(k)
            pos += (Y * W[:, None]).sum(axis=0)
            tot += W.sum()
        w = tuple(float(min(cap, max(1.0, (tot - p) / p))) if p > 0 else 1.0 for p in pos)
        self.set_class_weights(*w)
        return w

    def gradients(self, k: int):
        """(loss, gradient) of labelled snapshot k at the current weights."""
        g = np.empty(self.num_params, np.float32)
        loss = C.c_double()
        self._c(self._lib.agal_learn_gradients(self._h, k, g.ctypes.data_as(C.c_void_p), g.size, C.byref(loss)))
        return loss.value, g

    def train(self, first: int, last: int, epochs: int, lr: float = 1e-3, seed: int = 0) -> float:
        loss = C.c_double()
        self._c(self._lib.agal_learn_train(self._h, first, last, epochs, lr, seed, C.byref(loss)))
        return loss.value

    def predict(self, k: int) -> np.ndarray:
        n = C.c_int()
        self._c(self._lib.agal_learn_snapshot(self._h, k, C.byref(n), None, None, None))
        out = np.zeros((n.value, 2), np.float32)
        self._c(self._lib.agal_learn_predict_snapshot(self._h, k, out.ctypes.data_as(C.c_void_p)))
        return out

    def attach(self, case: Case, mode: int, judge_every: int = 4, threshold: float = 0.5) -> None:
        """mode 1: collect labelled snapshots, 2: predict (judged), 0: detach."""
        rc = self._lib.agal_learn_attach(case._h, self._h if mode else None, mode, judge_every, threshold)
        if rc != _lib.OK:
            raise AgalError(rc, "agal_learn_attach")
        case._learner = self if mode else None
        self._attached = [c for c in getattr(self, "_attached", []) if c is not case] + ([case] if mode else [])

    def set_horizon(self, horizon: int) -> None:
        """Look-ahead: snapshots taken at a regrid are labelled with the rule's
        decisions at that regrid and the next horizon - 1, and predictions
        apply at the regrid they are made (0: the one-regrid-delayed mode).
        Set before collecting."""
        self._c(self._lib.agal_learn_set_horizon(self._h, int(horizon)))

    def set_implicit(self, on: bool) -> None:
        """Inference convolutions as implicit GEMMs (default) or through
        materialised im2col columns; the logits are identical."""
        self._c(self._lib.agal_learn_set_implicit(self._h, 1 if on else 0))

    def set_thresholds(self, refine: float, coarsen: float) -> None:
        """Probability thresholds of the two outputs in predict mode."""
        self._c(self._lib.agal_learn_set_thresholds(self._h, refine, coarsen))

    def calibrate_thresholds(self, first: int, last: int) -> tuple:
        """Thresholds at which the network marks, over the labelled snapshots
        [first, last), as many blocks as the labels do among the blocks a mark
        can apply to (unrefined below the finest level for refinement, refined
        for coarsening); returns them as probabilities (apply with
        set_thresholds after attach).  Coarsening is never looser than
        probability 1/2: a wrongly removed level costs accuracy, a wrongly
        added one only time."""
        zs, ys, cs = [], [], []
        for k in range(first, last):
            X, Y, W = self.snapshot(k)
            Xb = X.reshape(len(W), self.cells, 8)[:, 0, :]
            v = W > 0
            zs.append(self.predict(k)[v])
            ys.append(Y[v])
            cs.append(np.stack([(Xb[v, 6] == 0) & (Xb[v, 5] < 1.0 - 1e-6), Xb[v, 6] == 1], axis=1))
        z, y, cand = np.concatenate(zs), np.concatenate(ys), np.concatenate(cs)
        out = []
        for o in range(2):
            zo = np.sort(z[cand[:, o], o])[::-1]
            npos = int(y[cand[:, o], o].sum())
            t = 0.0 if npos == 0 or npos >= len(zo) else float(zo[npos - 1: npos + 1].mean())
            out.append(float(1.0 / (1.0 + np.exp(-t))))
        out[1] = max(out[1], 0.5)
        return tuple(min(max(x, 1e-6), 1 - 1e-6) for x in out)

    def close(self) -> None:
        if getattr(self, "_h", None):
            for case in getattr(self, "_attached", []):   # the cases must not keep a dangling predictor
                if getattr(case, "_h", None):
                    self._lib.agal_learn_attach(case._h, None, 0, 1, 0.5)
            self._attached = []
            self._lib.agal_learn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Mesh(Case):
    """Facade with the reference Mesh method names (inc/mesh.h)."""

    def __init__(self, parser: Parser):
        super().__init__(parser.params)
        self.parser = parser

    def M_Advance_Step(self) -> None:
        self.advance()

    def M_AdvanceLoop(self, n_iter: Optional[int] = None) -> None:
        """mesh_advance.cu:381-466 without output: near-wall refinement, then
        the coarse steps with solution-based refinement every P_REFINE."""
        n = self.params.N_ITER_TOTAL if n_iter is None else n_iter
        self.M_Advance_RefineNearWall()
        self.advance_n(n, use_graph=True)

    def M_Advance_RefineNearWall(self) -> None:
        self.refine_near_wall()

    def M_Advance_RefineWithSolution(self) -> None:
        self.refine_with_solution()

    def M_Restart(self, var: int, iter: Optional[int] = None) -> int:
        """mesh_restart.cu: var 0 saves <P_DIR_NAME>restart.bin, 1 loads it;
        returns the stored loop index."""
        path = self.params.P_DIR_NAME.decode() + "restart.bin"
        if var == 0:
            it = self.refine_stats()["iter"] - 1 if iter is None else iter
            self.restart_save(path, it)
            return it
        return self.restart_load(path)

    def M_RefineAndCoarsenBlocks(self) -> None:
        self.refine_coarsen()


class Solver_LBM:
    """Facade with the reference Solver_LBM method names (inc/solver_lbm.h:153-179)."""

    def __init__(self, mesh: Mesh):
        self.mesh = mesh

    def S_SetIC(self, i_dev: int, L: int) -> int:
        self.mesh.set_ic(L)
        return 0

    def S_RefreshVariables(self, i_dev: int, L: int, var: int = 0) -> int:
        self.mesh.refresh(L)
        return 0

    def S_Advance(self, i_dev: int, L: int, tmp=None) -> int:
        self.mesh.advance(L)
        return 0

    def S_Interpolate(self, i_dev: int, L: int, var: int) -> int:
        self.mesh.interpolate(L, var)
        return 0

    def S_Average(self, i_dev: int, L: int, var: int) -> int:
        self.mesh.average(L, var)
        return 0

    def S_ComputeRefCriteria(self, i_dev: int, L: int, var: int) -> int:
        self.mesh.ref_criteria()
        return 0
