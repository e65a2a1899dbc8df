"""ctypes binding of the C ABI declared in include/agal_b200.h.

The shared library agal_b200/libagal_b200.so is built in-tree by
``python -m agal_b200.build``.  There is no fallback: if the library is
missing or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libagal_b200.so"

# status codes
OK = 0
ERR_PARAM, ERR_OOM, ERR_GAPS, ERR_TIMEOUT, ERR_CUDA, ERR_IO, ERR_STATE, ERR_UNSUPPORTED = range(-1, -9, -1)
ERR_NAMES = {0: "OK", -1: "AGAL_ERR_PARAM", -2: "AGAL_ERR_OOM", -3: "AGAL_ERR_GAPS", -4: "AGAL_ERR_TIMEOUT",
             -5: "AGAL_ERR_CUDA", -6: "AGAL_ERR_IO", -7: "AGAL_ERR_STATE", -8: "AGAL_ERR_UNSUPPORTED"}

# enumerations
D2Q9, D3Q19, D3Q27 = 0, 1, 2
BGK, MRT = 0, 2
INTERP_LINEAR, INTERP_CUBIC = 0, 2
STORE_FP32, STORE_FP64, STORE_FP16, STORE_BF16 = 0, 1, 2, 3
ROUND_STOCHASTIC, ROUND_NEAREST = 0, 1
BC_NONE, BC_LDC2D, BC_LDC3D, BC_FPSC2D, BC_FPSC3D = 0, 1, 2, 3, 4
IC_REST, IC_UNIFORM = 0, 1
REGION_NONE, REGION_BOUNDARY, REGION_BOX = 0, 1, 2
CRITERION_VORTICITY, CRITERION_Q, CRITERION_PERCENTILE, CRITERION_LEARNED = 0, 1, 2, 3
INTERP_INTERFACE, INTERP_ADDED = 0, 1
AVERAGE_INTERFACE, AVERAGE_BLOCK, AVERAGE_GRID = 0, 1, 2
MESH_REF_NW_CASES, MESH_REF_UNIFORM, MESH_REF_SOLUTION = 0, 2, 3

ARR_F, ARR_MACROS, ARR_CELLS_ID_MASK, ARR_CBLOCK_F_X, ARR_CBLOCK_ID_MASK, ARR_CBLOCK_ID_NBR, \
    ARR_CBLOCK_ID_NBR_CHILD, ARR_CBLOCK_ID_ONB, ARR_CBLOCK_ID_REF, ARR_CBLOCK_LEVEL, ARR_ID_SET, \
    ARR_GAP_SET = range(12)
ARR_CBLOCK_ID_ONB_SOLID, ARR_CELLS_F_X_B, ARR_CBLOCK_F_FF, ARR_NU_SGS = 12, 13, 14, 15

INT_KEYS = ["MAX_LEVELS_WALL", "MAX_LEVELS_INTERIOR", "N_ITER_TOTAL", "N_LEVEL_START", "Nx", "N_RESTART",
            "PERIODIC_X", "PERIODIC_Y", "PERIODIC_Z",
            "G_LOADTYPE", "G_PRINT", "G_VIS_TREE", "G_BIN_DENSITY", "G_BIN_APPROACH", "G_BIN_LEVELS",
            "G_BIN_SPEC", "G_BIN_MAKE_LINKS",
            "S_COLLISION", "S_INTERP", "S_INTERP_HYBRID", "S_AVERAGE", "S_CRITERION", "S_LES",
            "S_FORCE_ORDER", "S_FORCE_TYPE", "S_BC_TYPE",
            "P_REFINE", "N_PROBE", "N_PROBE_DENSITY", "N_PROBE_FREQUENCY", "N_PROBE_FORCE",
            "N_PROBE_F_START", "N_PROBE_F_FREQUENCY",
            "N_PROBE_AVE", "N_PROBE_AVE_FREQUENCY", "N_PROBE_AVE_START",
            "N_PRINT_LEVELS", "N_PRINT_LEVELS_VTHB", "N_PRINT_LEVELS_PATCH", "N_PRINT_LEVELS_IMAGE",
            "P_OUTPUT", "N_OUTPUT", "N_OUTPUT_START",
            "VOL_I_MIN", "VOL_I_MAX", "VOL_J_MIN", "VOL_J_MAX", "VOL_K_MIN", "VOL_K_MAX", "USE_CPU"]
DBL_KEYS = ["L_c", "L_fy", "L_fz", "v0", "G_NEAR_WALL_DISTANCE", "s1", "s2", "s3", "s4", "s5", "s6",
            "V_PROBE_TOL", "N_REFINE_START", "N_REFINE_INC", "N_REFINE_MAX",
            "S_FORCEVOLUME_Xm", "S_FORCEVOLUME_XM", "S_FORCEVOLUME_Ym", "S_FORCEVOLUME_YM",
            "S_FORCEVOLUME_Zm", "S_FORCEVOLUME_ZM"]
STR_KEYS = ["I_DIR_NAME", "P_DIR_NAME", "G_FILENAME"]


class AgalParams(C.Structure):
    """Mirror of ``agal_params`` (include/agal_b200.h)."""
    _fields_ = ([(k, C.c_int) for k in INT_KEYS] + [(k, C.c_double) for k in DBL_KEYS] +
                [(k, C.c_char * 256) for k in STR_KEYS] +
                [("velocity_set", C.c_int), ("collision", C.c_int), ("interp_order", C.c_int),
                 ("storage", C.c_int), ("bc_preset", C.c_int), ("ic_preset", C.c_int),
                 ("region_preset", C.c_int), ("ref_pct_hi", C.c_double), ("ref_pct_lo", C.c_double),
                 ("u_ref", C.c_double), ("ic_noise", C.c_double), ("seed", C.c_uint64),
                 ("n_maxcblocks", C.c_int64), ("mem_frac", C.c_double), ("device", C.c_int),
                 ("half_rounding", C.c_int)])


# (name, restype, argtypes) of every exported entry point.
PROTOS = [
    ("agal_params_default", C.c_int, [C.POINTER(AgalParams)]),
    ("agal_params_size", C.c_size_t, []),
    ("agal_params_read", C.c_int, [C.c_char_p, C.POINTER(AgalParams)]),
    ("agal_params_set", C.c_int, [C.POINTER(AgalParams), C.c_char_p, C.c_char_p]),
    ("agal_ctx_create", C.c_int, [C.POINTER(AgalParams), C.POINTER(C.c_void_p)]),
    ("agal_ctx_destroy", C.c_int, [C.c_void_p]),
    ("agal_last_error", C.c_char_p, [C.c_void_p]),
    ("agal_get_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    ("agal_set_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]),
    ("agal_set_ic", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_refresh", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_advance", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_advance_n", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("agal_array_bytes", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]),
    ("agal_dump", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    ("agal_load", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]),
    ("agal_restart_save", C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    ("agal_restart_load", C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int)]),
    ("agal_uniform_dims", C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    ("agal_uniform_render", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    ("agal_uniform_header", C.c_int, [C.c_void_p, C.c_char_p]),
    ("agal_uniform_frame", C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    ("agal_uniform_append", C.c_int, [C.c_void_p, C.c_char_p, C.c_int]),
    ("agal_mass_momentum", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("agal_mass_momentum_noalloc", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("agal_mass_momentum_async", C.c_int, [C.c_void_p, C.c_void_p]),
    ("agal_sync", C.c_int, [C.c_void_p]),
    ("agal_get_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("agal_autotune", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    ("agal_set_tuning", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_interpolate", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("agal_average", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("agal_ref_criteria", C.c_int, [C.c_void_p]),
    ("agal_refine_coarsen", C.c_int, [C.c_void_p]),
    ("agal_refine_with_solution", C.c_int, [C.c_void_p]),
    ("agal_refine_near_wall", C.c_int, [C.c_void_p]),
    ("agal_mesh_ref_criteria", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("agal_freeze_refined_cells", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_refine_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("agal_graph_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    ("agal_set_geometry", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    ("agal_geometry_read_stl", C.c_int, [C.c_char_p, C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong)]),
    ("agal_geometry_read_text", C.c_int, [C.POINTER(AgalParams), C.c_char_p, C.c_void_p, C.c_longlong,
                                          C.POINTER(C.c_longlong)]),
    ("agal_geometry_refine_length", C.c_int, [C.POINTER(AgalParams), C.c_void_p, C.c_longlong,
                                              C.POINTER(C.c_longlong)]),
    ("agal_import_geometry", C.c_int, [C.c_void_p]),
    ("agal_bins_get", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_longlong), C.c_void_p, C.c_void_p, C.c_void_p]),
    ("agal_voxelize_s1", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_update_solid_children", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_voxelize_s2", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_voxelize_s3", C.c_int, [C.c_void_p]),
    ("agal_link_lengths", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_geometry_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("agal_forces", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("agal_learn_gemm_bf16", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
    ("agal_batch_create", C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)]),
    ("agal_batch_destroy", C.c_int, [C.c_void_p]),
    ("agal_batch_advance_n", C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    ("agal_batch_sync", C.c_int, [C.c_void_p]),
    ("agal_batch_get_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("agal_batch_last_error", C.c_char_p, [C.c_void_p]),
    ("agal_batch_set_worklist", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_batch_autotune", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    ("agal_learn_create", C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    ("agal_learn_destroy", C.c_int, [C.c_void_p]),
    ("agal_learn_last_error", C.c_char_p, [C.c_void_p]),
    ("agal_learn_num_params", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("agal_learn_get_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    ("agal_learn_set_params", C.c_int, [C.c_void_p, C.c_void_p, C.c_longlong]),
    ("agal_learn_record", C.c_int, [C.c_void_p, C.c_void_p]),
    ("agal_learn_label", C.c_int, [C.c_void_p, C.c_void_p]),
    ("agal_learn_counts", C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    ("agal_learn_snapshot", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_void_p, C.c_void_p, C.c_void_p]),
    ("agal_learn_gradients", C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_longlong, C.POINTER(C.c_double)]),
    ("agal_learn_train", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64,
                                   C.POINTER(C.c_double)]),
    ("agal_learn_predict_snapshot", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("agal_learn_snapshot_decisions", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("agal_learn_set_class_weights", C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    ("agal_learn_set_thresholds", C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    ("agal_learn_attach", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double]),
    ("agal_learn_set_horizon", C.c_int, [C.c_void_p, C.c_int]),
    ("agal_learn_set_implicit", C.c_int, [C.c_void_p, C.c_int]),
]

_lib = None


def lib() -> C.CDLL:
    """Load libagal_b200.so (raises if it is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m agal_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, res, args in PROTOS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        if L.agal_params_size() != C.sizeof(AgalParams):
            raise RuntimeError("agal_params layout mismatch between the library and the Python binding")
        _lib = L
    return _lib


class AgalError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code
