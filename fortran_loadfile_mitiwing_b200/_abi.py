"""ctypes view of include/lbm_b200.h, shared by the product library and the
CPU oracle (which takes the same lbm_params struct)."""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liblbmb200.so")

LBM_OK = 0
LBM_DONE = 1
LBM_ERR_ARG = -1
LBM_ERR_CUDA = -2
LBM_ERR_STATE = -3
LBM_ERR_IO = -4
LBM_ERR_SOLVER = -5
LBM_ERR_NONFINITE = -6
LBM_ERR_RANGE = -7
LBM_ERR_SIZE = -8
LBM_ERR_INDEX = -9
LBM_TIMING_KERNELS = 1
LBM_TIMING_SPAN = 2
LBM_RESIDUAL_MAX_ROWS = 16384

LBM_PREC_FP32 = 0
LBM_PREC_FP64 = 1
LBM_PREC_FP16 = 2
LBM_PREC_BF16 = 3
PRECISIONS = {"fp32": LBM_PREC_FP32, "fp64": LBM_PREC_FP64, "fp16": LBM_PREC_FP16, "bf16": LBM_PREC_BF16}

LBM_FLAG_DENSE_SOLVE = 1

LBM_DELTA_PESKIN4 = 0
LBM_DELTA_SMOOTH = 1

STATUS_NAMES = {0: "LBM_OK", 1: "LBM_DONE", -1: "LBM_ERR_ARG", -2: "LBM_ERR_CUDA", -3: "LBM_ERR_STATE",
                -4: "LBM_ERR_IO", -5: "LBM_ERR_SOLVER", -6: "LBM_ERR_NONFINITE", -7: "LBM_ERR_RANGE",
                -8: "LBM_ERR_SIZE", -9: "LBM_ERR_INDEX"}

# device status bits of the kernels (csrc/lbm_common.cuh), for
# lbm_describe_status
LBM_ST_RANGE = 0x1
LBM_ST_SOLVER = 0x2
LBM_ST_NONFINITE = 0x4
LBM_ST_OVERFLOW = 0x8
LBM_ST_TIMEOUT = 0x10
LBM_ST_INDEX_KERNELS = {0x100: "ib_interp", 0x200: "ib_assemble", 0x400: "ib_factor", 0x800: "ib_solve",
                        0x1000: "ib_tile_scatter", 0x2000: "ib_tile_sort", 0x4000: "ib_tile_update",
                        0x8000: "ib_forces", 0x10000: "ib_residual", 0x20000: "kf_tma"}


class LbmParams(C.Structure):
    """struct lbm_params (include/lbm_b200.h)."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("wing_count", C.c_int32), ("points_per_wing", C.c_int32),
        ("delta_kernel", C.c_int32), ("precision", C.c_int32),
        ("flags", C.c_int32), ("reserved", C.c_int32),
        ("scale", C.c_double), ("ox", C.c_double), ("oy", C.c_double),
        ("uu", C.c_double), ("re", C.c_double),
        ("s", C.c_double * 9),
        ("xc", C.c_double), ("yc", C.c_double), ("xp", C.c_double), ("yp", C.c_double),
        ("mesh_max_scale", C.c_double),
    ]


# every entry point declared in include/lbm_b200.h: name -> (restype, argtypes)
_P = C.c_void_p
_D = C.POINTER(C.c_double)
ABI = {
    "lbm_default_params": (C.c_int, [C.POINTER(LbmParams)]),
    "lbm_create": (C.c_int, [C.POINTER(LbmParams), C.POINTER(_P)]),
    "lbm_destroy": (C.c_int, [_P]),
    "lbm_set_boundary": (C.c_int, [_P, C.c_int, _D, _D, C.c_int]),
    "lbm_read_boundary": (C.c_int, [_P, C.c_char_p]),
    "lbm_set_motion_table": (C.c_int, [_P, _D, C.c_int, C.c_int]),
    "lbm_load_motion_table": (C.c_int, [_P, C.c_char_p]),
    "lbm_parse_boundary_file": (C.c_int, [C.c_char_p, C.c_int, _D, _D]),
    "lbm_parse_motion_file": (C.c_int, [C.c_char_p, C.c_int, _D, C.c_int, C.POINTER(C.c_int)]),
    "lbm_init": (C.c_int, [_P, _D, _D]),
    "lbm_step": (C.c_int, [_P, _D]),
    "lbm_run": (C.c_int, [_P, C.c_int, _D, C.POINTER(C.c_int)]),
    "lbm_force_row_length": (C.c_int, [_P]),
    "lbm_get_fields": (C.c_int, [_P, _D, _D, _D]),
    "lbm_get_populations": (C.c_int, [_P, _D]),
    "lbm_set_populations": (C.c_int, [_P, _D]),
    "lbm_residual": (C.c_int, [_P, _D]),
    "lbm_mass": (C.c_int, [_P, _D]),
    "lbm_get_markers": (C.c_int, [_P, _D, _D, _D, C.POINTER(C.c_int)]),
    "lbm_set_timing": (C.c_int, [_P, C.c_int]),
    "lbm_get_timing": (C.c_int, [_P, _D, _D, _D, C.POINTER(C.c_int)]),
    "lbm_residual_device": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_int, C.c_int, _P, _D]),
    "lbm_get_launch_count": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    "lbm_step_index": (C.c_int, [_P]),
    "lbm_device_bytes": (C.c_int, [_P, C.POINTER(C.c_longlong)]),
    "lbm_last_error": (C.c_char_p, [_P]),
    "lbm_describe_status": (C.c_int, [C.c_uint, C.c_char_p, C.c_int]),
    "lbm_device_check": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "lbm_write_tecplot": (C.c_int, [_P, C.c_char_p, C.c_int, C.c_int, C.c_int]),
    "lbm_write_gforce": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, _D,
                                   _D]),
    "lbm_write_tecplot_fields": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_int, C.c_int, _D, _D, _D, C.c_int, C.c_int,
                                           _D, _D]),
    "lbm_save_checkpoint": (C.c_int, [_P, C.c_char_p]),
    "lbm_load_checkpoint": (C.c_int, [_P, C.c_char_p]),
    "lbm_save_flow_field": (C.c_int, [_P, C.c_char_p, _D, C.c_int]),
    "lbm_read_flow_field": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_int), _D, C.POINTER(C.c_int)]),
    "lbm_write_flow_field_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, _D, C.c_int, _D, _D,
                                            _D, _D]),
    "lbm_read_flow_field_file": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), _D,
                                           C.POINTER(C.c_int), _D, _D, _D, _D]),
    "lbm_batch_create": (C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P)]),
    "lbm_batch_destroy": (C.c_int, [_P]),
    "lbm_batch_add": (C.c_int, [_P, _P]),
    "lbm_batch_remove": (C.c_int, [_P, _P]),
    "lbm_batch_count": (C.c_int, [_P]),
    "lbm_batch_case_status": (C.c_int, [_P, C.c_int]),
    "lbm_batch_set_rows": (C.c_int, [_P, C.c_int]),
    "lbm_batch_set_occupancy": (C.c_int, [_P, C.c_int]),
    "lbm_batch_set_graphs": (C.c_int, [_P, C.c_int]),
    "lbm_batch_graph_stats": (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                        C.POINTER(C.c_longlong)]),
    "lbm_batch_get_timing": (C.c_int, [_P, _D, C.POINTER(C.c_int)]),
    "lbm_batch_run": (C.c_int, [_P, C.c_int, C.POINTER(_D), C.POINTER(C.c_int)]),
    "lbm_batch_last_error": (C.c_char_p, [_P]),
}


def header_declarations(header_path=None):
    """Names of the functions include/lbm_b200.h declares (parsed from the text)."""
    import re
    if header_path is None:
        header_path = os.path.join(os.path.dirname(HERE), "include", "lbm_b200.h")
    txt = open(header_path).read()
    return sorted(set(re.findall(r"LBM_API\s+(?:const\s+char\s*\*|int)\s*(lbm_\w+)\s*\(", txt)))


_lib = None


def load_library(path=None):
    """Loads liblbmb200.so (built in-tree) and binds the ABI. Raises if absent:
    there is no fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"CUDA library {p} is missing; build it with "
                           "python -m fortran_loadfile_mitiwing_b200.build")
    lib = C.CDLL(p)
    for name, (res, args) in ABI.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def dptr(a):
    """double* of a contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_D)
