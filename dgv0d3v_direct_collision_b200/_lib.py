"""ctypes binding of libdgv_b200.so (the C-ABI declared in include/dgv_b200.h).

The shared library is the product: there is no Python or CPU fallback.  If the
library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdgv_b200.so")

DGV_OK, DGV_EINVAL, DGV_ERANGE, DGV_ECUDA, DGV_ETIMEOUT, DGV_ENOMEM, DGV_ESTATE, DGV_EUNSUP = range(8)
DGV_PREC_F64, DGV_PREC_F32C, DGV_PREC_TC = 0, 1, 2
DGV_OPT_PROJECT, DGV_OPT_NCHUNKS, DGV_OPT_KTIMING, DGV_OPT_TCFORM, DGV_OPT_TCTILES, DGV_OPT_TCSETMB = 1, 2, 3, 4, 5, 6
DGV_OPT_WAIT_LIMIT_US, DGV_OPT_TEST_WITHHOLD, DGV_OPT_TCAUTOTUNE, DGV_OPT_FGLOBAL, DGV_OPT_TCPERSIST = 7, 8, 9, 10, 11
DGV_LAYOUT_F32, DGV_LAYOUT_TC_CHUNK, DGV_LAYOUT_TC_BLOCK, DGV_LAYOUT_TC_ADJ = 1, 2, 4, 8

STATUS_NAMES = {0: "DGV_OK", 1: "DGV_EINVAL", 2: "DGV_ERANGE", 3: "DGV_ECUDA", 4: "DGV_ETIMEOUT",
                5: "DGV_ENOMEM", 6: "DGV_ESTATE", 7: "DGV_EUNSUP"}

# every entry point include/dgv_b200.h declares
EXPORTS = [
    "dgv_ctx_create", "dgv_ctx_destroy", "dgv_last_error", "dgv_set_stream", "dgv_set_async",
    "dgv_set_option", "dgv_get_option", "dgv_release_layouts", "dgv_kernel_stats", "dgv_grid_info", "dgv_nodes", "dgv_load_A", "dgv_generate_A_synthetic",
    "dgv_A_info", "dgv_export_A", "dgv_collide", "dgv_collide_batched", "dgv_collide_cells", "dgv_spatial_oper", "dgv_set_regime",
    "dgv_regime_info",
    "dgv_step_rk", "dgv_step_rk_batched", "dgv_prepare_ab", "dgv_step_ab", "dgv_moments", "dgv_maxwellian", "dgv_project",
    "dgv_jvp", "dgv_vjp", "dgv_vjp_batched", "dgv_prepare_linear", "dgv_apply_linear", "dgv_collide_f64_noalloc",
    "dgv_compute_A", "dgv_read_A_files", "dgv_write_A_file", "dgv_read_A_arrays", "dgv_write_A_arrays", "dgv_file_error",
    "dgv_write_solution", "dgv_read_solution", "dgv_write_solution_arrays", "dgv_read_solution_arrays",
    "dgv_collide_group", "dgv_tc_plan",
]


class GridDesc(C.Structure):
    _fields_ = [("su", C.c_int32), ("sv", C.c_int32), ("sw", C.c_int32),
                ("Mu", C.c_int32), ("Mv", C.c_int32), ("Mw", C.c_int32),
                ("u_L", C.c_double), ("u_R", C.c_double), ("v_L", C.c_double),
                ("v_R", C.c_double), ("w_L", C.c_double), ("w_R", C.c_double),
                ("kappa", C.c_double)]


class DGVError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def load() -> C.CDLL:
    """Load the library and declare its signatures (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m dgv0d3v_direct_collision_b200.build` "
            "(nvcc, sm_100a). There is no fallback implementation.")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    sig = {
        "dgv_ctx_create": [C.POINTER(GridDesc), C.c_int, C.POINTER(vp)],
        "dgv_ctx_destroy": [vp],
        "dgv_set_stream": [vp, vp],
        "dgv_set_async": [vp, C.c_int],
        "dgv_set_option": [vp, C.c_int, i64],
        "dgv_kernel_stats": [vp, C.POINTER(dbl), C.POINTER(i64), C.POINTER(i64), C.c_int],
        "dgv_grid_info": [vp, C.POINTER(i64), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)],
        "dgv_nodes": [vp, vp, vp, vp, vp],
        "dgv_load_A": [vp, i64, vp, vp, vp, vp, C.c_int],
        "dgv_generate_A_synthetic": [vp, C.c_uint64, dbl, C.c_int],
        "dgv_A_info": [vp, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(dbl)],
        "dgv_export_A": [vp, C.POINTER(i64), vp, vp, vp, vp],
        "dgv_collide": [vp, vp, vp, i64, C.c_int],
        "dgv_collide_batched": [vp, i32, vp, vp, C.c_int],
        "dgv_collide_cells": [vp, i32, vp, vp, i32, i32, C.c_int],
        "dgv_collide_group": [i32, C.POINTER(vp), vp, vp, vp, C.c_int, vp],
        "dgv_tc_plan": [vp, i32, C.POINTER(i64), C.POINTER(i64), C.POINTER(dbl)],
        "dgv_compute_A": [vp, dbl, dbl, dbl, dbl, C.c_int],
        "dgv_read_A_files": [vp, C.POINTER(C.c_char_p), i32],
        "dgv_write_A_file": [vp, C.c_char_p, i64],
        "dgv_read_A_arrays": [C.POINTER(C.c_char_p), i32, i32, C.POINTER(i64), vp, vp, vp, vp],
        "dgv_write_A_arrays": [C.c_char_p, i32, i64, vp, vp, vp, vp, i64],
        "dgv_set_regime": [vp, dbl, dbl],
        "dgv_regime_info": [vp, C.POINTER(i32), C.POINTER(dbl)],
        "dgv_spatial_oper": [vp, vp, vp, dbl, C.c_int],
        "dgv_step_rk": [vp, vp, vp, dbl, C.c_int, C.c_int],
        "dgv_step_rk_batched": [vp, i32, vp, vp, dbl, C.c_int, C.c_int],
        "dgv_prepare_ab": [vp, vp, dbl, C.c_int, C.c_int],
        "dgv_step_ab": [vp, vp, dbl, C.c_int],
        "dgv_write_solution": [vp, C.c_char_p, vp, dbl, dbl],
        "dgv_read_solution": [vp, C.c_char_p, vp, C.POINTER(dbl), C.POINTER(dbl)],
        "dgv_write_solution_arrays": [C.c_char_p, i32, i32, dbl, dbl, vp],
        "dgv_read_solution_arrays": [C.c_char_p, C.POINTER(i32), C.POINTER(i32), C.POINTER(dbl), C.POINTER(dbl), vp],
        "dgv_moments": [vp, vp, vp],
        "dgv_maxwellian": [vp, dbl, dbl, dbl, dbl, dbl, vp],
        "dgv_project": [vp, vp, i32],
        "dgv_jvp": [vp, vp, vp, vp, C.c_int],
        "dgv_vjp": [vp, vp, vp, vp, C.c_int],
        "dgv_vjp_batched": [vp, i32, vp, vp, vp, C.c_int],
        "dgv_get_option": [vp, C.c_int, C.POINTER(C.c_int64)],
        "dgv_release_layouts": [vp, C.c_int, C.POINTER(C.c_int64)],
        "dgv_prepare_linear": [vp, vp],
        "dgv_apply_linear": [vp, vp, vp, C.c_int],
        "dgv_collide_f64_noalloc": [vp, vp, vp, i32, vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.dgv_last_error.argtypes = [vp]
    L.dgv_last_error.restype = C.c_char_p
    L.dgv_file_error.argtypes = []
    L.dgv_file_error.restype = C.c_char_p
    _lib = L
    return L
