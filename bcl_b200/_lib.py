"""ctypes binding of the bclx C ABI (include/bclx.h).

The shared library is built in place by ``bcl_b200.build`` (nvcc, sm_100a).
There is no fallback: if the library cannot be loaded, every entry point
raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbclx.so")

# status codes (bclx_status_t)
(TUNE_LIGHT_UB, TUNE_LEARN_TARGET, TUNE_BTABLE_MAX_BYTES, TUNE_SPMM_ROWS, TUNE_SPMM_LONG_ROW,
 TUNE_SPMM_LONG_BLOCKS, TUNE_SPMM_SCHEDULE, TUNE_ITEM_OUTPUTS, TUNE_WIDE_LIGHT, TUNE_SPMM_PANEL_MAJOR) = range(10)
OK, ERR_INVALID, ERR_DTYPE, ERR_CUDA, ERR_NO_MEMORY, ERR_INDEX_OVERFLOW, ERR_DEVICE_TIMEOUT, ERR_NO_DEVICE = range(8)
STATUS_NAMES = {
    OK: "BCLX_OK", ERR_INVALID: "BCLX_ERR_INVALID", ERR_DTYPE: "BCLX_ERR_DTYPE", ERR_CUDA: "BCLX_ERR_CUDA",
    ERR_NO_MEMORY: "BCLX_ERR_NO_MEMORY", ERR_INDEX_OVERFLOW: "BCLX_ERR_INDEX_OVERFLOW",
    ERR_DEVICE_TIMEOUT: "BCLX_ERR_DEVICE_TIMEOUT", ERR_NO_DEVICE: "BCLX_ERR_NO_DEVICE",
}

# value types (bclx_dtype_t)
F32, I32, BF16 = 0, 1, 2

i64, i32, vp = ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p


class CSRDesc(ctypes.Structure):
    """bclx_csr_t"""
    _fields_ = [("m", i64), ("n", i64), ("nnz", i64), ("row_ptr", vp), ("col_ind", vp), ("vals", vp),
                ("dtype", i32), ("pad_", i32)]


class SpGrid(ctypes.Structure):
    """bclx_spgrid_t"""
    _fields_ = [("m", i64), ("n", i64), ("tile_m", i64), ("tile_n", i64), ("grid_m", i64), ("grid_n", i64),
                ("tiles", vp), ("dtype", i32), ("pad_", i32)]


class SpGridOut(ctypes.Structure):
    """bclx_spgrid_out_t"""
    _fields_ = [("m", i64), ("n", i64), ("tile_m", i64), ("tile_n", i64), ("grid_m", i64), ("grid_n", i64),
                ("tile_row_ptr", vp), ("tile_offset", vp), ("col_ind", vp), ("vals", vp), ("dtype", i32),
                ("pad_", i32)]


class DGrid(ctypes.Structure):
    """bclx_dgrid_t"""
    _fields_ = [("m", i64), ("n", i64), ("tile_m", i64), ("tile_n", i64), ("grid_m", i64), ("grid_n", i64),
                ("tiles", vp), ("dtype", i32), ("pad_", i32)]


assert ctypes.sizeof(CSRDesc) == 56

# name -> (argtypes); every function returns int (status) unless listed in _RESTYPES
SIGNATURES = {
    "bclx_context_create": [ctypes.c_int, ctypes.POINTER(vp)],
    "bclx_context_destroy": [vp],
    "bclx_context_set_stream": [vp, vp],
    "bclx_context_synchronize": [vp],
    "bclx_context_release_cached": [vp],
    "bclx_context_set_tuning": [vp, i32, i64],
    "bclx_context_get_tuning": [vp, i32, ctypes.POINTER(i64)],
    "bclx_last_error": [],
    "bclx_version": [],
    "bclx_launch_count": [],
    "bclx_spgemm_symbolic": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut),
                             ctypes.POINTER(vp), ctypes.POINTER(i64)],
    "bclx_spgemm_numeric": [vp, vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut),
                            i32, i32],
    "bclx_spgemm_plan_destroy": [vp],
    "bclx_spgemm_symbolic_sub": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut),
                                 vp, vp, ctypes.POINTER(vp), ctypes.POINTER(i64)],
    "bclx_spgemm_numeric_staged": [vp, vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut),
                                   i32],
    "bclx_spgemm_plan_tune": [vp, i32, i32, i32],
    "bclx_spgemm_plan_stats": [vp, ctypes.POINTER(i64)],
    "bclx_tile_accumulate_symbolic": [vp, vp, i32, i64, i64, i32, vp, ctypes.POINTER(vp), ctypes.POINTER(i64)],
    "bclx_tile_accumulate_numeric": [vp, vp, vp, i32, ctypes.POINTER(CSRDesc)],
    "bclx_spgemm_tile_noalloc": [ctypes.POINTER(CSRDesc), ctypes.POINTER(CSRDesc), vp, vp, vp, i64,
                                 ctypes.POINTER(i64), vp],
    "bclx_spgemm_learned_run": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut), vp,
                                ctypes.POINTER(vp), ctypes.POINTER(i64)],
    "bclx_spgemm_learned_finish": [vp, vp, ctypes.POINTER(SpGridOut)],
    "bclx_spgemm_learned_run_sub": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut), vp,
                                    vp, vp, ctypes.POINTER(vp), ctypes.POINTER(i64)],
    "bclx_spgemm_learned_stats": [vp, ctypes.POINTER(i64)],
    "bclx_spgemm_row_features": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(SpGrid), ctypes.POINTER(SpGridOut), vp,
                                 vp],
    "bclx_spgemm_plan_row_counts": [vp, vp],
    "bclx_mlp_num_params": [],
    "bclx_mlp_predict": [vp, vp, i64, vp, vp],
    "bclx_mlp_gradient": [vp, vp, vp, i64, vp, vp],
    "bclx_mlp_train": [vp, vp, vp, i64, vp, i32, ctypes.c_float, vp],
    "bclx_spmm_tile": [vp, i64, i64, i64, i64, vp, vp, vp, vp, vp, i64, i64, i32],
    "bclx_spmm_grid": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(DGrid), ctypes.POINTER(DGrid)],
    "bclx_spmm_grid_rowwise": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(DGrid), ctypes.POINTER(DGrid)],
    "bclx_spmm_grid_sub": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(DGrid), ctypes.POINTER(DGrid), vp, vp],
    "bclx_dmatrix_sum": [vp, ctypes.POINTER(DGrid), vp],
    "bclx_spmatrix_binary_op": [vp, ctypes.POINTER(SpGrid), ctypes.POINTER(DGrid), i32],
    "bclx_csr_to_tiles": [vp, ctypes.POINTER(CSRDesc), ctypes.POINTER(SpGridOut)],
    "bclx_tiles_to_csr": [vp, ctypes.POINTER(SpGrid), vp, vp, vp],
}
_RESTYPES = {"bclx_last_error": ctypes.c_char_p, "bclx_launch_count": ctypes.c_longlong}


class BclxError(RuntimeError):
    def __init__(self, fn: str, status: int, detail: str):
        super().__init__(f"{fn} failed: {STATUS_NAMES.get(status, status)}" + (f" ({detail})" if detail else ""))
        self.status = status


_lib = None


def load(build_if_missing: bool = True):
    """Load libbclx.so (building it with nvcc first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        from . import build as _build
        _build.build()
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"bclx CUDA library not found at {LIB_PATH}; run `python -m bcl_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    """Call an entry point and raise BclxError on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != OK:
        detail = lib.bclx_last_error()
        raise BclxError(name, rc, detail.decode() if detail else "")


def exported_symbols():
    return list(SIGNATURES)
