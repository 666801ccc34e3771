"""ctypes bindings of libybhost.so (the host factor producer, include/ybhost.h) and libybgpu.so
(the GPU path, include/ybgpu.h).

Both are loaded from this package's directory; libybgpu.so is loaded only at the first call that
needs it, so host-only work never maps it. There is no fallback: if a library is missing or fails
to load, every call raises, so nothing silently runs on the CPU instead.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libybgpu.so"
HOST_LIB_PATH = HERE / "libybhost.so"

i32, i64, u64, dbl, vp = C.c_int32, C.c_int64, C.c_uint64, C.c_double, C.c_void_p
P_i64 = C.POINTER(C.c_int64)
P_i32 = C.POINTER(C.c_int32)
P_dbl = C.POINTER(C.c_double)

YB_OK = 0
YB_ERROR_INVALID_ARGUMENT = 1
YB_ERROR_SHAPE_MISMATCH = 2
YB_ERROR_TOO_LARGE = 3
YB_ERROR_NOT_POSITIVE_DEFINITE = 4
YB_ERROR_SINGULAR = 5
YB_NO_DEVICE = 6
YB_ERROR_CUDA = 7
YB_ERROR_NOT_SYMMETRIC = 8
YB_ERROR_DEVICE_TIMEOUT = 9
YB_ERROR_INTERNAL = 10
YB_CHOLESKY = 1
YB_LU = 2
YB_ORDER_NATURAL = 0
YB_ORDER_AMD = 1
YB_ORDER_COLAMD = 3
YB_FP64 = 0
YB_FP32 = 1

# name -> (restype, argtypes), libybhost.so
HOST_SIGNATURES: dict[str, tuple] = {
    "yb_last_error_message": (i32, [C.c_char_p, C.c_size_t]),
    "yb_matrix_from_triplets": (i32, [i64, i64, i64, vp, vp, vp, i32, i32, C.POINTER(vp)]),
    "yb_matrix_select": (i32, [vp, i64, vp, i64, vp, C.POINTER(vp)]),
    "yb_matrix_reorient": (i32, [vp, C.POINTER(vp)]),
    "yb_matrix_info": (i32, [vp, P_i64, P_i64, P_i64, P_i32, P_i32]),
    "yb_matrix_export": (i32, [vp, vp, vp, vp]),
    "yb_matrix_free": (None, [vp]),
    "yb_ordering": (i32, [vp, i32, vp]),
    "yb_host_cholesky": (i32, [vp, i32, C.POINTER(vp)]),
    "yb_host_lu": (i32, [vp, i32, dbl, C.POINTER(vp)]),
    "yb_host_factor_info": (i32, [vp, P_i32, P_i32, P_i64, P_i64, P_i64]),
    "yb_host_factor_export": (i32, [vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    "yb_host_etree": (i32, [vp, vp]),
    "yb_host_factor_free": (None, [vp]),
}

# name -> (restype, argtypes), libybgpu.so
SIGNATURES: dict[str, tuple] = {
    "yb_gpu_new": (i32, [i32, C.POINTER(vp)]),
    "yb_gpu_free": (None, [vp]),
    "yb_gpu_name": (i32, [vp, C.c_char_p, C.c_size_t]),
    "yb_gpu_memory": (i32, [vp, C.POINTER(u64), C.POINTER(u64)]),
    "yb_gpu_properties": (i32, [vp, P_i32, P_i32, P_i32, P_i64]),
    "yb_gpu_stream": (vp, [vp]),
    "yb_gpu_synchronize": (i32, [vp, vp]),
    "yb_factor_from_cholesky": (i32, [vp, i64, vp, vp, vp, vp, C.POINTER(vp)]),
    "yb_factor_from_lu": (i32, [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(vp)]),
    "yb_factor_from_lu_transposed": (i32, [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(vp)]),
    "yb_factor_free": (None, [vp]),
    "yb_factor_dim": (i64, [vp]),
    "yb_factor_block_width": (i64, [vp]),
    "yb_factor_set_block_width": (i32, [vp, i64]),
    "yb_factor_timings": (i32, [vp, P_dbl, P_dbl, P_dbl, P_i64]),
    "yb_factor_reset_timings": (i32, [vp]),
    "yb_factor_plan_info": (i32, [vp, P_i32, P_i32, P_i64, P_i64, P_i32, P_i32]),
    "yb_factor_set_tile": (i32, [vp, i32, i32, i32, i32]),
    "yb_factor_get_tile": (i32, [vp, i32, P_i32, P_i32, P_i32]),
    "yb_factor_set_tile_kind": (i32, [vp, i32, i32]),
    "yb_factor_set_stream": (i32, [vp, i32, i32, i32, i32, i32]),
    "yb_factor_stream_info": (i32, [vp, i32, P_i32, P_i32, P_i64, P_i64, P_i32, P_i32, P_i32]),
    "yb_factor_withhold_lane_page": (i32, [vp, i32]),
    "yb_factor_check_error": (i32, [vp]),
    "yb_factor_set_phase_clock": (i32, [vp, vp]),
    "yb_factor_set_tail_level": (i32, [vp, i32, i32]),
    "yb_factor_set_domain": (i32, [vp, i32, i32, i32, i32, i32]),
    "yb_factor_autotune": (i32, [vp, i32, i64, vp, P_dbl]),
    "yb_factor_lane_info": (i32, [vp, i32, vp]),
    "yb_factor_set_lane_rhs_per_lane": (i32, [vp, i32, i32]),
    "yb_factor_set_lane_min_count": (i32, [vp, i32, i64]),
    "yb_factor_set_refine_lane_min_count": (i32, [vp, i64]),
    "yb_factor_lane_min_counts": (i32, [vp, i32, P_i64, P_i64]),
    "yb_factor_time_lane": (i32, [vp, i32]),
    "yb_factor_lane_times": (i32, [vp, P_dbl, P_dbl, P_dbl, P_i64]),
    "yb_factor_set_lane": (i32, [vp, i32, i32, i32]),
    "yb_factor_domain_info": (i32, [vp, i32, P_i32, P_i32, P_i32, P_i64, P_i64, P_i64, P_dbl]),
    "yb_domain_layout_cholesky": (i32, [i64, vp, vp, vp, vp, i32, i32, i32, i32, vp, vp, vp, vp, vp]),
    "yb_lane_layout_cholesky": (i32, [i64, vp, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp]),
    "yb_lane_layout_lu": (i32, [i64, vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, i32, i32, i32, vp, vp, vp, vp, vp]),
    "yb_solve_many": (i32, [vp, vp, i64, vp]),
    "yb_solve_many_transpose": (i32, [vp, vp, i64, vp]),
    "yb_solve_many_mixed": (i32, [vp, vp, i64, vp, i32, dbl, vp, vp]),
    "yb_solve_many_device": (i32, [vp, vp, i64, vp, i64, i64, i32, vp]),
    "yb_solve_many_device_noalloc": (i32, [vp, vp, i64, vp, i64, i64, i32, vp]),
    "yb_factor_attach_matrix": (i32, [vp, vp, vp, vp]),
    "yb_factor_from_lu_complex": (i32, [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(vp)]),
    "yb_factor_attach_matrix_complex": (i32, [vp, vp, vp, vp]),
    "yb_solve_batch_complex": (i32, [i64, vp, vp, vp, vp, i32, i32, dbl, vp, vp, vp]),
    "yb_pair_solves": (i32, [vp, i64, vp, vp, C.POINTER(vp)]),
    "yb_pair_updates": (i32, [vp, vp, i64, vp, vp, vp, vp, C.POINTER(vp)]),
    "yb_block_columns": (i64, [vp]),
    "yb_block_singular": (i32, [vp, vp]),
    "yb_block_solutions": (i32, [vp, vp]),
    "yb_block_maxima": (i32, [vp, vp, vp, vp]),
    "yb_block_product": (i32, [vp, vp, vp, vp]),
    "yb_block_product_maxima": (i32, [vp, vp, vp, vp, vp, vp]),
    "yb_block_free": (None, [vp]),
    "yb_operator_new": (i32, [vp, i64, vp, vp, vp, C.POINTER(vp)]),
    "yb_operator_rows": (i64, [vp]),
    "yb_operator_set_offset": (i32, [vp, vp]),
    "yb_operator_set_weights": (i32, [vp, vp]),
    "yb_operator_free": (None, [vp]),
    "yb_dc_network_new": (i32, [vp, i64, i64, vp, vp, vp, i64, C.POINTER(vp)]),
    "yb_dc_network_free": (None, [vp]),
    "yb_dc_network_factor": (vp, [vp]),
    "yb_dc_bridges": (i32, [vp, vp]),
    "yb_dc_ptdf_columns": (i32, [vp, i64, vp, vp]),
    "yb_dc_ptdf_transfers": (i32, [vp, i64, vp, vp, vp]),
    "yb_dc_lodf_columns": (i32, [vp, i64, vp, vp]),
    "yb_dc_outage_loadings_batch": (i32, [vp, i64, vp, vp, vp, vp, i32, vp, vp, vp, vp]),
    "yb_dc_set_slack_weights": (i32, [vp, vp]),
    "yb_dc_solve_many": (i32, [vp, i64, vp, vp, vp, vp]),
    "yb_dc_outage_solutions": (i32, [vp, i64, vp, vp, vp, vp, vp, vp, vp, vp]),
    "yb_dc_adjoint_new": (i32, [vp, i64, C.POINTER(vp)]),
    "yb_dc_adjoint_forward": (i32, [vp, vp, vp, dbl, vp, vp]),
    "yb_dc_adjoint_backward": (i32, [vp, vp, vp]),
    "yb_dc_adjoint_free": (None, [vp]),
    "yb_solve_many_refined_device": (i32, [vp, vp, i64, vp, i64, i64, i32, dbl, vp, vp, vp]),
}

_lib: C.CDLL | None = None
_host_lib: C.CDLL | None = None


class YbError(RuntimeError):
    """A failed libybgpu call: `status` is the YB_* code, the message the library's."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


def _open(path: Path, signatures: dict) -> C.CDLL:
    if not path.exists():
        raise RuntimeError(f"{path} is not built: run `python -c 'import __graft_entry__ as g; g.build()'`")
    handle = C.CDLL(str(path), mode=os.RTLD_LOCAL)
    for name, (res, args) in signatures.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    return handle


def host_lib() -> C.CDLL:
    """libybhost.so: the host factor producer and the last-error store."""
    global _host_lib
    if _host_lib is None:
        _host_lib = _open(HOST_LIB_PATH, HOST_SIGNATURES)
    return _host_lib


def lib() -> C.CDLL:
    """libybgpu.so: the GPU path (it loads libybhost.so beside it)."""
    global _lib
    if _lib is None:
        host_lib()
        _lib = _open(LIB_PATH, SIGNATURES)
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    host_lib().yb_last_error_message(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> int:
    if status != YB_OK:
        raise YbError(status, last_error())
    return status


def ptr(array) -> int | None:
    """The data pointer of a numpy array (or None for None)."""
    if array is None:
        return None
    return array.ctypes.data
