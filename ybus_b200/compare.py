"""For comparison only: ybus_cuda's own route to the solve (cuSPARSE SpSM on the two triangles of
a Cholesky factor, blocks of `width` right-hand sides; ybus_cuda/src/sparse.rs:371-420), from
libybcompare.so, which no solve of libybgpu.so loads. The bench times it beside the library's
solves on the same device arrays."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import HERE, ptr

_lib = None


def _open() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "libybcompare.so"
        if not path.exists():
            raise RuntimeError(f"{path} is not built")
        _lib = C.CDLL(str(path), mode=os.RTLD_LOCAL)
        _lib.ybc_spsm_solve.restype = C.c_int32
        _lib.ybc_spsm_solve.argtypes = [C.c_int64] + [C.c_void_p] * 8 + [C.c_int64, C.c_void_p, C.c_int64, C.c_int64,
                                                                        C.c_int64, C.c_void_p, C.c_char_p, C.c_size_t]
    return _lib


def spsm_solve(chol, d_rhs: int, d_out: int, count: int, width: int) -> float:
    """Solves `count` right-hand sides (device pointers, column-major n x count) with `chol` (a
    host.HostCholesky) by cuSPARSE SpSM in blocks of `width`; returns the solves' milliseconds."""
    arrs = [np.ascontiguousarray(a, t) for a, t in ((chol.l.ptr, np.int64), (chol.l.idx, np.int64),
                                                     (chol.l.val, np.float64), (chol.lt.ptr, np.int64),
                                                     (chol.lt.idx, np.int64), (chol.lt.val, np.float64),
                                                     (chol.perm, np.int64))]
    ms = C.c_double()
    msg = C.create_string_buffer(512)
    n = chol.n
    rc = _open().ybc_spsm_solve(n, *[ptr(a) for a in arrs], d_rhs, n, d_out, n, count, width, C.byref(ms), msg,
                                len(msg))
    if rc != 0:
        raise RuntimeError(f"cuSPARSE comparison failed: {msg.value.decode(errors='replace')}")
    return ms.value
