"""The C ABI library loads and exports every entry point include/ybgpu.h declares, and its
host-side checks reject bad input with status codes (CPU only: no compute on a GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from ybus_b200 import _lib, host

HEADER = Path(__file__).resolve().parent.parent / "include" / "ybgpu.h"


def declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yb_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) > 20
    lib = _lib.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_every_declared_symbol_has_a_python_signature():
    assert set(declared()) <= set(_lib.SIGNATURES), sorted(set(declared()) - set(_lib.SIGNATURES))


def test_error_codes_and_messages():
    lib = _lib.lib()
    out = C.c_void_p()
    r = np.array([0, 5], np.int64)
    c = np.array([0, 0], np.int64)
    v = np.array([1.0, 2.0])
    status = lib.yb_matrix_from_triplets(2, 2, 2, r.ctypes.data, c.ctypes.data, v.ctypes.data, 1, 0, C.byref(out))
    assert status == _lib.YB_ERROR_INVALID_ARGUMENT
    assert "outside" in _lib.last_error()


def test_not_positive_definite_and_not_symmetric():
    m = host.Matrix.from_triplets(2, 2, [0, 1, 0, 1], [0, 1, 1, 0], [1.0, 1.0, 2.0, 2.0])
    with pytest.raises(_lib.YbError) as e:
        host.cholesky(m)
    assert e.value.status == _lib.YB_ERROR_NOT_POSITIVE_DEFINITE
    m = host.Matrix.from_triplets(2, 2, [0, 1, 0], [0, 1, 1], [2.0, 2.0, 1.0])
    with pytest.raises(_lib.YbError) as e:
        host.cholesky(m)
    assert e.value.status == _lib.YB_ERROR_NOT_SYMMETRIC


def test_singular_lu_is_reported():
    m = host.Matrix.from_triplets(2, 2, [0, 0], [0, 1], [1.0, 1.0], by_rows=False)
    with pytest.raises(_lib.YbError) as e:
        host.lu(m)
    assert e.value.status == _lib.YB_ERROR_SINGULAR


def test_gpu_new_without_a_device_is_none_not_an_error():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from ybus_b200 import Gpu
    assert Gpu.new() is None
