"""The C ABI libraries load and export every entry point include/ybhost.h and include/ybgpu.h
declare (libybhost.so and libybgpu.so), and their host-side checks reject bad input with status
codes (CPU only: no compute on a GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from ybus_b200 import _lib, host

INCLUDE = Path(__file__).resolve().parent.parent / "include"


def declared(header):
    text = (INCLUDE / header).read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yb_\w+)\s*\(", text)))


@pytest.mark.parametrize("header,which", [("ybhost.h", "host"), ("ybgpu.h", "gpu")])
def test_every_declared_symbol_is_exported(header, which):
    names = declared(header)
    assert len(names) > 10
    lib = _lib.host_lib() if which == "host" else _lib.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("header,which", [("ybhost.h", "host"), ("ybgpu.h", "gpu")])
def test_every_declared_symbol_has_a_python_signature(header, which):
    sigs = _lib.HOST_SIGNATURES if which == "host" else _lib.SIGNATURES
    assert set(declared(header)) <= set(sigs), sorted(set(declared(header)) - set(sigs))


def test_the_host_library_stands_alone():
    # the host producer needs no GPU library: a fresh interpreter that factors a matrix maps
    # libybhost.so and not libybgpu.so
    import subprocess
    import sys
    code = ("import numpy as np; from ybus_b200 import host; "
            "m = host.Matrix.from_triplets(2, 2, [0, 1], [0, 1], [4.0, 9.0]); host.cholesky(m); "
            "maps = open('/proc/self/maps').read(); print('libybhost.so' in maps, 'libybgpu.so' in maps)")
    root = Path(__file__).resolve().parent.parent
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, check=True)
    assert out.stdout.split() == ["True", "False"], out.stdout + out.stderr


def test_error_codes_and_messages():
    lib = _lib.host_lib()
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
