"""The solve entry point that allocates nothing (yb_solve_many_device_noalloc), for callers that
cannot have a library allocate device memory during a solve: programs whose own pool allocator
holds the GPU's memory, and latency-bound loops that cannot take an allocation's synchronisation.
Its solutions must agree with the ordinary device entry point's (yb_solve_many_device) to the
solve tests' bar on two calls in a row, since the fixed scratch array it uses keeps the previous
call's contents. This file is collected last so a run that stops at its first failure has run
every other test first."""
import ctypes as C

import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import random_spd, right_hand_sides, worst_relative_difference
from ybus_b200 import FP32, FP64, GpuFactor, _lib, grids, host

pytestmark = pytest.mark.gpu

BAR = 1e-12


def _noalloc(factor, b, x, count, precision):
    return _lib.lib().yb_solve_many_device_noalloc(factor._h, b.data_ptr(), factor.dim(), x.data_ptr(), factor.dim(),
                                                   count, precision, None)


def _grid_factor():
    g = grids.make_grid(2000, 700, grids.SEED_BASE + 1)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, 2000)
    return host.cholesky(host.Matrix.from_triplets(2000, 2000, r, c, v).select(keep, keep))


@pytest.mark.parametrize("case", ["fixture", "grid"])
def test_noalloc_solve_matches_the_device_entry_point_twice(gpu, case):
    import torch
    chol = host.cholesky(random_spd(300, 3, 7)) if case == "fixture" else _grid_factor()
    rhs = right_hand_sides(chol.n, 45, 11) if case == "fixture" else \
        np.random.default_rng(4).standard_normal((300, chol.n))
    factor = GpuFactor.from_cholesky(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    ref = torch.empty_like(b)
    factor.solve_many_device(b.data_ptr(), ref.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    expected = ref.cpu().numpy()
    assert worst_relative_difference(expected, orc.solve_many(chol, rhs, threads=8)) < BAR
    xs = [torch.full_like(b, float("nan")) for _ in range(2)]
    torch.cuda.synchronize()
    free = []
    for call, x in enumerate(xs):
        free.append(torch.cuda.mem_get_info()[0])
        assert _noalloc(factor, b, x, rhs.shape[0], FP64) == _lib.YB_OK, _lib.last_error()
        gpu.synchronize()
        d = worst_relative_difference(x.cpu().numpy(), expected)
        assert d < BAR, f"call {call}: {d:e}"
    # the entry point's whole contract: the device's free memory is what it was before either call
    # (the fixed array and the kernels were placed when the GPU was opened)
    free.append(torch.cuda.mem_get_info()[0])
    assert free[0] == free[1] == free[2], free


def test_noalloc_solve_in_fp32_and_narrow_tiles(gpu):
    import torch
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 40, 11)
    factor = GpuFactor.from_cholesky(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    cpu = orc.solve_many(chol, rhs)
    for tile in (1, 4, 32):
        factor.set_tile(FP32, tile, 256, 2)
        for _ in range(2):
            x = torch.zeros_like(b)
            assert _noalloc(factor, b, x, 40, FP32) == _lib.YB_OK, _lib.last_error()
            gpu.synchronize()
            assert worst_relative_difference(x.cpu().numpy(), cpu) < 1e-4


def test_noalloc_solve_rejects_working_vectors_beyond_the_array(gpu):
    import torch
    # a path graph of 70,000 buses: one block's FP64 vectors at tile width 32 need 17.9 MB > 16 MiB
    n = 70_000
    i = np.arange(n)
    r = np.concatenate([i, i[:-1], i[1:]])
    c = np.concatenate([i, i[1:], i[:-1]])
    v = np.concatenate([np.full(n, 4.0), np.full(n - 1, -1.0), np.full(n - 1, -1.0)])
    chol = host.cholesky(host.Matrix.from_triplets(n, n, r, c, v))
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile(FP64, 32, 256, 1)
    b = torch.ones((1, n), dtype=torch.float64, device="cuda")
    x = torch.empty_like(b)
    assert _noalloc(factor, b, x, 1, FP64) == _lib.YB_ERROR_TOO_LARGE
    assert "16 MiB" in _lib.last_error()
    # a narrower tile fits, and solves
    factor.set_tile(FP64, 1, 256, 1)
    assert _noalloc(factor, b, x, 1, FP64) == _lib.YB_OK, _lib.last_error()
    gpu.synchronize()
    cpu = orc.solve_many(chol, np.ones((1, n)))
    assert worst_relative_difference(x.cpu().numpy(), cpu) < BAR
