"""The device error path, made to run without a fault. A lane solve whose first warp of block 0
is denied the copy of one page (yb_factor_withhold_lane_page: the host sets it, the kernel just
does not issue that copy) waits for it for the kernel's bounded one second, gives up, waits
(bounded) for its copies in flight, takes its block's remaining barriers and returns. The library
then reports YB_ERROR_DEVICE_TIMEOUT: through yb_factor_check_error after a device-array solve, by
itself after a host-array solve. The context stays usable, and the next solve is correct and
reports nothing."""
import time

import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import worst_relative_difference
from ybus_b200 import FP64, CudaError, GpuFactor, _lib, grids, host

pytestmark = pytest.mark.gpu

LANE = 5


@pytest.fixture(scope="module")
def grid_factor():
    g = grids.make_grid(2000, 700, grids.SEED_BASE + 1)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, 2000)
    chol = host.cholesky(host.Matrix.from_triplets(2000, 2000, r, c, v).select(keep, keep))
    rhs = np.random.default_rng(21).standard_normal((96, chol.n))
    return chol, rhs, orc.solve_many(chol, rhs, threads=8)


# page 0 is among the copies issued before the stream starts, page 5 among those issued as pages end
@pytest.mark.parametrize("page", [0, 5])
def test_a_wait_that_runs_out_is_reported_and_the_gpu_stays_usable(gpu, grid_factor, page):
    import torch
    chol, rhs, cpu = grid_factor
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    assert _lib.lib().yb_factor_withhold_lane_page(factor._h, page) == _lib.YB_OK
    t0 = time.perf_counter()
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    waited = time.perf_counter() - t0
    with pytest.raises(CudaError) as err:
        factor.check_error()
    assert err.value.status == _lib.YB_ERROR_DEVICE_TIMEOUT
    assert 0.9 < waited < 30.0, waited  # the one-second limit, twice at most (the wait and the drain)
    factor.check_error()  # reported once, then cleared
    # the setting applied once: the next solve runs whole, is correct and reports nothing
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    factor.check_error()
    assert worst_relative_difference(x.cpu().numpy(), cpu) < 1e-12


def test_the_host_array_solve_reports_the_timeout_by_itself(gpu, grid_factor):
    chol, rhs, cpu = grid_factor
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    factor.set_block_width(rhs.shape[0])
    assert _lib.lib().yb_factor_withhold_lane_page(factor._h, 2) == _lib.YB_OK
    with pytest.raises(CudaError) as err:
        factor.solve_many(rhs)
    assert err.value.status == _lib.YB_ERROR_DEVICE_TIMEOUT
    assert worst_relative_difference(factor.solve_many(rhs), cpu) < 1e-12


def test_withholding_takes_a_page_index_or_nothing(gpu, grid_factor):
    chol, _, _ = grid_factor
    factor = GpuFactor.from_cholesky(gpu, chol)
    assert _lib.lib().yb_factor_withhold_lane_page(factor._h, -2) == _lib.YB_ERROR_INVALID_ARGUMENT
    assert _lib.lib().yb_factor_withhold_lane_page(factor._h, -1) == _lib.YB_OK
