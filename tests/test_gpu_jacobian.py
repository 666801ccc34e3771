"""The Newton-Raphson Jacobian's LU solve on the GPU (the reference's second matrix for its GPU
survey, ybus_powerflow/examples/cuda_survey.rs:213-235, through `GpuFactor::from_lu`): the 10,000-
bus network's Jacobian (order 17,998) factored by AMD LU on the host, 4,096 right-hand sides
solved and transposed-solved through the C ABI, against the oracle's LU solves (lu.rs:640-649,
770-785, 506-533) at the reference's bar."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import worst_relative_difference
from ybus_b200 import FP64, GpuFactor, configs

pytestmark = pytest.mark.gpu

BAR = 1e-12
AUTO, GLOBAL, LANE = 0, 2, 5  # yb_factor_set_tile_kind's kinds


@pytest.fixture(scope="module")
def system():
    return configs.jacobian_system()


@pytest.mark.parametrize("kind", [AUTO, LANE, GLOBAL])
def test_jacobian_solves_match_the_oracle(gpu, system, kind):
    import torch
    factor = GpuFactor.from_lu(gpu, system.lu)
    factor.set_tile_kind(FP64, kind)
    rhs = system.rhs
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    factor.time_lane(True)
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    factor.check_error()
    # at 4,096 right-hand sides the automatic choice takes the lane solve: the forest of L's and
    # U's joint pattern orders both sweeps of the pivoted LU
    assert (factor.lane_times()["launches"] > 0) == (kind != GLOBAL)
    factor.time_lane(False)
    xs = x.cpu().numpy()
    sample = np.arange(0, rhs.shape[0], 97)
    assert worst_relative_difference(xs[sample], orc.solve_many_lu(system.lu, rhs[sample], threads=8)) < BAR
    # every 17th solution's relative residual against the matrix itself, against the oracle's own
    # solution's: the LU factor's threshold pivoting sets both (up to 2.3e-10 here), and solutions
    # that differ by rounding move it by a small factor (1.6 at most measured)
    p, i, v = system.jacobian.to_csr().arrays()
    cols = np.arange(0, rhs.shape[0], 17)
    cpu = orc.solve_many_lu(system.lu, rhs[cols], threads=8)
    for k, c in zip(cols, cpu):
        mine, theirs = orc.relative_residual(p, i, v, xs[k], rhs[k]), orc.relative_residual(p, i, v, c, rhs[k])
        assert mine <= 4.0 * theirs + 1e-13, (k, mine, theirs)


def test_the_automatic_threshold_takes_the_lane_solve_from_two_groups(gpu, system):
    # the Jacobian's domain tiles hold one column: the lane solve is the faster from 64 right-hand
    # sides on, and the automatic choice takes it there
    factor = GpuFactor.from_lu(gpu, system.lu)
    assert factor.domain_info(FP64)["tile"] == 1
    assert factor.lane_min_count(FP64) == 64
    rhs = system.rhs[:256]
    factor.time_lane(True)
    x = factor.solve_many(rhs)
    assert factor.lane_times()["launches"] > 0
    factor.time_lane(False)
    assert worst_relative_difference(x, orc.solve_many_lu(system.lu, rhs, threads=8)) < BAR


def test_jacobian_solves_in_blocks_of_sixteen_warps(gpu, system):
    # 128 groups of 32 on 148 SMs: blocks of 16 warps, one an SM, halve each warp's chain of rows
    import torch
    factor = GpuFactor.from_lu(gpu, system.lu)
    factor.set_tile_kind(FP64, LANE)
    factor.set_lane(FP64, 16)
    assert factor.lane_info(FP64)["warps"] == 16
    rhs = system.rhs
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    factor.check_error()
    sample = np.arange(0, rhs.shape[0], 89)
    assert worst_relative_difference(x.cpu().numpy()[sample], orc.solve_many_lu(system.lu, rhs[sample], threads=8)) < BAR


def test_jacobian_transposed_solves_match_the_oracle(gpu, system):
    factor = GpuFactor.from_lu(gpu, system.lu)
    rhs = system.rhs[:256]
    cpu = orc.solve_many_lu(system.lu, rhs, threads=8, transpose=True)
    assert worst_relative_difference(factor.solve_many_transpose(rhs), cpu) < BAR


def test_the_transposed_factor_takes_the_lane_solve(gpu, system):
    # A' = Q U' L' P: U' (not unit) forward, L' backward; the joint pattern's forest orders both
    factor = GpuFactor.from_lu_transposed(gpu, system.lu)
    factor.set_tile_kind(FP64, LANE)
    assert factor.lane_info(FP64)["slots"] <= 64
    rhs = system.rhs[:512]
    factor.time_lane(True)
    x = factor.solve_many(rhs)
    assert factor.lane_times()["launches"] > 0
    factor.time_lane(False)
    factor.check_error()
    assert worst_relative_difference(x, orc.solve_many_lu(system.lu, rhs, threads=8, transpose=True)) < BAR


def test_the_autotuner_finds_a_faster_solve_for_the_jacobian(gpu, system):
    # at 1,024 right-hand sides (32 lane blocks) the Jacobian's domain tiles hold one column in
    # shared memory; the autotuner also times the lane and the global-scratch solves and keeps what
    # is fastest
    factor = GpuFactor.from_lu(gpu, system.lu)
    best = factor.autotune(FP64, 1024)
    assert best["ms"] > 0
    rhs = system.rhs[:300]
    assert worst_relative_difference(factor.solve_many(rhs), orc.solve_many_lu(system.lu, rhs, threads=8)) < BAR
