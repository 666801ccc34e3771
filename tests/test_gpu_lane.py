"""The lane solve (one right-hand side per lane, the factor's rows in an elimination-tree postorder,
b and x through a work array in solve order) against the oracle's CPU solves: counts around a
warp's 32, dense columns split over several records, FP32, leading dimensions above n, repeats bit
for bit, and the 10,000-bus grid. All calls go through the C ABI."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import random_spd, random_square, right_hand_sides, star_spd, worst_relative_difference
from ybus_b200 import FP32, FP64, CudaError, GpuFactor, grids, host

pytestmark = pytest.mark.gpu

BAR = 1e-12
LANE = 5


@pytest.mark.parametrize("warps", [1, 2, 4, 8, 9, 16])
@pytest.mark.parametrize("count", [1, 31, 32, 33, 200])
def test_lane_solve_matches_the_cpu(gpu, count, warps):
    # 9 and 16: the kernel instance for blocks of more than 8 warps, one block an SM
    chol = host.cholesky(random_spd(200, 3, 7))
    rhs = right_hand_sides(200, count, 11)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    factor.set_lane(FP64, warps)
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs))
    assert d < BAR, f"count {count} warps {warps}: {d:e}"
    factor.check_error()


@pytest.mark.parametrize("warps", [1, 3])
def test_dense_columns_over_several_records(gpu, warps):
    # 512-byte pages hold 31 entries: the dense columns take several records each
    chol = host.cholesky(random_spd(150, 30, 7))
    rhs = right_hand_sides(150, 70, 3)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    factor.set_lane(FP64, warps, 512)
    info = factor.lane_info(FP64)
    assert info["slots"] >= 1 and info["pages"] >= 1 and info["page_bytes"] == 512
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs))
    assert d < BAR, f"{d:e}"


@pytest.mark.parametrize("prec,bar", [(FP64, BAR), (FP32, 1e-4)])
def test_a_top_row_with_partials_over_several_records(gpu, prec, bar):
    # a star: 199 one-row domains update the hub, the one top row; on 256-byte pages its partial
    # sums take several records in a row, run by one warp
    chol = host.cholesky(star_spd(200))
    rhs = right_hand_sides(200, 70, 5)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(prec, LANE)
    factor.set_lane(prec, 8, 256)
    info = factor.lane_info(prec)
    assert info["top"] >= 1 and info["partials"] > 14
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs))
    assert d < bar, f"{d:e}"
    factor.check_error()


def test_device_arrays_with_leading_dimensions_and_fp32(gpu):
    import torch
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 45, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = GpuFactor.from_cholesky(gpu, chol)
    for prec, bar in ((FP64, BAR), (FP32, 1e-4)):
        factor.set_tile_kind(prec, LANE)
        b = torch.zeros((45, 310), dtype=torch.float64, device="cuda")
        b[:, :300] = torch.from_numpy(rhs).cuda()
        x = torch.full((45, 320), 7.0, dtype=torch.float64, device="cuda")
        factor.solve_many_device(b.data_ptr(), x.data_ptr(), 45, prec, None, ldb=310, ldx=320)
        gpu.synchronize()
        xs = x.cpu().numpy()
        assert worst_relative_difference(xs[:, :300], cpu) < bar
        assert np.all(xs[:, 300:] == 7.0), "rows past n are not written"


def test_repeated_lane_solves_give_the_same_bits(gpu):
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 100, 17)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    first = factor.solve_many(rhs)
    for _ in range(3):
        assert np.array_equal(factor.solve_many(rhs).view(np.uint64), first.view(np.uint64))


def test_the_automatic_choice_takes_the_lane_solve_from_its_threshold(gpu):
    chol = host.cholesky(random_spd(120, 3, 9))
    rhs = right_hand_sides(120, 96, 5)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_lane_min_count(FP64, 64)
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs))
    assert d < BAR


def test_an_lu_factor_solves_or_is_refused(gpu):
    lu = host.lu(random_square(250, 4, 3))
    rhs = right_hand_sides(250, 40, 5)
    factor = GpuFactor.from_lu(gpu, lu)
    factor.set_tile_kind(FP64, LANE)
    try:
        factor.lane_info(FP64)
    except CudaError:
        with pytest.raises(CudaError):
            factor.solve_many(rhs)
        return
    assert worst_relative_difference(factor.solve_many(rhs), orc.solve_many(lu, rhs)) < BAR


def test_lane_solve_on_the_10k_grid(gpu):
    import torch
    g = grids.make_grid(10000, 3500, grids.SEED_BASE + 2)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, 10000)
    bp = host.Matrix.from_triplets(10000, 10000, r, c, v).select(keep, keep)
    chol = host.cholesky(bp)
    rhs = np.random.default_rng(5).standard_normal((1000, chol.n))
    factor = GpuFactor.from_cholesky(gpu, chol)
    assert factor.lane_info(FP64)["slots"] <= 48
    # its domain tiles hold two columns: the automatic choice keeps the domain solve below 1,536
    assert factor.domain_info(FP64)["tile"] >= 2 and factor.lane_min_count(FP64) == 1536
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    for prec, bar, warps in ((FP64, BAR, 1), (FP64, BAR, 6), (FP64, BAR, 8), (FP64, BAR, 12), (FP64, BAR, 16),
                             (FP32, 1e-3, 4), (FP32, 1e-3, 16)):
        factor.set_tile_kind(prec, LANE)
        factor.set_lane(prec, warps)
        assert factor.lane_info(prec)["warps"] == warps
        x.zero_()
        factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], prec, None)
        gpu.synchronize()
        factor.check_error()
        xs = x.cpu().numpy()
        sample = np.arange(0, 1000, 37)
        d = worst_relative_difference(xs[sample], orc.solve_many(chol, rhs[sample], threads=8))
        assert d < bar, f"precision {prec}: {d:e}"
        if prec == FP64:
            p, i, v = bp.arrays()
            assert max(orc.relative_residual(p, i, v, xs[k], rhs[k]) for k in range(0, 1000, 97)) < 1e-11


def test_a_factor_with_too_many_live_values_takes_another_solve(gpu):
    # a random pattern keeps hundreds of values alive: the automatic choice passes the lane solve by
    chol = host.cholesky(random_spd(500, 2, 13))
    rhs = right_hand_sides(500, 64, 17)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_lane_min_count(FP64, 0)
    with pytest.raises(CudaError):
        factor.lane_info(FP64)
    assert worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs)) < BAR


def test_a_block_larger_than_one_launch_of_work(gpu):
    # 27,000 right-hand sides of the 10,000-bus grid need 2.2 GB of work array, over the 2 GB one
    # launch fills: two launches, checked on both sides of their boundary
    import torch
    g = grids.make_grid(10000, 3500, grids.SEED_BASE + 2)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, 10000)
    chol = host.cholesky(host.Matrix.from_triplets(10000, 10000, r, c, v).select(keep, keep))
    count = 27000
    gen = torch.Generator(device="cuda").manual_seed(3)
    b = torch.randn((count, chol.n), dtype=torch.float64, device="cuda", generator=gen)
    x = torch.full_like(b, float("nan"))
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), count, FP64, None)
    gpu.synchronize()
    factor.check_error()
    per_launch = (2 << 30) // (chol.n * 32 * 8) * 32  # right-hand sides one launch takes
    assert per_launch < count
    sample = np.unique(np.r_[0, 1, per_launch - 1, per_launch, per_launch + 1, count - 1, np.arange(5, count, 1777)])
    idx = torch.from_numpy(sample).cuda()
    bs, xs = b[idx].cpu().numpy(), x[idx].cpu().numpy()
    assert not np.isnan(xs).any()
    assert worst_relative_difference(xs, orc.solve_many(chol, bs, threads=8)) < BAR


def test_lane_launch_times_are_recorded_when_asked(gpu):
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 100, 11)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(FP64, LANE)
    factor.solve_many(rhs)
    assert factor.lane_times()["launches"] == 0, "nothing is recorded while timing is off"
    factor.time_lane(True)
    x = factor.solve_many(rhs)
    factor.solve_many(rhs)
    t = factor.lane_times()
    assert t["launches"] == 2 and t["gather_ms"] > 0 and t["solve_ms"] > 0 and t["scatter_ms"] > 0
    assert factor.lane_times()["launches"] == 0, "a read clears the record"
    factor.time_lane(False)
    factor.solve_many(rhs)
    assert factor.lane_times()["launches"] == 0
    assert worst_relative_difference(x, orc.solve_many(chol, rhs)) < BAR


# ---- two right-hand sides per lane (64 per block) --------------------------------------------------

@pytest.mark.parametrize("warps", [1, 3, 8])
@pytest.mark.parametrize("count", [1, 63, 64, 65, 200])
@pytest.mark.parametrize("prec,bar", [(FP64, BAR), (FP32, 1e-4)])
def test_two_per_lane_matches_the_cpu(gpu, count, warps, prec, bar):
    chol = host.cholesky(random_spd(200, 3, 7))
    rhs = right_hand_sides(200, count, 11)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile_kind(prec, LANE)
    factor.set_lane(prec, warps)
    factor.set_lane_rhs_per_lane(prec, 2)
    assert factor.lane_info(prec)["rpl"] == 2
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs))
    assert d < bar, f"count {count} warps {warps}: {d:e}"
    factor.check_error()


@pytest.mark.parametrize("page", [256, 512])
def test_two_per_lane_with_records_split_over_pages(gpu, page):
    # dense columns and a star's top row: records and partial sums over several records
    for chol in (host.cholesky(random_spd(150, 30, 7)), host.cholesky(star_spd(200))):
        rhs = right_hand_sides(chol.n, 90, 3)
        factor = GpuFactor.from_cholesky(gpu, chol)
        factor.set_tile_kind(FP64, LANE)
        factor.set_lane(FP64, 8, page)
        factor.set_lane_rhs_per_lane(FP64, 2)
        d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs))
        assert d < BAR, f"{d:e}"
        factor.check_error()


def test_two_per_lane_on_the_10k_grid_and_the_same_bits_as_one(gpu):
    # the full 13,499-column PTDF block with the automatic layout for two per lane, against the
    # oracle on sampled columns; and on one layout (8 warps, 512-byte pages) for both, column for
    # column the same bits as one right-hand side per lane (the same operations in the same order;
    # layouts of other warp counts cut other domains and sum in another order)
    import torch
    from ybus_b200 import configs
    g = configs.grid_10k()
    chol = host.cholesky(configs.bprime(g))
    rhs = configs.branch_rhs(g)
    factor = GpuFactor.from_cholesky(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    x1, x2 = torch.empty_like(b), torch.empty_like(b)
    factor.set_tile_kind(FP64, LANE)
    factor.set_lane_rhs_per_lane(FP64, 2)
    factor.solve_many_device(b.data_ptr(), x2.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    factor.check_error()
    sample = np.arange(0, rhs.shape[0], 211)
    assert worst_relative_difference(x2.cpu().numpy()[sample], orc.solve_many(chol, rhs[sample], threads=8)) < BAR
    factor.set_lane(FP64, 8, 512)
    factor.solve_many_device(b.data_ptr(), x2.data_ptr(), rhs.shape[0], FP64, None)
    factor.set_lane_rhs_per_lane(FP64, 1)
    factor.solve_many_device(b.data_ptr(), x1.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    factor.check_error()
    assert np.array_equal(x1.cpu().numpy(), x2.cpu().numpy())
