"""The domain solve (one thread block per SM, the tile's vector in shared memory, per-warp
domains under a dense top block) against the oracle's CPU solves: every tile width, block shape
and cut on the reference's fixture matrices, FP32, the LU fallback and the 10,000-bus grid. All
calls go through the C ABI."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import random_spd, random_square, right_hand_sides, worst_relative_difference
from ybus_b200 import FP32, FP64, GpuFactor, grids, host

pytestmark = pytest.mark.gpu

BAR = 1e-12
DOMAIN, LANE, GLOBAL = 4, 5, 2


@pytest.mark.parametrize("tile", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("warps,ring,page,cut", [(16, 2, 2048, -1), (8, 3, 1024, -1), (4, 2, 512, 2), (1, 2, 1024, -1),
                                                 (16, 2, 2048, 1), (16, 4, 1024, 100000)])
def test_domain_solve_every_shape(gpu, tile, warps, ring, page, cut):
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 37, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_tile(FP64, tile, 256, 1)
    factor.set_tile_kind(FP64, DOMAIN)
    factor.set_domain(FP64, warps, ring, page, cut)
    d = worst_relative_difference(factor.solve_many(rhs), cpu)
    assert d < BAR, f"tile {tile}: {d:e}"
    if tile == 1:
        many = np.concatenate([right_hand_sides(300, 400, 3)] * 3)
        d = worst_relative_difference(factor.solve_many(many), orc.solve_many(chol, many))
        assert d < BAR, f"many tiles: {d:e}"
    factor.check_error()


def test_domain_solve_is_the_automatic_choice_and_repeats_bit_for_bit(gpu):
    chol = host.cholesky(random_spd(500, 2, 13))
    rhs = right_hand_sides(500, 70, 17)
    factor = GpuFactor.from_cholesky(gpu, chol)
    info = factor.domain_info(FP64)
    assert info["tile"] >= 1 and info["records"] > 0
    first = factor.solve_many(rhs)
    assert worst_relative_difference(first, orc.solve_many(chol, rhs)) < BAR
    for _ in range(3):
        assert np.array_equal(factor.solve_many(rhs).view(np.uint64), first.view(np.uint64))


def test_domain_solve_in_fp32(gpu):
    import torch
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 40, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = GpuFactor.from_cholesky(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    for tile in (1, 4, 8, 16):
        factor.set_tile(FP32, tile, 512, 1)
        factor.set_tile_kind(FP32, DOMAIN)
        factor.solve_many_device(b.data_ptr(), x.data_ptr(), 40, FP32, None)
        gpu.synchronize()
        assert worst_relative_difference(x.cpu().numpy(), cpu) < 1e-4


def test_lu_solves_with_the_automatic_choice(gpu):
    lu = host.lu(random_square(250, 4, 3))
    rhs = right_hand_sides(250, 45, 5)
    factor = GpuFactor.from_lu(gpu, lu)
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(lu, rhs))
    assert d < BAR


def test_domain_solve_on_the_10k_grid(gpu):
    import torch
    g = grids.make_grid(10000, 3500, grids.SEED_BASE + 2)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, 10000)
    bp = host.Matrix.from_triplets(10000, 10000, r, c, v).select(keep, keep)
    chol = host.cholesky(bp)
    rhs = np.random.default_rng(5).standard_normal((1000, chol.n))
    factor = GpuFactor.from_cholesky(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    for prec, bar, tile in ((FP64, BAR, 2), (FP32, 1e-3, 4)):
        assert factor.domain_info(prec)["tile"] == tile  # the automatic choice: the widest that fits
        factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], prec, None)
        gpu.synchronize()
        factor.check_error()
        xs = x.cpu().numpy()
        sample = np.arange(0, 1000, 37)
        d = worst_relative_difference(xs[sample], orc.solve_many(chol, rhs[sample], threads=8))
        assert d < bar, f"precision {prec}: {d:e}"


def test_autotune_keeps_the_fastest_domain_shape_and_the_same_solutions(gpu):
    chol = host.cholesky(random_spd(800, 2, 19))
    rhs = right_hand_sides(800, 130, 23)
    cpu = orc.solve_many(chol, rhs)
    factor = GpuFactor.from_cholesky(gpu, chol)
    for prec, bar in ((FP64, BAR), (FP32, 1e-4)):
        best = factor.autotune(prec, 256)
        assert 0 < best["ms"] < 1e3
        if best["kind"] == DOMAIN:
            assert best["warps"] in (8, 12, 16) and best["ring"] in (2, 3)
            assert best["page_bytes"] in (1536, 2048) and best["tile"] >= 1
            assert factor.domain_info(prec)["tile"] == best["tile"]
        elif best["kind"] == GLOBAL:
            assert best["tile"] in (1, 2, 4, 8, 16, 32) and best["warps"] in (8, 16)
            assert factor.tile(prec)[:2] == (best["tile"], 32 * best["warps"])
        else:
            assert best["kind"] == LANE and best["warps"] in (4, 6, 8, 12, 16) and best["tile"] == 0
            assert factor.lane_info(prec)["warps"] == best["warps"]
        if prec == FP64:
            d = worst_relative_difference(factor.solve_many(rhs), cpu)
            assert d < bar, f"{d:e}"
    factor.check_error()


def test_autotune_on_a_single_row_still_solves(gpu):
    chol = host.cholesky(random_spd(1, 100, 1))
    rhs = right_hand_sides(1, 40, 2)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.autotune(FP64, 16)
    assert worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs)) < BAR


def test_autotune_on_a_large_block_of_a_grid_keeps_the_faster_solve(gpu):
    g = grids.make_grid(2000, 700, grids.SEED_BASE + 1)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, 2000)
    chol = host.cholesky(host.Matrix.from_triplets(2000, 2000, r, c, v).select(keep, keep))
    factor = GpuFactor.from_cholesky(gpu, chol)
    best = factor.autotune(FP64, 8192)
    assert best["kind"] in (DOMAIN, LANE, GLOBAL) and best["ms"] > 0
    rhs = np.random.default_rng(9).standard_normal((300, chol.n))
    assert worst_relative_difference(factor.solve_many(rhs), orc.solve_many(chol, rhs)) < BAR
