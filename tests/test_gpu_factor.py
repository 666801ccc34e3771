"""GPU solves against the oracle's CPU solves (ybus_cuda/tests/gpu_factor_test.rs): SPD (Cholesky)
and unsymmetric (LU with pivoting) factors, 2x2 blocks, a single row, block widths narrower and
wider than the number of right-hand sides, every tile width, repeated runs bit for bit, and the
full 10,000-bus PTDF block. All calls go through the C ABI."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import random_spd, random_square, right_hand_sides, two_by_two_blocks, worst_relative_difference
from ybus_b200 import FP32, FP64, GpuFactor, ShapeMismatch, grids, host

pytestmark = pytest.mark.gpu

# The GPU's solutions agree with the CPU's to within rounding (gpu_factor_test.rs:16)
BAR = 1e-12


def upload(gpu, f):
    return GpuFactor.from_cholesky(gpu, f) if isinstance(f, host.HostCholesky) else GpuFactor.from_lu(gpu, f)


def test_cholesky_solves_match_the_cpu_at_every_block_width(gpu):
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 37, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = upload(gpu, chol)
    for width in [1, 5, 37, 64, 1024, 4096]:
        factor.set_block_width(width)
        solved = factor.solve_many(rhs)
        d = worst_relative_difference(solved, cpu)
        assert d < BAR, f"width {width}: {d:e}"


SHARED, GLOBAL, STREAM = 1, 2, 3


@pytest.mark.parametrize("kind", [SHARED, GLOBAL])
@pytest.mark.parametrize("tile", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("threads", [64, 256, 512])
def test_every_tile_width_and_block_size(gpu, kind, tile, threads):
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 37, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = upload(gpu, chol)
    factor.set_tile(FP64, tile, threads, 1 if kind == SHARED else 2)
    factor.set_tile_kind(FP64, kind)
    d = worst_relative_difference(factor.solve_many(rhs), cpu)
    assert d < BAR, f"kind {kind} tile {tile} threads {threads}: {d:e}"


@pytest.mark.parametrize("tile", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("warps,ring,page,narrow", [(8, 4, 2048, 0), (4, 2, 1024, 0), (1, 3, 1024, 0),
                                                    (8, 4, 1024, 100000), (8, 4, 2048, 1), (16, 2, 1536, 3)])
def test_streamed_solve_every_layout(gpu, tile, warps, ring, page, narrow):
    # small pages force chunked records; narrow=100000 puts every level on warp 0 (split rows),
    # narrow=1 none; 2,000 right-hand sides make several tiles per block at tile width 1
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 37, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = upload(gpu, chol)
    factor.set_tile(FP64, tile, 256, 1)
    factor.set_tile_kind(FP64, STREAM)
    factor.set_stream(FP64, warps, ring, page, narrow)
    d = worst_relative_difference(factor.solve_many(rhs), cpu)
    assert d < BAR, f"tile {tile}: {d:e}"
    if tile == 1:
        many = right_hand_sides(300, 400, 3)
        many = np.concatenate([many] * 5)
        d = worst_relative_difference(factor.solve_many(many), orc.solve_many(chol, many))
        assert d < BAR, f"many tiles: {d:e}"
    factor.check_error()


@pytest.mark.parametrize("tile", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("tail_level", [-1, 0, 1, 2, 5])
def test_dense_tail_block(gpu, tile, tail_level):
    # the top of the tree solved as one block by its explicit inverse, from level 1 (nearly the
    # whole factor) to none, Cholesky (backward block too) and LU (where it may not close)
    chol = host.cholesky(random_spd(300, 3, 7))
    lu = host.lu(random_square(250, 4, 3))
    for f, n in ((chol, 300), (lu, 250)):
        rhs = right_hand_sides(n, 45, 11)
        cpu = orc.solve_many(f, rhs)
        factor = upload(gpu, f)
        factor.set_tile(FP64, tile, 256, 1)
        factor.set_tile_kind(FP64, STREAM)
        factor.set_stream(FP64, 8, 4, 2048, 0)
        factor.set_tail_level(FP64, tail_level)
        d = worst_relative_difference(factor.solve_many(rhs), cpu)
        assert d < BAR, f"tile {tile} tail {tail_level}: {d:e}"
        factor.check_error()


@pytest.mark.parametrize("kind", [SHARED, GLOBAL, STREAM])
def test_lu_with_every_tile_solve(gpu, kind):
    lu = host.lu(random_square(250, 4, 3))
    rhs = right_hand_sides(250, 45, 5)
    cpu = orc.solve_many(lu, rhs)
    factor = upload(gpu, lu)
    for tile in (1, 4, 16):
        factor.set_tile(FP64, tile, 256, 1)
        factor.set_tile_kind(FP64, kind)
        d = worst_relative_difference(factor.solve_many(rhs), cpu)
        assert d < BAR, f"kind {kind} tile {tile}: {d:e}"


def test_lu_solves_match_the_cpu_with_pivoting(gpu):
    lu = host.lu(random_square(250, 4, 3))
    assert any(i != p for i, p in enumerate(lu.row_perm)), "the fixture should pivot off the diagonal"
    rhs = right_hand_sides(250, 20, 5)
    cpu = orc.solve_many(lu, rhs)
    factor = upload(gpu, lu)
    factor.set_block_width(8)
    d = worst_relative_difference(factor.solve_many(rhs), cpu)
    assert d < BAR, f"{d:e}"


@pytest.mark.parametrize("kind", [0, SHARED, GLOBAL, STREAM])
def test_transposed_lu_solves_match_the_cpu(gpu, kind):
    # Lu::solve_transpose (lu.rs:506-533) as the factor of A': forward with U', back with L'
    a = random_square(250, 4, 3)
    lu = host.lu(a)
    rhs = right_hand_sides(250, 45, 5)
    cpu = orc.solve_many_lu(lu, rhs, transpose=True)
    factor = GpuFactor.from_lu_transposed(gpu, lu)
    factor.set_tile_kind(FP64, kind)
    x = factor.solve_many(rhs)
    d = worst_relative_difference(x, cpu)
    assert d < BAR, f"kind {kind}: {d:e}"
    dense = a.to_dense()
    assert np.abs(x @ dense - rhs).max() < 1e-9 * np.abs(rhs).max() * np.abs(dense).max() * 250
    # the untransposed factor of the same LU solves A x = b
    assert worst_relative_difference(upload(gpu, lu).solve_many(rhs), orc.solve_many(lu, rhs)) < BAR


def test_transposed_lu_of_a_single_row(gpu):
    lu = host.lu(host.Matrix.from_triplets(1, 1, np.array([0]), np.array([0]), np.array([-2.5]), by_rows=False))
    rhs = right_hand_sides(1, 9, 3)
    x = GpuFactor.from_lu_transposed(gpu, lu).solve_many(rhs)
    assert worst_relative_difference(x, orc.solve_many_lu(lu, rhs, transpose=True)) < BAR


def test_two_by_two_blocks_and_a_single_row(gpu):
    lu = host.lu(two_by_two_blocks(40))
    rhs = right_hand_sides(80, 3, 1)
    factor = upload(gpu, lu)
    d = worst_relative_difference(factor.solve_many(rhs), orc.solve_many(lu, rhs))
    assert d < BAR, f"{d:e}"
    # A single row, bit for bit, at block widths on both sides of 64
    one = host.lu(host.Matrix.from_triplets(1, 1, [0], [0], [3.0], by_rows=False))
    rhs = np.array([[j - 70.5] for j in range(200)])
    factor = upload(gpu, one)
    for width in [1, 64, 65, 1024]:
        factor.set_block_width(width)
        assert factor.block_width() == min(width, 64)
        assert np.array_equal(factor.solve_many(rhs), orc.solve_many(one, rhs))


def test_repeated_solves_give_the_same_bits(gpu):
    chol = host.cholesky(random_spd(500, 2, 13))
    rhs = right_hand_sides(500, 50, 17)
    factor = upload(gpu, chol)
    factor.set_block_width(16)
    first = factor.solve_many(rhs)
    factor.set_block_width(7)
    factor.set_block_width(16)
    for _ in range(3):
        again = factor.solve_many(rhs)
        assert np.array_equal(again.view(np.uint64), first.view(np.uint64))


@pytest.mark.parametrize("pinned", [False, True])
def test_host_array_solve_overlaps_many_chunks(gpu, pinned):
    # 5,000 right-hand sides pass through the copy pipeline in chunks of 625 and a halving tail
    # (625, 320, 256, 49): 10 chunks, more than twice round its 4 slots
    import torch
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 5000, 29)
    factor = upload(gpu, chol)
    b, out = np.ascontiguousarray(rhs), np.zeros_like(rhs)
    if pinned:
        tb, tx = torch.from_numpy(b).pin_memory(), torch.zeros(out.shape, dtype=torch.float64).pin_memory()
        b, out = tb.numpy(), tx.numpy()
    factor.solve_many_into(b, out)
    assert factor.timings().blocks == 10
    sample = np.arange(0, 5000, 41)
    assert worst_relative_difference(out[sample], orc.solve_many(chol, rhs[sample])) < BAR
    again = np.zeros_like(out)
    factor.set_block_width(3)  # blocks narrower than a chunk: one chunk per block
    factor.solve_many_into(b, again)
    assert np.array_equal(again[:7].view(np.uint64), out[:7].view(np.uint64)) or \
        worst_relative_difference(again[sample], out[sample]) < BAR


def test_empty_and_mismatched_right_hand_sides(gpu):
    chol = host.cholesky(random_spd(10, 20, 1))
    factor = upload(gpu, chol)
    assert factor.solve_many([]).shape[0] == 0
    with pytest.raises(ShapeMismatch) as e:
        factor.solve_many([np.zeros(10), np.zeros(9)])
    assert (e.value.expected, e.value.found) == (10, 9)
    assert factor.timings().blocks == 0
    factor.solve_many([np.ones(10)])
    assert factor.timings().blocks == 1
    factor.reset_timings()
    assert factor.timings().blocks == 0


def test_device_api_on_torch_memory_and_stream(gpu):
    import torch
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 40, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = upload(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    # a torch stream of its own (the legacy default stream's handle is 0, which means the
    # library's own stream at the C ABI)
    side = torch.cuda.Stream()
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), 40, FP64, side.cuda_stream)
    side.synchronize()
    assert worst_relative_difference(x.cpu().numpy(), cpu) < BAR
    # and on the library's own stream
    x.zero_()
    torch.cuda.synchronize()
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), 40, FP64, None)
    gpu.synchronize()
    assert worst_relative_difference(x.cpu().numpy(), cpu) < BAR


def test_fp32_substitution_is_close(gpu):
    import torch
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 40, 11)
    cpu = orc.solve_many(chol, rhs)
    factor = upload(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    for kind in (SHARED, GLOBAL, STREAM):
        for tile in [1, 4, 8, 16, 32]:
            factor.set_tile(FP32, tile, 512, 1)
            factor.set_tile_kind(FP32, kind)
            factor.solve_many_device(b.data_ptr(), x.data_ptr(), 40, FP32, None)
            gpu.synchronize()
            d = worst_relative_difference(x.cpu().numpy(), cpu)
            assert d < 1e-4, f"kind {kind} tile {tile}: {d:e}"


def _ptdf_case(n_bus, extra, seed):
    g = grids.make_grid(n_bus, extra, seed)
    r, c, v = grids.bbus_triplets(g)
    bbus = host.Matrix.from_triplets(n_bus, n_bus, r, c, v)
    keep = np.arange(1, n_bus)
    bp = bbus.select(keep, keep)
    chol = host.cholesky(bp)
    # RHS_k = b_k (e_f - e_t) over the non-slack buses
    rhs = np.zeros((g.n_branch, n_bus))
    k = np.arange(g.n_branch)
    rhs[k, g.frm] += g.susceptance
    rhs[k, g.to] -= g.susceptance
    return g, bp, chol, np.ascontiguousarray(rhs[:, 1:])


def test_full_ptdf_block_on_the_10k_grid(gpu):
    import torch
    g, bp, chol, rhs = _ptdf_case(10000, 3500, grids.SEED_BASE + 2)
    assert rhs.shape == (13499, 9999)
    factor = upload(gpu, chol)
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    torch.cuda.synchronize()
    for kind in (GLOBAL, 0):
        factor.set_tile_kind(FP64, kind)
        x.zero_()
        torch.cuda.synchronize()
        factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, None)
        gpu.synchronize()
    xs = x.cpu().numpy()
    sample = np.random.default_rng(0).choice(rhs.shape[0], 96, replace=False)
    cpu = orc.solve_many(chol, rhs[sample], threads=8)
    d = worst_relative_difference(xs[sample], cpu)
    assert d < BAR, f"{d:e}"
    # every column: relative residual at FP64 rounding level
    p, i, v = bp.arrays()
    worst = max(orc.relative_residual(p, i, v, xs[k], rhs[k]) for k in range(0, rhs.shape[0], 7))
    assert worst < 1e-11, worst


def test_the_cusparse_comparison_solves_the_same(gpu):
    # ybus_cuda's own route (cuSPARSE SpSM, libybcompare.so), kept for the bench's side-by-side
    # timing: the same solutions as the oracle, every block width, a last block padded
    import torch

    from ybus_b200 import compare
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 70, 11)
    cpu = orc.solve_many(chol, rhs)
    b = torch.from_numpy(rhs).cuda()
    for width in (1, 16, 64, 256):
        x = torch.zeros_like(b)
        ms = compare.spsm_solve(chol, b.data_ptr(), x.data_ptr(), 70, width)
        assert ms > 0
        assert worst_relative_difference(x.cpu().numpy(), cpu) < BAR, f"width {width}"


@pytest.mark.parametrize("seed", [3, 8])
def test_host_array_transposed_solve(gpu, seed):
    # Lu::solve_transpose (lu.rs:506-533) through yb_solve_many_transpose: the factor of A' made
    # from the LU factor's arrays at the first call, then kept; a Cholesky factor solves as itself
    a = random_square(250, 4, seed)
    lu = host.lu(a)
    factor = GpuFactor.from_lu(gpu, lu)
    rhs = right_hand_sides(250, 30, seed)
    cpu = orc.solve_many_lu(lu, rhs, transpose=True)
    for _ in range(2):
        assert worst_relative_difference(factor.solve_many_transpose(rhs), cpu) < 1e-12
    assert worst_relative_difference(factor.solve_many(rhs), orc.solve_many_lu(lu, rhs)) < 1e-12
    chol = host.cholesky(random_spd(120, 5, seed))
    cf = GpuFactor.from_cholesky(gpu, chol)
    r2 = right_hand_sides(120, 9, seed)
    assert np.array_equal(cf.solve_many_transpose(r2), cf.solve_many(r2))


def test_host_array_refined_solve(gpu):
    # yb_solve_many_mixed: FP32 substitution and FP64 refinement with host arrays, to the tolerance
    a = random_spd(400, 3, 5)
    chol = host.cholesky(a)
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.attach_matrix(a)
    factor.set_block_width(16)  # several blocks
    rhs = right_hand_sides(400, 50, 9)
    x, steps, ratio = factor.solve_many_mixed(rhs, 4, 1e-10)
    p, i, v = a.to_csr().arrays()
    oracle_ratio = np.array([orc.relative_residual(p, i, v, x[k], rhs[k]) for k in range(50)])
    assert ratio.max() <= 1e-10 and oracle_ratio.max() <= 1.05e-10
    assert (steps >= 1).all() and (steps <= 4).all()
    assert worst_relative_difference(x, orc.solve_many(chol, rhs)) < 1e-8
