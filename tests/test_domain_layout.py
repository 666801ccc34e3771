"""The domain solve's layout, checked on the CPU: the record streams the layout builder makes,
executed by a host interpreter of the kernel's semantics, solve the reference's fixture matrices
and the synthetic grids to the oracle's solutions (no GPU)."""
import numpy as np
import pytest

import oracle.oracle as orc
from domain_interp import parse, run
from fixtures import random_spd, right_hand_sides, worst_relative_difference
from ybus_b200 import grids, host


def slots(chol):
    in_slot = np.empty(chol.n, np.int64)
    in_slot[chol.perm] = np.arange(chol.n)
    return in_slot


def grid_factor(n_bus, extra, seed):
    g = grids.make_grid(n_bus, extra, seed)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, n_bus)
    return host.cholesky(host.Matrix.from_triplets(n_bus, n_bus, r, c, v).select(keep, keep))


@pytest.mark.parametrize("cut", [-1, 1, 3, 6, 100])
@pytest.mark.parametrize("warps,page", [(16, 2048), (4, 1024), (1, 512)])
def test_domain_records_solve_the_fixture(cut, warps, page):
    chol = host.cholesky(random_spd(300, 3, 7))
    rhs = right_hand_sides(300, 5, 11)
    lay = host.domain_layout(chol, 8, warps, page, cut)
    s = slots(chol)
    d = worst_relative_difference(run(lay, chol.n, s, s, rhs), orc.solve_many(chol, rhs))
    assert d < 1e-12, f"cut {cut} (chosen {lay['cut']}, top {lay['top']}): {d:e}"


def test_domain_records_in_fp32_are_close():
    chol = host.cholesky(random_spd(200, 4, 3))
    rhs = right_hand_sides(200, 3, 5)
    lay = host.domain_layout(chol, 4, 8, 1024, -1)
    s = slots(chol)
    assert worst_relative_difference(run(lay, chol.n, s, s, rhs), orc.solve_many(chol, rhs)) < 1e-4


def test_domain_layout_of_the_2000_bus_grid():
    chol = grid_factor(2000, 700, grids.SEED_BASE + 1)
    rhs = np.random.default_rng(3).standard_normal((3, chol.n))
    lay = host.domain_layout(chol, 8, 16, 2048, -1)
    assert 0 < lay["top"] <= 768 and lay["stages"] == 6
    # every row appears exactly once per sweep; lanes per row times rows never exceed a warp
    recs = [r for w in parse(lay) for r in w]
    assert all(r[2][0].shape[0] << r[2][5] <= 32 for r in recs if r[1] == 4)
    s = slots(chol)
    d = worst_relative_difference(run(lay, chol.n, s, s, rhs), orc.solve_many(chol, rhs))
    assert d < 1e-12, d


def test_a_cut_with_no_top_block_needs_no_barrier():
    chol = host.cholesky(random_spd(120, 3, 9))
    lay = host.domain_layout(chol, 8, 16, 2048, 10_000)
    assert lay["top"] == 0 and lay["stages"] == 1
    rhs = right_hand_sides(120, 2, 1)
    s = slots(chol)
    assert worst_relative_difference(run(lay, chol.n, s, s, rhs), orc.solve_many(chol, rhs)) < 1e-12


def test_layout_rejects_bad_shapes():
    chol = host.cholesky(random_spd(50, 5, 2))
    with pytest.raises(Exception):
        host.domain_layout(chol, 6, 16, 2048, -1)
    with pytest.raises(Exception):
        host.domain_layout(chol, 8, 16, 100, -1)
