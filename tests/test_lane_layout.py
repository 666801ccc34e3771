"""The lane solve's layout, checked on the CPU: the record streams the layout builder makes,
executed by a host interpreter of the kernel's semantics (warps between block barriers), solve the
reference's fixture matrices, the synthetic grids and pivoted LU factors (a Newton-Raphson
Jacobian among them) to the oracle's solutions, with few live values (no GPU)."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import random_spd, random_square, right_hand_sides, star_spd, worst_relative_difference
from lane_interp import run
from ybus_b200 import YbError, configs, grids, host


def grid_factor(n_bus, extra, seed):
    g = grids.make_grid(n_bus, extra, seed)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, n_bus)
    return host.cholesky(host.Matrix.from_triplets(n_bus, n_bus, r, c, v).select(keep, keep))


@pytest.mark.parametrize("warps", [1, 3, 8, 16])
@pytest.mark.parametrize("page", [256, 2048])
@pytest.mark.parametrize("fill", [2, 6, 30])
def test_lane_records_solve_the_fixture(page, fill, warps):
    # fill 30: dense columns that take several records each on the smallest page
    chol = host.cholesky(random_spd(150, fill, 7))
    rhs = right_hand_sides(150, 5, 11)
    lay = host.lane_layout(chol, 8, page, warps=warps)
    d = worst_relative_difference(run(lay, chol.n, rhs), orc.solve_many(chol, rhs))
    assert d < 1e-12, f"page {page} warps {warps}: {d:e}"
    # every entry of L below its diagonal in each sweep's records, but a dense top's (its rows
    # are then one dense map, not substitution records)
    assert lay["fwd_entries"] == lay["bwd_entries"] <= int(np.asarray(chol.l.ptr)[-1]) - chol.n
    if warps == 1:
        assert lay["fwd_entries"] == int(np.asarray(chol.l.ptr)[-1]) - chol.n


def test_lane_records_in_fp32_are_close():
    chol = host.cholesky(random_spd(200, 4, 3))
    rhs = right_hand_sides(200, 3, 5)
    lay = host.lane_layout(chol, 4, 1024, warps=4)
    assert worst_relative_difference(run(lay, chol.n, rhs), orc.solve_many(chol, rhs)) < 1e-4


@pytest.mark.parametrize("warps", [1, 4, 8])
def test_the_10k_grid_keeps_few_live_values(warps):
    chol = grid_factor(10000, 3500, grids.SEED_BASE + 2)
    lay = host.lane_layout(chol, 8, 2048, warps=warps)
    # the postorder with larger subtrees first keeps a few tens of values alive per lane
    assert lay["slots"] <= 48, lay["slots"]
    if warps > 1:
        assert lay["domains"] >= warps and lay["top"] < chol.n // 10, (lay["domains"], lay["top"])
    assert sorted(lay["in_pos"]) == list(range(chol.n))
    rhs = np.random.default_rng(3).standard_normal((2, chol.n))
    d = worst_relative_difference(run(lay, chol.n, rhs), orc.solve_many(chol, rhs))
    assert d < 1e-12, d


def test_too_many_live_values_is_refused():
    chol = host.cholesky(random_spd(120, 30, 9))
    with pytest.raises(YbError):
        host.lane_layout(chol, 8, 2048, max_slots=4)


def test_a_single_row_and_a_diagonal_matrix():
    for n, fill in ((1, 100), (40, 0)):
        for warps in (1, 4):
            chol = host.cholesky(random_spd(n, fill, 5))
            rhs = right_hand_sides(n, 3, 2)
            lay = host.lane_layout(chol, 8, 512, warps=warps)
            assert worst_relative_difference(run(lay, n, rhs), orc.solve_many(chol, rhs)) < 1e-12


def test_a_top_row_with_more_partials_than_a_record_holds():
    # a star: every leaf is a domain of its own and the hub, the one top row, takes a partial from
    # each; on 256-byte pages its sums span several records, each adding into what the last stored
    chol = host.cholesky(star_spd(200))
    rhs = right_hand_sides(200, 4, 3)
    lay = host.lane_layout(chol, 8, 256, warps=8)
    assert lay["top"] >= 1 and lay["partials"] > 14
    assert worst_relative_difference(run(lay, 200, rhs), orc.solve_many(chol, rhs)) < 1e-12


@pytest.mark.parametrize("value_bytes,warps,page", [(8, 8, 512), (8, 3, 2048), (4, 8, 1024)])
def test_two_right_hand_sides_per_lane_scale_only_the_offsets(value_bytes, warps, page):
    # with two right-hand sides per lane a slot or row holds 64 values: the same records, in the same
    # pages, with every byte offset doubled; they still solve through the interpreter
    chol = grid_factor(2000, 700, grids.SEED_BASE + 1)
    one = host.lane_layout(chol, value_bytes, page, warps=warps, rpl=1)
    two = host.lane_layout(chol, value_bytes, page, warps=warps, rpl=2)
    assert two["rpl"] == 2 and one["rpl"] == 1
    for key in ("slots", "pages", "domains", "top", "partials", "fwd_entries", "bwd_entries"):
        assert one[key] == two[key], key
    assert np.array_equal(one["warp_page"], two["warp_page"])
    assert np.array_equal(one["in_pos"], two["in_pos"]) and np.array_equal(one["out_pos"], two["out_pos"])
    rhs = np.random.default_rng(5).standard_normal((3, chol.n))
    bar = 1e-12 if value_bytes == 8 else 1e-4
    assert worst_relative_difference(run(two, chol.n, rhs), orc.solve_many(chol, rhs)) < bar
    assert not np.array_equal(one["blob"], two["blob"])


@pytest.mark.parametrize("warps", [1, 4, 8])
@pytest.mark.parametrize("seed", [3, 4])
def test_lane_records_of_a_pivoted_lu_solve_it(seed, warps):
    # a threshold-pivoted LU (P A Q = L U): U's entries need not follow L's elimination tree, so
    # the forest is the tree of both triangles' joint pattern; b's rows enter by P, x's leave by Q
    a = random_square(250, 4, seed)
    lu = host.lu(a)
    rhs = right_hand_sides(250, 6, seed + 1)
    lay = host.lane_layout(lu, 8, 1024, 256, warps)
    assert worst_relative_difference(run(lay, lu.n, rhs), orc.solve_many_lu(lu, rhs)) < 1e-12
    assert not np.array_equal(lay["in_pos"], lay["out_pos"])


@pytest.mark.parametrize("warps", [1, 8, 16])
def test_lane_records_of_a_jacobian_lu_solve_it(warps):
    # the Newton-Raphson Jacobian of a 2,000-bus network (order 3,598), AMD LU on the host
    s = configs.jacobian_system(2000, count=4)
    lay = host.lane_layout(s.lu, 8, 1024, 256, warps)
    assert lay["slots"] <= 64  # few enough for the automatic choice to take the lane solve
    assert worst_relative_difference(run(lay, s.lu.n, s.rhs), orc.solve_many_lu(s.lu, s.rhs)) < 1e-12
