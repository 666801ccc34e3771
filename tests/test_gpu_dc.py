"""The DC callers on the GPU (ybus_powerflow/tests/cuda_dc_test.rs, dc_sensitivity_test.rs,
dc_outage_test.rs) against the oracle: PTDF columns and transfers, LODF columns with bridge
columns NaN and -1 on the outaged branch, LODF-predicted post-outage flows against the rank-one
SMW outage, and the batched N-1 screening of injection scenarios (FP64 fused, FP32 with
refinement, the CUDA graph replayed) against the oracle's rank-one outage solves. All through
the C ABI."""
import numpy as np
import pytest

import oracle.oracle as orc
from ybus_b200 import FP32, FP64, grids, host
from ybus_b200.dc import DcNetwork
from dc_cases import cpu_model, flows_of, oracle_screening

pytestmark = pytest.mark.gpu

BAR = 1e-10  # the reference's bar for its DC workloads (cuda_dc_test.rs:25)


def ring_with_a_spur():
    """Six buses in a ring plus a seventh hanging off bus 3 (its branch is a bridge)."""
    frm = np.array([0, 1, 2, 3, 4, 5, 3])
    to = np.array([1, 2, 3, 4, 5, 0, 6])
    x = np.array([0.1, 0.2, 0.15, 0.3, 0.25, 0.12, 0.2])
    return grids.Grid(n_bus=7, frm=frm, to=to, x=x, points=np.zeros((7, 2)))


@pytest.mark.parametrize("case", ["ring", "grid2k"])
def test_ptdf_columns_and_transfers_match_the_oracle(gpu, case):
    g = ring_with_a_spur() if case == "ring" else grids.make_grid(2000, 700, grids.SEED_BASE + 1)
    net = DcNetwork.from_grid(gpu, g)
    bp, chol, position = cpu_model(g)
    buses = np.arange(g.n_bus) if case == "ring" else np.random.default_rng(3).choice(g.n_bus, 150, replace=False)
    ptdf = net.ptdf_columns(buses)
    rhs = np.zeros((buses.size, chol.n))
    for j, bus in enumerate(buses):
        if position[bus] >= 0:
            rhs[j, position[bus]] = 1.0
    theta = orc.solve_many(chol, rhs)
    for j in range(buses.size):
        expected = flows_of(g, theta[j], position)
        assert np.abs(ptdf[j] - expected).max() <= BAR * max(1.0, np.abs(expected).max())
    assert np.all(ptdf[list(buses).index(0)] == 0.0) if 0 in buses else True  # the slack's column
    f, t = buses[:20], buses[::-1][:20]
    tr = net.ptdf_transfers(f, t)
    assert np.allclose(tr, ptdf[:20] - ptdf[::-1][:20], atol=1e-12)


@pytest.mark.parametrize("case", ["ring", "grid2k"])
def test_lodf_columns_mask_bridges_and_predict_outage_flows(gpu, case):
    g = ring_with_a_spur() if case == "ring" else grids.make_grid(2000, 700, grids.SEED_BASE + 1)
    net = DcNetwork.from_grid(gpu, g)
    bp, chol, position = cpu_model(g)
    bridge = net.bridges()
    assert np.array_equal(bridge, orc.bridges(g.n_bus, g.frm, g.to))
    branches = np.arange(g.n_branch) if case == "ring" else np.random.default_rng(4).choice(g.n_branch, 60, replace=False)
    lodf = net.lodf_columns(branches)
    # a base flow from random injections
    rng = np.random.default_rng(5)
    p = rng.normal(0, 0.1, g.n_bus)
    p[0] = -p[1:].sum()
    theta = orc.solve_many(chol, p[position >= 0][None, :])[0]
    base = flows_of(g, theta, position)
    b = g.susceptance
    for j, k in enumerate(branches):
        if bridge[k]:
            assert np.isnan(lodf[j]).all()
            continue
        assert lodf[j][k] == -1.0
        # post-outage flows by the rank-one SMW outage (dc/outage.rs:126-241) vs LODF's prediction
        after = orc.outage_flows_smw(lambda c: orc.solve_many(chol, c[None, :])[0], chol.n, position, g.frm, g.to, b,
                                     [k], theta)
        expected = flows_of(g, after, position)
        expected[k] = 0.0
        predicted = base + lodf[j] * base[k]
        assert np.abs(predicted - expected).max() <= 1e-9 * max(1.0, np.abs(expected).max())
    if case == "ring":
        assert bridge.tolist() == [False] * 6 + [True]


def screening_case(n_bus, extra, seed, cases, max_scen):
    g = grids.make_grid(n_bus, extra, seed)
    rng = np.random.default_rng(seed + 7)
    bridge = orc.bridges(g.n_bus, g.frm, g.to)
    outaged = rng.choice(np.flatnonzero(~bridge), cases, replace=False)
    counts = rng.integers(1, max_scen + 1, cases)
    sp = np.concatenate([[0], np.cumsum(counts)])
    inj = rng.normal(0, 0.1, (sp[-1], g.n_bus))
    inj[:, 0] = -inj[:, 1:].sum(axis=1)
    weights = 1.0 / rng.uniform(0.5, 2.0, g.n_branch)
    return g, outaged, sp, inj, weights


@pytest.mark.parametrize("precision,bar", [(FP64, 1e-10), (FP32, 1e-8)])
def test_batched_outage_screening_matches_the_oracle(gpu, precision, bar):
    g, outaged, sp, inj, weights = screening_case(2000, 700, grids.SEED_BASE + 3, 40, 8)
    net = DcNetwork.from_grid(gpu, g)
    _, chol, position = cpu_model(g)
    rows, values, bad, sing = net.outage_loadings_batch(outaged, sp, inj, weights, precision)
    assert not bad.any() and not sing.any()
    er, ev = oracle_screening(g, chol, position, outaged, sp, inj, weights)
    assert np.abs(values - ev).max() <= bar * np.abs(ev).max()
    # the same branch, unless two loadings tie to within the bar
    differ = np.flatnonzero(rows != er)
    for j in differ:
        f_gpu = values[j]
        assert abs(f_gpu - ev[j]) <= bar * ev[j]
    assert differ.size <= 1


def test_the_captured_graph_replays_new_inputs(gpu):
    g, outaged, sp, inj, weights = screening_case(2000, 700, grids.SEED_BASE + 4, 25, 5)
    net = DcNetwork.from_grid(gpu, g)
    first = net.outage_loadings_batch(outaged, sp, inj, weights)
    again = net.outage_loadings_batch(outaged, sp, inj, weights)  # replays the graph
    assert all(np.array_equal(a, b) for a, b in zip(first, again))
    scaled = net.outage_loadings_batch(outaged, sp, 2.0 * inj, weights)  # same sizes, new inputs
    assert np.array_equal(scaled[0], first[0])
    assert np.allclose(scaled[1], 2.0 * first[1], rtol=1e-12)
    other = net.outage_loadings_batch(outaged[:10], sp[:11], inj[: sp[10]], weights)  # new sizes
    assert np.array_equal(other[0], first[0][: sp[10]])
