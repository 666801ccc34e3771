"""The DC callers' whole-solution paths on the GPU, through the C ABI, against the oracle:

- PTDF columns with a distributed slack (ybus_powerflow/src/dc/sensitivity.rs:101-126, 256-277:
  PTDF - (PTDF w) 1', the weights normalized), whose columns weighted by w sum to zero;
- batched DC solves with the angles placed over the buses and the flows formed on the device
  (`DcGpuStudy::solve_many`, dc/gpu.rs:214-260), with the check `DcStudy::place` makes (an angle
  not finite or above 1e5, dc.rs:558-564) returned as a flag;
- outages of one to three branches as whole solutions (`DcStudy::outage`, dc/outage.rs:126-241:
  W = D^-1 - C'Y, theta' = x + Y W^-1 C'x; `DcGpuStudy::solve_branch_outages`, dc/gpu.rs:273-322)
  against the oracle's rank-k SMW and, on a ring with chords, against refactoring the network
  without the branches (dc_outage_test.rs:103-126's property); an outage that islands a bus
  flagged singular;
- the N-1 screening's suspect flag (dc/gpu.rs:406-410)."""
import numpy as np
import pytest

import oracle.oracle as orc
from dc_cases import cpu_model, flows_of
from test_gpu_dc import BAR, ring_with_a_spur
from ybus_b200 import grids
from ybus_b200.dc import ANGLE_SUSPECT, FLOW_NOT_FINITE, DcNetwork

pytestmark = pytest.mark.gpu


def _grid2k():
    return grids.make_grid(2000, 700, grids.SEED_BASE + 1)


def _connected_without(g, removed) -> bool:
    keep = np.ones(g.n_branch, bool)
    keep[list(removed)] = False
    parent = list(range(g.n_bus))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    for f, t in zip(g.frm[keep], g.to[keep]):
        parent[find(int(f))] = find(int(t))
    return len({find(i) for i in range(g.n_bus)}) == 1


@pytest.mark.parametrize("case", ["ring", "grid2k"])
def test_distributed_slack_ptdf_columns(gpu, case):
    g = ring_with_a_spur() if case == "ring" else _grid2k()
    net = DcNetwork.from_grid(gpu, g)
    _, chol, position = cpu_model(g)
    rng = np.random.default_rng(11)
    weights = rng.uniform(0.0, 2.0, g.n_bus)
    buses = np.arange(g.n_bus) if case == "ring" else rng.choice(g.n_bus, 120, replace=False)
    single = net.ptdf_columns(buses)
    net.set_slack_weights(weights)
    shifted = net.ptdf_columns(buses)
    # the oracle: H e_j - H w, w normalized to sum to 1 (the slack's share injects nothing)
    w = weights / weights.sum()
    hw = flows_of(g, orc.solve_many(chol, w[position >= 0][None, :])[0], position)
    scale = max(1.0, np.abs(single).max())
    for j, bus in enumerate(buses):
        e = np.zeros(chol.n)
        if position[bus] >= 0:
            e[position[bus]] = 1.0
        expected = flows_of(g, orc.solve_many(chol, e[None, :])[0], position) - hw
        assert np.abs(shifted[j] - expected).max() <= BAR * scale, bus
    if case == "ring":  # every column: sum_j w_j (H e_j - H w) = H w - H w = 0
        assert np.abs(w @ shifted).max() <= BAR * scale
        assert np.abs(shifted[0] + hw).max() <= BAR * scale  # the slack's column is -H w
    # transfers do not depend on the slack, and None restores the single slack
    f, t = buses[:10], buses[::-1][:10]
    assert np.allclose(net.ptdf_transfers(f, t), single[:10] - single[::-1][:10], atol=1e-12)
    net.set_slack_weights(None)
    assert np.array_equal(net.ptdf_columns(buses), single)


def test_slack_weights_must_have_a_finite_nonzero_sum(gpu):
    from ybus_b200 import CudaError
    net = DcNetwork.from_grid(gpu, ring_with_a_spur())
    with pytest.raises(CudaError):
        net.set_slack_weights(np.zeros(7))
    with pytest.raises(CudaError):
        net.set_slack_weights(np.array([1.0, np.inf, 0, 0, 0, 0, 0]))


@pytest.mark.parametrize("case", ["ring", "grid2k"])
def test_dc_solve_many_places_angles_and_forms_flows(gpu, case):
    g = ring_with_a_spur() if case == "ring" else _grid2k()
    net = DcNetwork.from_grid(gpu, g)
    _, chol, position = cpu_model(g)
    rng = np.random.default_rng(12)
    p = rng.normal(0.0, 0.1, (40, g.n_bus))
    p[:, 0] = -p[:, 1:].sum(axis=1)
    theta, flows, flags = net.solve_many(p)
    cpu = orc.solve_many(chol, p[:, position >= 0], threads=8)
    assert (flags == 0).all()
    for s in range(p.shape[0]):
        expected = np.zeros(g.n_bus)
        expected[position >= 0] = cpu[s][position[position >= 0]]
        assert np.abs(theta[s] - expected).max() <= 1e-12 * np.abs(expected).max()
        assert theta[s][0] == 0.0
        ef = flows_of(g, cpu[s], position)
        assert np.abs(flows[s] - ef).max() <= 1e-12 * np.abs(ef).max()
    # an injection too large to trust (angles above 1e5, the reference's check) is flagged
    big = p[:2].copy()
    big[1, 1] = 1e9
    _, _, flags = net.solve_many(big)
    assert flags[0] == 0 and flags[1] & ANGLE_SUSPECT and not flags[1] & FLOW_NOT_FINITE


def ring_with_chords():
    """Six buses in a ring and its three long diagonals (every bus of degree 3): no outage of two
    branches islands a bus, some of three do."""
    frm = np.array([0, 1, 2, 3, 4, 5, 0, 1, 2])
    to = np.array([1, 2, 3, 4, 5, 0, 3, 4, 5])
    x = np.array([0.1, 0.2, 0.15, 0.3, 0.25, 0.12, 0.4, 0.35, 0.18])
    return grids.Grid(n_bus=6, frm=frm, to=to, x=x, points=np.zeros((6, 2)))


def _outage_sets(g, ks, count, seed):
    """`count` sets of k branches (k cycling through ks) whose removal keeps the grid connected."""
    rng = np.random.default_rng(seed)
    sets = []
    for _ in range(100 * count):
        if len(sets) == count:
            break
        k = ks[len(sets) % len(ks)]
        rows = sorted(rng.choice(g.n_branch, k, replace=False).tolist())
        if _connected_without(g, rows):
            sets.append(rows)
    assert len(sets) == count, "too few outage sets keep the network connected"
    return sets


@pytest.mark.parametrize("case", ["ring", "grid2k"])
def test_multi_branch_outages_match_the_oracle(gpu, case):
    g = ring_with_chords() if case == "ring" else _grid2k()
    net = DcNetwork.from_grid(gpu, g)
    _, chol, position = cpu_model(g)
    sets = _outage_sets(g, [1, 2, 3], 6 if case == "ring" else 30, 13)
    rng = np.random.default_rng(14)
    counts = rng.integers(1, 4, len(sets))
    sp = np.concatenate([[0], np.cumsum(counts)])
    p = rng.normal(0.0, 0.1, (int(sp[-1]), g.n_bus))
    p[:, 0] = -p[:, 1:].sum(axis=1)
    theta, flows, flags, singular = net.outage_solutions(sets, sp, p)
    assert not singular.any() and (flags == 0).all()
    b = g.susceptance
    solve = lambda c: orc.solve_many(chol, c[None, :])[0]
    base = orc.solve_many(chol, p[:, position >= 0], threads=8)
    for c, rows in enumerate(sets):
        for s in range(sp[c], sp[c + 1]):
            after = orc.outage_flows_smw(solve, chol.n, position, g.frm, g.to, b, rows, base[s])
            expected = np.zeros(g.n_bus)
            expected[position >= 0] = after[position[position >= 0]]
            scale = np.abs(expected).max()
            assert np.abs(theta[s] - expected).max() <= BAR * scale, (rows, s)
            ef = flows_of(g, after, position)
            ef[rows] = 0.0
            assert np.abs(flows[s] - ef).max() <= BAR * max(1.0, np.abs(ef).max()), (rows, s)
            assert (flows[s][rows] == 0.0).all()
    if case == "ring":
        # the outage's angles equal those of the network refactored without the branches
        for c, rows in enumerate(sets):
            keep = np.setdiff1d(np.arange(g.n_branch), rows)
            h = grids.Grid(n_bus=g.n_bus, frm=g.frm[keep], to=g.to[keep], x=g.x[keep], points=g.points)
            _, chol_h, pos_h = cpu_model(h)
            for s in range(sp[c], sp[c + 1]):
                direct = orc.solve_many(chol_h, p[s][None, pos_h >= 0])[0]
                expected = np.zeros(g.n_bus)
                expected[pos_h >= 0] = direct[pos_h[pos_h >= 0]]
                assert np.abs(theta[s] - expected).max() <= 1e-9 * np.abs(expected).max(), (rows, s)


def test_single_branch_outages_as_whole_solutions(gpu):
    g = _grid2k()
    net = DcNetwork.from_grid(gpu, g)
    _, chol, position = cpu_model(g)
    bridge = net.bridges()
    rng = np.random.default_rng(15)
    rows = rng.choice(np.flatnonzero(~bridge), 50, replace=False).tolist() + [int(np.flatnonzero(bridge)[0])]
    p = rng.normal(0.0, 0.1, g.n_bus)
    p[0] = -p[1:].sum()
    theta, flows, flags, singular = net.solve_branch_outages(p, rows)
    assert singular.tolist() == [False] * 50 + [True]  # the bridge's W = 1/b - c'y is zero
    base = orc.solve_many(chol, p[position >= 0][None, :])[0]
    solve = lambda c: orc.solve_many(chol, c[None, :])[0]
    for j, k in enumerate(rows[:50]):
        after = orc.outage_flows_smw(solve, chol.n, position, g.frm, g.to, g.susceptance, [k], base)
        ef = flows_of(g, after, position)
        ef[k] = 0.0
        assert np.abs(flows[j] - ef).max() <= BAR * max(1.0, np.abs(ef).max()), k
    # the bridge's case keeps the base angles (the caller decides, as the reference's CPU fallback)
    expected = np.zeros(g.n_bus)
    expected[position >= 0] = base[position[position >= 0]]
    assert np.abs(theta[50] - expected).max() <= 1e-12 * np.abs(expected).max()


def test_an_outage_that_islands_a_bus_is_singular(gpu):
    g = ring_with_chords()
    net = DcNetwork.from_grid(gpu, g)
    # bus 1's three branches 0 (0-1), 1 (1-2) and 7 (1-4) out island it; two of them do not
    p = np.zeros((2, g.n_bus))
    p[:, 2], p[:, 0] = 0.5, -0.5
    assert not _connected_without(g, [0, 1, 7]) and _connected_without(g, [0, 1])
    theta, flows, flags, singular = net.outage_solutions([[0, 1, 7], [0, 1]], [0, 1, 2], p)
    assert singular.tolist() == [True, False]


def test_screening_flags_a_scenario_with_suspect_angles(gpu):
    g = _grid2k()
    net = DcNetwork.from_grid(gpu, g)
    bridge = net.bridges()
    k = int(np.flatnonzero(~bridge)[0])
    rng = np.random.default_rng(16)
    p = rng.normal(0.0, 0.1, (3, g.n_bus))
    p[:, 0] = -p[:, 1:].sum(axis=1)
    p[2, 5] = 1e9
    rows, values, flags, sing = net.outage_loadings_batch([k], [0, 3], p)
    assert flags[0] == 0 and flags[1] == 0 and flags[2] & ANGLE_SUSPECT
    assert not sing.any()
