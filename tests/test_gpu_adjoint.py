"""The adjoint of the flow loss Σ softplus(|f| − 0.8·limit)² on the synthetic 2,000-bus grid: the GPU's loss and gradients with respect to the injections
and the branch susceptances against the CPU's, computed from the oracle's solves and transposed
solve, and against central finite differences (h = 1e-6) at random coordinates."""
import numpy as np
import pytest

import oracle.oracle as orc
from ybus_b200 import grids, host
from ybus_b200.dc import DcNetwork, FlowLoss

pytestmark = pytest.mark.gpu


def setup(seed=11, count=64, n_bus=2000, extra=700):
    g = grids.make_grid(n_bus, extra, grids.SEED_BASE + seed)
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, 0.1, (count, n_bus))
    p[:, 0] = -p[:, 1:].sum(axis=1)
    limits = rng.uniform(0.5, 2.0, g.n_branch)
    return g, p, limits


def cpu(g, p, limits, x=None):
    x = g.x if x is None else x
    gg = grids.Grid(n_bus=g.n_bus, frm=g.frm, to=g.to, x=x, points=g.points)
    r, c, v = grids.bbus_triplets(gg)
    keep = np.arange(1, g.n_bus)
    chol = host.cholesky(host.Matrix.from_triplets(g.n_bus, g.n_bus, r, c, v).select(keep, keep))
    position = -np.ones(g.n_bus, np.int64)
    position[keep] = np.arange(keep.size)
    return orc.flow_loss_and_gradient(chol, g.n_bus, g.frm, g.to, 1.0 / x, position, p, limits)


def test_gradients_match_the_cpu_transposed_solve(gpu):
    g, p, limits = setup()
    net = DcNetwork.from_grid(gpu, g)
    loss_fn = FlowLoss(net, p.shape[0])
    loss, flows = loss_fn.forward(p, limits, flows=True)
    gp, gb = loss_fn.backward()
    loss_c, gp_c, gb_c = cpu(g, p, limits)
    assert abs(loss - loss_c) <= 1e-12 * abs(loss_c)
    assert np.abs(gp - gp_c).max() <= 1e-10 * np.abs(gp_c).max()
    assert np.abs(gb - gb_c).max() <= 1e-10 * np.abs(gb_c).max()
    assert (gp[:, 0] == 0.0).all()
    # a second backward gives the same bits
    gp2, gb2 = loss_fn.backward()
    assert np.array_equal(gp, gp2) and np.array_equal(gb, gb2)


def test_gradients_match_central_differences(gpu):
    # Central differences with h = 1e-6 (relative to b for the susceptances) carry a rounding noise
    # of about eps * loss / h, far above 1e-6 of a small gradient component; the error is measured
    # against the gradient's largest component
    g, p, limits = setup(seed=12, count=16, n_bus=600, extra=200)
    net = DcNetwork.from_grid(gpu, g)
    loss_fn = FlowLoss(net, p.shape[0])
    loss_fn.forward(p, limits)
    gp, gb = loss_fn.backward()
    h = 1e-6
    rng = np.random.default_rng(3)
    scale_p = np.abs(gp).max()
    for _ in range(20):
        r, i = rng.integers(p.shape[0]), rng.integers(1, g.n_bus)
        pp, pm = p.copy(), p.copy()
        pp[r, i] += h
        pm[r, i] -= h
        fd = (loss_fn.forward(pp, limits) - loss_fn.forward(pm, limits)) / (2 * h)
        assert abs(fd - gp[r, i]) <= 1e-6 * scale_p, (r, i, fd, gp[r, i])
    scale_b = np.abs(gb).max()
    b = 1.0 / g.x
    for k in rng.choice(g.n_branch, 10, replace=False):
        step = h * b[k]
        vals = []
        for sgn in (1, -1):
            x = g.x.copy()
            x[k] = 1.0 / (b[k] + sgn * step)
            vals.append(FlowLoss(DcNetwork(gpu, g.n_bus, g.frm, g.to, x), p.shape[0]).forward(p, limits))
        fd = (vals[0] - vals[1]) / (2 * step)
        assert abs(fd - gb[k]) <= 1e-6 * scale_b, (k, fd, gb[k])
