"""DC helpers of the GPU tests: B′ over the unknowns with its oracle factor, branch flows from
angles, and the oracle's N-1 screening of injection scenarios (the rank-one SMW outage of
ybus_powerflow/src/dc/outage.rs:126-241 per scenario, then the column maximum of
ybus_cuda/src/kernels.cu:78-128)."""
import numpy as np

import oracle.oracle as orc
from ybus_b200 import grids, host


def cpu_model(g, slack=0):
    """B′ over the unknowns, its oracle factor, Bf over the buses, and the unknown of each bus."""
    r, c, v = grids.bbus_triplets(g)
    keep = np.array([i for i in range(g.n_bus) if i != slack])
    bp = host.Matrix.from_triplets(g.n_bus, g.n_bus, r, c, v).select(keep, keep)
    chol = host.cholesky(bp)
    position = -np.ones(g.n_bus, np.int64)
    position[keep] = np.arange(keep.size)
    return bp, chol, position


def flows_of(g, theta_unknown, position):
    """b (theta_from - theta_to) per branch, the slack's angle 0 (Bf's stamps)."""
    th = np.zeros(g.n_bus)
    th[position >= 0] = theta_unknown[position[position >= 0]]
    b = g.susceptance
    return b * th[g.frm] + (-b) * th[g.to]


def oracle_screening(g, chol, position, outaged, sp, inj, weights):
    b = g.susceptance
    solve = lambda c: orc.solve_many(chol, c[None, :])[0]
    rows, values = [], []
    for c, k in enumerate(outaged):
        scen = inj[sp[c]:sp[c + 1]]
        thetas = orc.solve_many(chol, scen[:, position >= 0])
        for theta in thetas:
            after = orc.outage_flows_smw(solve, chol.n, position, g.frm, g.to, b, [k], theta)
            f = flows_of(g, after, position)
            f[k] = 0.0
            row, value, bad = orc.column_max(f, weights)
            rows.append(-1 if row is None else row)
            values.append(value)
    return np.array(rows), np.array(values)
