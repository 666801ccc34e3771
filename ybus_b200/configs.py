"""The seeded synthetic workloads of the solve path, one builder per configuration, shared by the
parity tests and the bench so that both run the same inputs.

Every grid comes from `grids.make_grid` (points in the unit square, a random spanning tree of the
k = 4 nearest-neighbour graph plus extra neighbour edges, x log-uniform in [0.005, 0.5], bus 0 the
slack); seeds are `grids.SEED_BASE + configuration number`.

1. 2,000 buses, 700 extra edges (2,699 branches); 256 unit right-hand sides e_j, j uniform over
   the non-slack buses; FP64.
2. 10,000 buses, 3,500 extra edges (13,499 branches); the 13,499 branch right-hand sides
   A'diag(1/x)e_k over the non-slack buses (b_k (e_f - e_t), the slack's entry dropped).
3. The 10,000-bus grid; 2,000 distinct non-bridge outages; per outage U[1, 64] injection scenarios
   p ~ N(0, 0.1) at every bus with the slack taking the balance; branch weights 1 / U[0.5, 2].
4. The 10,000-bus grid; 1,024 injection scenarios as in 3; branch limits U[0.5, 2.0].
5. 16 complex Ybus networks of N log-uniform in [500, 70,000] buses (1.3 branches per bus, r/x in
   [0.1, 0.5], shunt b in [0, 0.05]); 128 complex right-hand sides N(0,1) + iN(0,1) each.

Beside them, the Newton-Raphson Jacobian of a complex network (the reference's other matrix for its
GPU survey, ybus_powerflow/examples/cuda_survey.rs:213-235): bus 0 the slack, a fifth of the
others PV, voltages near flat, LU-factored with AMD as the survey does.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import grids, host

N_BUS_SMALL, EXTRA_SMALL = 2000, 700
N_BUS, EXTRA = 10000, 3500
N1_OUTAGES, N1_MAX_SCENARIOS = 2000, 64
ADJOINT_SCENARIOS = 1024
COMPLEX_NETWORKS, COMPLEX_RANGE, COMPLEX_RHS = 16, (500, 70000), 128


def bprime(g: grids.Grid, slack: int = 0) -> host.Matrix:
    """B' of a grid: Bbus (ybus's `Bdc::new` stamps) without the slack's row and column."""
    r, c, v = grids.bbus_triplets(g)
    keep = np.array([i for i in range(g.n_bus) if i != slack], np.int64)
    return host.Matrix.from_triplets(g.n_bus, g.n_bus, r, c, v).select(keep, keep)


def branch_rhs(g: grids.Grid) -> np.ndarray:
    """(n_branch, n_bus - 1): column k of A'diag(1/x) over the non-slack buses (slack bus 0)."""
    rhs = np.zeros((g.n_branch, g.n_bus))
    k = np.arange(g.n_branch)
    rhs[k, g.frm] += g.susceptance
    rhs[k, g.to] -= g.susceptance
    return np.ascontiguousarray(rhs[:, 1:])


def grid_small() -> grids.Grid:
    return grids.make_grid(N_BUS_SMALL, EXTRA_SMALL, grids.SEED_BASE + 1)


def grid_10k() -> grids.Grid:
    return grids.make_grid(N_BUS, EXTRA, grids.SEED_BASE + 2)


def unit_rhs_2k(count: int = 256) -> tuple[grids.Grid, np.ndarray]:
    """Configuration 1: the 2,000-bus grid and `count` unit right-hand sides over its unknowns."""
    g = grid_small()
    rng = np.random.default_rng(grids.SEED_BASE + 1)
    j = rng.integers(1, g.n_bus, count)  # buses 1..N-1; unknown j - 1
    rhs = np.zeros((count, g.n_bus - 1))
    rhs[np.arange(count), j - 1] = 1.0
    return g, rhs


@dataclasses.dataclass
class N1Cases:
    grid: grids.Grid
    outaged: np.ndarray  # int64 [cases]
    scenario_ptr: np.ndarray  # int64 [cases + 1]
    injections: np.ndarray  # float64 [scenarios, n_bus]
    weights: np.ndarray  # float64 [n_branch]


def n1_cases(g: grids.Grid, bridge: np.ndarray, outages: int = N1_OUTAGES, max_scenarios: int = N1_MAX_SCENARIOS,
             seed: int = grids.SEED_BASE + 3) -> N1Cases:
    """Configuration 3 on grid `g` with its bridge flags: distinct non-bridge outages, each with
    U[1, max_scenarios] injection scenarios summing to zero against the slack (bus 0)."""
    rng = np.random.default_rng(seed)
    outaged = rng.choice(np.flatnonzero(~np.asarray(bridge, bool)), outages, replace=False)
    counts = rng.integers(1, max_scenarios + 1, outaged.size)
    sp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    inj = rng.normal(0.0, 0.1, (int(sp[-1]), g.n_bus))
    inj[:, 0] = -inj[:, 1:].sum(axis=1)
    weights = 1.0 / rng.uniform(0.5, 2.0, g.n_branch)
    return N1Cases(g, outaged.astype(np.int64), sp, inj, weights)


def adjoint_scenarios(g: grids.Grid, count: int = ADJOINT_SCENARIOS,
                      seed: int = grids.SEED_BASE + 4) -> tuple[np.ndarray, np.ndarray]:
    """Configuration 4 on grid `g`: (injections (count, n_bus), branch limits (n_branch))."""
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, 0.1, (count, g.n_bus))
    p[:, 0] = -p[:, 1:].sum(axis=1)
    limits = rng.uniform(0.5, 2.0, g.n_branch)
    return p, limits


def complex_sizes(networks: int = COMPLEX_NETWORKS, seed: int = grids.SEED_BASE + 5) -> np.ndarray:
    """Configuration 5's network orders, log-uniform over the range, largest first."""
    rng = np.random.default_rng(seed)
    lo, hi = COMPLEX_RANGE
    return np.sort(np.exp(rng.uniform(np.log(lo), np.log(hi), networks)).astype(int))[::-1]


@dataclasses.dataclass
class ComplexNetwork:
    n: int
    ybus: host.Matrix  # CSC, complex128
    lu: host.HostLu
    rhs: np.ndarray  # complex128 (count, n)


def complex_network(n_bus: int, index: int, count: int = COMPLEX_RHS, seed: int = grids.SEED_BASE + 5) -> ComplexNetwork:
    """Network `index` of configuration 5: its Ybus (pi-model stamps), COLAMD LU and right-hand sides."""
    gc = grids.make_complex_grid(int(n_bus), grids.SEED_BASE + 60 + index)
    r, c, v = grids.ybus_triplets(gc)
    a = host.Matrix.from_triplets(int(n_bus), int(n_bus), r, c, v, by_rows=False)
    rng = np.random.default_rng(seed * 100 + index)
    b = rng.standard_normal((count, int(n_bus))) + 1j * rng.standard_normal((count, int(n_bus)))
    return ComplexNetwork(int(n_bus), a, host.lu(a, host.COLAMD), b)


JACOBIAN_PV_SHARE, JACOBIAN_RHS = 0.2, 4096


@dataclasses.dataclass
class JacobianSystem:
    n_bus: int
    pv: np.ndarray  # int64: the PV buses
    pq: np.ndarray  # int64: the PQ buses
    voltage: np.ndarray  # complex128 [n_bus]
    ybus: object  # scipy CSC, complex128
    jacobian: host.Matrix  # CSC, float64, (len(pv) + 2 len(pq)) square
    lu: host.HostLu
    rhs: np.ndarray  # float64 (count, order)


def power_injections(ybus, v: np.ndarray) -> np.ndarray:
    """S = V conj(Ybus V) at every bus (`newtonpf`'s mismatch without the schedule)."""
    return v * np.conj(ybus @ v)


def jacobian_matrix(ybus, v: np.ndarray, pv: np.ndarray, pq: np.ndarray):
    """The Newton-Raphson Jacobian at voltages `v` (`AcModel::jacobian`, ybus_powerflow/src/ac.rs:
    1134-1150): the real power at the PV and PQ buses and the reactive power at the PQ buses
    differentiated by the angles at the PV and PQ buses and the magnitudes at the PQ buses, in that
    order, from the published derivatives of S = V conj(Ybus V):
    dS/dtheta = j diag(V) conj(diag(I) - Ybus diag(V)) and
    dS/d|V| = diag(V) conj(Ybus diag(V/|V|)) + conj(diag(I)) diag(V/|V|), I = Ybus V.
    Returns a scipy CSC matrix."""
    import scipy.sparse as sp
    i = ybus @ v
    dv = sp.diags(v)
    dn = sp.diags(v / np.abs(v))
    ds_da = 1j * dv @ np.conj(sp.diags(i) - ybus @ dv)
    ds_dm = dv @ np.conj(ybus @ dn) + np.conj(sp.diags(i)) @ dn
    pvpq = np.concatenate([pv, pq])
    ds_da, ds_dm = sp.csr_matrix(ds_da), sp.csr_matrix(ds_dm)
    j11 = ds_da[pvpq][:, pvpq].real
    j12 = ds_dm[pvpq][:, pq].real
    j21 = ds_da[pq][:, pvpq].imag
    j22 = ds_dm[pq][:, pq].imag
    return sp.bmat([[j11, j12], [j21, j22]], format="csc")


def jacobian_system(n_bus: int = N_BUS, count: int = JACOBIAN_RHS, seed: int = grids.SEED_BASE + 7) -> JacobianSystem:
    """The Jacobian of a seeded complex network of `n_bus` buses, its AMD LU on the host and
    `count` right-hand sides N(0, 1)."""
    import scipy.sparse as sp
    gc = grids.make_complex_grid(int(n_bus), seed)
    r, c, v = grids.ybus_triplets(gc)
    ybus = sp.csc_matrix((v, (r, c)), shape=(n_bus, n_bus))
    rng = np.random.default_rng(seed)
    others = np.arange(1, n_bus)
    pv = np.sort(rng.choice(others, int(round(JACOBIAN_PV_SHARE * others.size)), replace=False)).astype(np.int64)
    pq = np.setdiff1d(others, pv).astype(np.int64)
    vm = rng.uniform(0.95, 1.05, n_bus)
    va = rng.normal(0.0, 0.05, n_bus)
    va[0] = 0.0
    voltage = vm * np.exp(1j * va)
    jm = jacobian_matrix(ybus, voltage, pv, pq).tocoo()
    m = jm.shape[0]
    jac = host.Matrix.from_triplets(m, m, jm.row.astype(np.int64), jm.col.astype(np.int64), jm.data, by_rows=False)
    lu = host.lu(jac, host.AMD)
    rhs = np.random.default_rng(seed + 1).standard_normal((count, m))
    return JacobianSystem(int(n_bus), pv, pq, voltage, ybus, jac, lu, rhs)
