"""Seeded synthetic power grids for the solve path's workloads.

Each grid is a connected network of ``n_bus`` buses placed uniformly in the unit square:

1. the k=4 nearest-neighbour graph of the points, symmetrised;
2. a random spanning tree of that graph (Kruskal over uniform random edge weights); if the
   neighbour graph is disconnected, its components are joined by their nearest pairs of points;
3. ``extra`` further distinct neighbour edges not in the tree, drawn uniformly;
4. branch reactance x log-uniform in [0.005, 0.5] (p.u.); bus 0 is the slack.

The DC matrices follow ybus's ``Bdc::new`` (ybus_powerflow/src/dc.rs:79-113): each branch of
susceptance b = 1/x stamps (f,f,+b), (f,t,-b), (t,f,-b), (t,t,+b) into Bbus and (k,f,+b),
(k,t,-b) into Bf; B' is Bbus over the non-slack buses.

The complex networks of the multi-network batch add a series resistance r = x * U[0.1, 0.5] and a
shunt susceptance U[0, 0.05] split over the branch ends, stamped as the pi model of
ybus_powerflow/src/ac.rs:56-190 (Ys = 1/(r + jx), Bc/2 at each end, no taps).
"""
from __future__ import annotations

import dataclasses

import numpy as np
from scipy.spatial import cKDTree

SEED_BASE = 20261203


@dataclasses.dataclass
class Grid:
    n_bus: int
    frm: np.ndarray  # int64 [n_branch]
    to: np.ndarray  # int64 [n_branch]
    x: np.ndarray  # float64 [n_branch]
    points: np.ndarray  # float64 [n_bus, 2]
    r: np.ndarray | None = None
    shunt_b: np.ndarray | None = None

    @property
    def n_branch(self) -> int:
        return int(self.frm.size)

    @property
    def susceptance(self) -> np.ndarray:
        return 1.0 / self.x


class _UnionFind:
    def __init__(self, n: int):
        self.parent = np.arange(n)

    def find(self, a: int) -> int:
        parent = self.parent
        root = a
        while parent[root] != root:
            root = parent[root]
        while parent[a] != root:
            parent[a], a = root, parent[a]
        return root

    def union(self, a: int, b: int) -> bool:
        ra, rb = self.find(a), self.find(b)
        if ra == rb:
            return False
        self.parent[rb] = ra
        return True


def _knn_edges(points: np.ndarray, k: int) -> np.ndarray:
    tree = cKDTree(points)
    _, nearest = tree.query(points, k=k + 1)
    i = np.repeat(np.arange(points.shape[0]), k)
    j = nearest[:, 1:].reshape(-1)
    a, b = np.minimum(i, j), np.maximum(i, j)
    keep = a != b
    edges = np.unique(np.stack([a[keep], b[keep]], axis=1), axis=0)
    return edges.astype(np.int64)


def make_grid(n_bus: int, extra: int, seed: int, k: int = 4,
              x_range: tuple[float, float] = (0.005, 0.5)) -> Grid:
    """A connected grid of ``n_bus`` buses with ``n_bus - 1 + extra`` branches."""
    rng = np.random.default_rng(seed)
    points = rng.random((n_bus, 2))
    edges = _knn_edges(points, k)
    weights = rng.random(edges.shape[0])
    order = np.argsort(weights, kind="stable")
    uf = _UnionFind(n_bus)
    in_tree = np.zeros(edges.shape[0], dtype=bool)
    tree_edges = []
    for e in order:
        a, b = int(edges[e, 0]), int(edges[e, 1])
        if uf.union(a, b):
            in_tree[e] = True
            tree_edges.append((a, b))
    # Join components by their nearest pairs of points, smallest component first
    roots = np.array([uf.find(i) for i in range(n_bus)])
    while np.unique(roots).size > 1:
        labels, counts = np.unique(roots, return_counts=True)
        small = labels[np.argmin(counts)]
        inside = np.flatnonzero(roots == small)
        outside = np.flatnonzero(roots != small)
        dist, near = cKDTree(points[outside]).query(points[inside], k=1)
        best = int(np.argmin(dist))
        a, b = int(inside[best]), int(outside[near[best]])
        uf.union(a, b)
        tree_edges.append((min(a, b), max(a, b)))
        roots = np.array([uf.find(i) for i in range(n_bus)])
    candidates = np.flatnonzero(~in_tree)
    extra = min(extra, candidates.size)
    chosen = np.sort(rng.choice(candidates, size=extra, replace=False)) if extra else np.zeros(0, np.int64)
    all_edges = np.concatenate([np.array(tree_edges, dtype=np.int64).reshape(-1, 2), edges[chosen]])
    lo, hi = np.log(x_range[0]), np.log(x_range[1])
    x = np.exp(rng.uniform(lo, hi, size=all_edges.shape[0]))
    return Grid(n_bus=n_bus, frm=all_edges[:, 0].copy(), to=all_edges[:, 1].copy(), x=x, points=points)


def make_complex_grid(n_bus: int, seed: int) -> Grid:
    """A grid for the complex batch: 1.3 branches per bus, r/x in [0.1, 0.5], shunt b in [0, 0.05]."""
    extra = int(round(0.3 * n_bus)) + 1
    g = make_grid(n_bus, extra, seed)
    rng = np.random.default_rng(seed + 1)
    g.r = g.x * rng.uniform(0.1, 0.5, size=g.n_branch)
    g.shunt_b = rng.uniform(0.0, 0.05, size=g.n_branch)
    return g


def bbus_triplets(g: Grid):
    """Bbus stamps in ybus's order: per branch (f,f,b), (f,t,-b), (t,f,-b), (t,t,b)."""
    b = g.susceptance
    rows = np.stack([g.frm, g.frm, g.to, g.to], axis=1).reshape(-1)
    cols = np.stack([g.frm, g.to, g.frm, g.to], axis=1).reshape(-1)
    vals = np.stack([b, -b, -b, b], axis=1).reshape(-1)
    return rows.astype(np.int64), cols.astype(np.int64), vals.astype(np.float64)


def bf_triplets(g: Grid):
    """Bf stamps: per branch k, (k,f,b), (k,t,-b)."""
    b = g.susceptance
    k = np.arange(g.n_branch, dtype=np.int64)
    rows = np.stack([k, k], axis=1).reshape(-1)
    cols = np.stack([g.frm, g.to], axis=1).reshape(-1)
    vals = np.stack([b, -b], axis=1).reshape(-1)
    return rows.astype(np.int64), cols.astype(np.int64), vals.astype(np.float64)


def ybus_triplets(g: Grid):
    """Complex Ybus pi-model stamps (no taps): Ys = 1/(r + jx), Bc/2 at each end."""
    ys = 1.0 / (g.r + 1j * g.x)
    half = 0.5j * g.shunt_b
    yff = ys + half
    ytt = ys + half
    rows = np.stack([g.frm, g.frm, g.to, g.to], axis=1).reshape(-1)
    cols = np.stack([g.frm, g.to, g.frm, g.to], axis=1).reshape(-1)
    vals = np.stack([yff, -ys, -ys, ytt], axis=1).reshape(-1)
    return rows.astype(np.int64), cols.astype(np.int64), vals.astype(np.complex128)
