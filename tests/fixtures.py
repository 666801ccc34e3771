"""Deterministic test matrices and right-hand sides, restating the fixtures of ybus's GPU tests
(ybus_cuda/tests/common/mod.rs:20-90, ybus_cuda/tests/gpu_pairs_test.rs:72-106) so the parity
tests here run the reference's own cases: the same LCG, the same matrices, the same seeds.
"""
from __future__ import annotations

import numpy as np

from ybus_b200 import host

MASK = (1 << 64) - 1


class Lcg:
    """`x <- x * 6364136223846793005 + 1442695040888963407 (mod 2^64)`, output `x >> 33`."""

    def __init__(self, seed: int):
        self.state = seed & MASK

    def next(self) -> int:
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & MASK
        return self.state >> 33

    def value(self) -> float:
        return (self.next() % 2001) / 1000.0 - 1.0


def random_spd_triplets(n: int, fill_percent: int, seed: int):
    """A pseudo-random symmetric, diagonally dominant matrix with a positive diagonal."""
    rng = Lcg(seed)
    rows, cols, vals = [], [], []
    row_sums = [0.0] * n
    for i in range(n):
        for j in range(i):
            if rng.next() % 100 < fill_percent:
                value = -((rng.next() % 1000) + 1.0) / 997.0
                rows += [i, j]
                cols += [j, i]
                vals += [value, value]
                row_sums[i] -= value
                row_sums[j] -= value
    for i, s in enumerate(row_sums):
        rows.append(i)
        cols.append(i)
        vals.append(s + 1.0 + i / n)
    return rows, cols, vals


def random_spd(n: int, fill_percent: int, seed: int) -> host.Matrix:
    r, c, v = random_spd_triplets(n, fill_percent, seed)
    return host.Matrix.from_triplets(n, n, r, c, v, by_rows=True)


def star_spd(n: int) -> host.Matrix:
    """A diagonally dominant star: row 0 coupled to every other row, no other couplings."""
    r, c, v = [], [], []
    hub = 1.0
    for i in range(1, n):
        w = -(1.0 + (i % 7) / 7.0)
        r += [0, i, i]
        c += [i, 0, i]
        v += [w, w, 2.0 - w]
        hub -= w
    r.append(0), c.append(0), v.append(hub)
    return host.Matrix.from_triplets(n, n, r, c, v, by_rows=True)


def random_square(n: int, fill_percent: int, seed: int) -> host.Matrix:
    """A pseudo-random unsymmetric matrix with a small diagonal, so the LU pivots off it (CSC)."""
    rng = Lcg(seed)
    rows, cols, vals = [], [], []
    for i in range(n):
        for j in range(n):
            if i != j and rng.next() % 100 < fill_percent:
                rows.append(i)
                cols.append(j)
                vals.append(3.0 * rng.value())
        rows.append(i)
        cols.append(i)
        vals.append(0.1 + abs(rng.value()))
    return host.Matrix.from_triplets(n, n, rows, cols, vals, by_rows=False)


def two_by_two_blocks(blocks: int) -> host.Matrix:
    """2x2 blocks along a chain coupled to their neighbours, as a Jacobian's (CSC)."""
    t = []
    for b in range(blocks):
        p, q = 2 * b, 2 * b + 1
        t += [(p, p, 4.0), (p, q, 1.0), (q, p, -0.5), (q, q, 3.0)]
        if b + 1 < blocks:
            r, s = p + 2, q + 2
            t += [(p, r, -1.0), (r, p, -1.0), (q, s, -0.7), (s, q, -0.8)]
    r, c, v = zip(*t)
    return host.Matrix.from_triplets(2 * blocks, 2 * blocks, r, c, v, by_rows=False)


def right_hand_sides(n: int, count: int, seed: int) -> np.ndarray:
    rng = Lcg(seed)
    return np.array([[rng.value() for _ in range(n)] for _ in range(count)], dtype=np.float64).reshape(count, n)


def pairs(n: int, count: int, seed: int):
    """(plus, minus) unknowns or None (ybus_cuda/tests/gpu_pairs_test.rs:72-84)."""
    rng = Lcg(seed)
    out = []
    for k in range(count):
        plus = rng.next() % n if k % 5 != 3 else None
        minus = rng.next() % n if k % 7 != 2 else None
        if minus is not None and minus == plus:
            minus = None
        out.append((plus, minus))
    return out


def operator_matrix(rows: int, n: int, seed: int) -> host.Matrix:
    """A random rows x n operator, 3 entries per row (gpu_pairs_test.rs:87-97), CSR."""
    rng = Lcg(seed)
    r, c, v = [], [], []
    for i in range(rows):
        for _ in range(3):
            r.append(i)
            c.append(rng.next() % n)
            v.append(rng.value())
    return host.Matrix.from_triplets(rows, n, r, c, v, by_rows=True)


def worst_relative_difference(gpu: np.ndarray, cpu: np.ndarray) -> float:
    """Largest |gpu − cpu| per solution relative to the CPU solution's largest entry
    (ybus_cuda/tests/common/mod.rs:92-109)."""
    worst = 0.0
    for g, c in zip(gpu, cpu):
        scale = max(float(np.abs(c).max()) if c.size else 0.0, np.finfo(float).tiny)
        worst = max(worst, float(np.abs(g - c).max()) / scale if c.size else 0.0)
    return worst
