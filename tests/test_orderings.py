"""The host factor producer's orderings and symbolic analysis against the reference's own
known-answer tests, restated (CPU only):

- COLAMD (ybus_sparse/tests/colamd_test.rs:75-121): a valid column permutation for square and
  rectangular patterns, the same from either orientation and on every call; with empty columns, a
  dense row and a dense column, the dense column ordered last; an empty matrix and one with no
  entries; AMD refusing a rectangular matrix.
- The Cholesky analysis (ybus_sparse/tests/factorization_test.rs:233-270): for the reference's
  random SPD matrices, the elimination tree is each column's first row below it in the
  brute-force elimination's filled pattern, and L's pattern is that filled pattern."""
import numpy as np
import pytest

from fixtures import Lcg, random_spd
from ybus_b200 import host
from ybus_b200._lib import YbError


def random_pattern(m, n, per_row, seed):
    """colamd_test.rs:25-35: about per_row entries per row at random columns, with values."""
    rng = Lcg(seed)
    r, c, v = [], [], []
    for row in range(m):
        for _ in range(per_row):
            col = rng.next() % n
            r.append(row), c.append(col), v.append(((rng.next() % 2001) - 1000.0) / 317.0)
    return np.array(r, np.int64), np.array(c, np.int64), np.array(v)


def is_permutation(perm, n) -> bool:
    return perm.size == n and np.array_equal(np.sort(perm), np.arange(n))


@pytest.mark.parametrize("m,n,per_row,seed", [(80, 30, 4, 2), (30, 80, 6, 3), (200, 200, 2, 4)])
def test_colamd_is_a_permutation_the_same_either_way(m, n, per_row, seed):
    r, c, v = random_pattern(m, n, per_row, seed)
    csr = host.Matrix.from_triplets(m, n, r, c, v, by_rows=True)
    csc = host.Matrix.from_triplets(m, n, r, c, v, by_rows=False)
    perm = csr.ordering(host.COLAMD)
    assert is_permutation(perm, n)
    assert np.array_equal(csc.ordering(host.COLAMD), perm)
    assert np.array_equal(csr.ordering(host.COLAMD), perm)


def test_colamd_orders_the_dense_column_last():
    # the diagonal without every tenth entry, a dense row (5), a dense column (7), the superdiagonal
    n = 300
    r = [i for i in range(n) if i % 10 != 3] + [5] * n + list(range(n)) + list(range(n - 1))
    c = [i for i in range(n) if i % 10 != 3] + list(range(n)) + [7] * n + list(range(1, n))
    v = [1.0] * (len(r) - (n - 1)) + [2.0] * (n - 1)
    a = host.Matrix.from_triplets(n, n, r, c, v, by_rows=False)
    perm = a.ordering(host.COLAMD)
    assert is_permutation(perm, n)
    assert perm[-1] == 7, "the dense column is ordered last"


def test_colamd_of_empty_shapes_and_amd_needs_a_square_matrix():
    empty = host.Matrix.from_triplets(0, 0, [], [], [], by_rows=False)
    assert empty.ordering(host.COLAMD).size == 0
    none = host.Matrix.from_triplets(4, 3, [], [], [], by_rows=False)
    assert is_permutation(none.ordering(host.COLAMD), 3)
    with pytest.raises(YbError):
        none.ordering(host.AMD)


def _filled(dense_pattern):
    """The brute-force elimination's pattern of L (factorization_test.rs:233-243)."""
    n = dense_pattern.shape[0]
    filled = np.tril(dense_pattern).astype(bool)
    for k in range(n):
        below = [i for i in range(k + 1, n) if filled[i, k]]
        for a, i in enumerate(below):
            for j in below[: a + 1]:
                filled[i, j] = True
    return filled


@pytest.mark.parametrize("n,fill,seed", [(1, 0, 1), (12, 20, 2), (40, 8, 3), (60, 4, 4), (30, 50, 5)])
@pytest.mark.parametrize("ordering", [host.NATURAL, host.AMD])
def test_cholesky_analysis_matches_brute_force_elimination(n, fill, seed, ordering):
    a = random_spd(n, fill, seed)
    chol = host.cholesky(a, ordering)
    perm = chol.perm
    assert is_permutation(perm, n)
    assert np.array_equal(perm, a.ordering(ordering))
    dense = a.to_dense() != 0.0
    filled = _filled(dense[np.ix_(perm, perm)])
    # the parent of j is the first row below j with an entry in column j (-1: a root)
    parent = np.array([next((i for i in range(j + 1, n) if filled[i, j]), -1) for j in range(n)])
    assert np.array_equal(chol.parent, parent), (n, ordering)
    # L's pattern (CSR, diagonal last per row) is the filled pattern
    pattern = np.zeros((n, n), bool)
    for i in range(n):
        pattern[i, chol.l.idx[chol.l.ptr[i]:chol.l.ptr[i + 1]]] = True
    assert np.array_equal(pattern, filled)
    counts = filled.sum(axis=0)  # column counts, diagonal included
    assert counts.sum() == chol.l.idx.size
