"""The oracle pinned against the reference's own known-answer tests and fixtures, and the host
factor producer checked against it (CPU only)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle.oracle as orc
from fixtures import (Lcg, pairs, random_spd, random_spd_triplets, random_square, right_hand_sides,
                      two_by_two_blocks, worst_relative_difference)
from ybus_b200 import host


def test_lcg_matches_the_reference_generator():
    # x <- x * 6364136223846793005 + 1442695040888963407 mod 2^64, output x >> 33
    rng = Lcg(7)
    x = 7
    for _ in range(5):
        x = (x * 6364136223846793005 + 1442695040888963407) % 2**64
        assert rng.next() == x >> 33
    assert -1.0 <= Lcg(3).value() <= 1.0


def test_single_row_solves_bit_for_bit():
    # ybus_cuda/tests/gpu_factor_test.rs:74-86: A = [3] by LU, b = j - 70.5
    one = host.lu(host.Matrix.from_triplets(1, 1, [0], [0], [3.0], by_rows=False))
    assert one.l.val.tolist() == [1.0] and one.u.val.tolist() == [3.0]
    b = np.array([[j - 70.5] for j in range(200)])
    x = orc.solve_many_lu(one, b)
    assert np.array_equal(x[:, 0], b[:, 0] / 3.0)


def test_single_row_pair_known_answer():
    # ybus_cuda/tests/gpu_pairs_test.rs:265-280: A = [4], pair (0, None) -> 0.25
    one = host.lu(host.Matrix.from_triplets(1, 1, [0], [0], [4.0], by_rows=False))
    assert orc.solve_many_lu(one, np.array([[1.0]]))[0, 0] == 0.25


def test_singular_update_known_answer():
    # gpu_pairs_test.rs:168-185: an empty pair with a zero weight is singular and gives x
    base = np.linspace(-1, 1, 7)
    y = np.zeros(7)
    out, singular = orc.pair_update(base, y, None, None, 0.5, 0.0)
    assert singular
    assert np.array_equal(out, base)
    out, singular = orc.pair_update(base, np.ones(7), 2, 5, 0.25, 3.0)
    assert not singular


def test_column_max_tie_rule():
    # kernels.cu:78-128: smallest row on a tie, None when every product is zero, non-finite flagged
    row, value, bad = orc.column_max(np.array([0.0, -2.0, 1.0, 2.0]))
    assert (row, value, bad) == (1, 2.0, False)
    row, value, bad = orc.column_max(np.zeros(5))
    assert (row, value, bad) == (None, 0.0, False)
    row, value, bad = orc.column_max(np.array([1.0, np.nan, -3.0, np.inf]), np.array([1.0, 1.0, 0.5, 1.0]))
    assert (row, value, bad) == (2, 1.5, True)


@pytest.mark.parametrize("n,fill,seed", [(300, 3, 7), (500, 2, 13), (10, 20, 1), (200, 3, 21)])
def test_cholesky_factor_reconstructs(n, fill, seed):
    a = random_spd(n, fill, seed)
    chol = host.cholesky(a)
    assert sorted(chol.perm.tolist()) == list(range(n))
    assert orc.cholesky_reconstruction_error(chol, a.to_dense()) < 1e-13
    # each row of L ends with its diagonal, each row of Lᵀ starts with it
    for i in range(n):
        assert chol.l.idx[chol.l.ptr[i + 1] - 1] == i
        assert chol.lt.idx[chol.lt.ptr[i]] == i


def test_amd_reduces_fill():
    a = random_spd(300, 3, 7)
    amd = host.cholesky(a, host.AMD)
    natural = host.cholesky(a, host.NATURAL)
    assert amd.l.idx.size < natural.l.idx.size


@pytest.mark.parametrize("build", [lambda: random_square(250, 4, 3), lambda: random_square(150, 4, 22),
                                   lambda: two_by_two_blocks(40)])
def test_lu_factor_reconstructs(build):
    a = build()
    f = host.lu(a)
    assert orc.lu_reconstruction_error(f, a.to_dense()) < 1e-12


def test_lu_fixture_pivots_off_the_diagonal():
    # gpu_factor_test.rs:42-47: the fixture must pivot
    f = host.lu(random_square(250, 4, 3))
    assert any(i != p for i, p in enumerate(f.row_perm))


def test_colamd_lu_reconstructs():
    a = random_square(120, 5, 9)
    f = host.lu(a, host.COLAMD)
    assert sorted(f.col_perm.tolist()) == list(range(120))
    assert orc.lu_reconstruction_error(f, a.to_dense()) < 1e-12


def test_complex_lu_reconstructs_and_solves():
    rng = np.random.default_rng(5)
    n = 80
    r, c, v = random_spd_triplets(n, 5, 3)
    v = np.array(v) * (1 + 0.3j)
    a = host.Matrix.from_triplets(n, n, r, c, v, by_rows=False)
    f = host.lu(a, host.COLAMD)
    assert f.is_complex
    assert orc.lu_reconstruction_error(f, a.to_dense()) < 1e-12
    b = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    x = orc.solve_many_lu(f, b)
    dense = a.to_dense()
    for k in range(3):
        assert np.abs(dense @ x[k] - b[k]).max() < 1e-11 * np.abs(b[k]).max()


def _scipy_csr(a: host.Matrix):
    rows, cols, _, by_rows, _ = a.info()
    p, i, v = a.arrays()
    return (sp.csr_matrix((v, i, p), shape=(rows, cols)) if by_rows else sp.csc_matrix((v, i, p), shape=(rows, cols)))


def test_oracle_solves_match_scipy():
    a = random_spd(300, 3, 7)
    chol = host.cholesky(a)
    b = right_hand_sides(300, 37, 11)
    x = orc.solve_many(chol, b)
    ref = spla.spsolve(_scipy_csr(a).tocsc(), b.T).T
    assert worst_relative_difference(x, ref) < 1e-12
    sq = random_square(250, 4, 3)
    f = host.lu(sq)
    b2 = right_hand_sides(250, 20, 5)
    x2 = orc.solve_many(f, b2)
    ref2 = spla.spsolve(_scipy_csr(sq).tocsc(), b2.T).T
    assert worst_relative_difference(x2, ref2) < 1e-11
    xt = orc.solve_many_lu(f, b2, transpose=True)
    ref_t = spla.spsolve(_scipy_csr(sq).T.tocsc(), b2.T).T
    assert worst_relative_difference(xt, ref_t) < 1e-11


def test_par_solve_many_is_bit_identical_to_serial():
    chol = host.cholesky(random_spd(500, 2, 13))
    b = right_hand_sides(500, 50, 17)
    one = orc.solve_many(chol, b, threads=1)
    four = orc.solve_many(chol, b, threads=4)
    assert np.array_equal(one.view(np.uint64), four.view(np.uint64))


def _ring():
    """The ring of ybus's DC tests (ybus_powerflow/tests/dc_outage_test.rs:103-126), in-service
    branches only, buses 1-4 and 6 renumbered 0-4 (bus 1 the reference): a ring with a chord,
    a parallel pair, a tapped branch and a pendant bus (a bridge)."""
    # (from, to, x, tap)
    branches = [(0, 1, 0.1, 0.0), (0, 1, 0.3, 0.0), (1, 2, 0.2, 0.0), (2, 3, 0.15, 1.05), (3, 0, 0.25, 0.0),
                (0, 2, 0.4, 0.0), (3, 4, 0.2, 0.0)]
    frm = np.array([b[0] for b in branches])
    to = np.array([b[1] for b in branches])
    b = np.array([1.0 / (x * (tap if tap else 1.0)) for _, _, x, tap in branches])
    return 5, frm, to, b


def _bprime(nbus, frm, to, b, keep):
    rows = np.concatenate([frm, frm, to, to])
    cols = np.concatenate([frm, to, frm, to])
    vals = np.concatenate([b, -b, -b, b])
    # ybus's stamp order: per branch (f,f), (f,t), (t,f), (t,t)
    order = np.stack([frm, frm, to, to], 1).reshape(-1), np.stack([frm, to, frm, to], 1).reshape(-1)
    v = np.stack([b, -b, -b, b], 1).reshape(-1)
    m = host.Matrix.from_triplets(nbus, nbus, order[0], order[1], v, by_rows=True)
    return m.select(keep, keep)


def test_smw_outage_matches_refactoring_on_the_ring():
    # dc_outage_test.rs:38-59: the rank-k update agrees with refactoring to 1e-9
    nbus, frm, to, b = _ring()
    keep = np.arange(1, nbus)
    position = np.full(nbus, -1)
    position[keep] = np.arange(keep.size)
    p = np.array([0.0, -0.4, 0.2 - 0.3, -0.5, -0.15])[keep]  # Pd/100 with bus 3's 20 MW generator
    bp = _bprime(nbus, frm, to, b, keep)
    chol = host.cholesky(bp)
    base = orc.solve_many(chol, p[None, :])[0]
    bridges = orc.bridges(nbus, frm, to)
    assert bridges.tolist() == [False, False, False, False, False, False, True]
    for k in range(frm.size):
        if bridges[k]:
            continue
        theta = orc.outage_flows_smw(lambda c: orc.solve_many(chol, c[None, :])[0], keep.size, position, frm, to, b,
                                     [k], base)
        keep_br = np.array([j for j in range(frm.size) if j != k])
        re = host.cholesky(_bprime(nbus, frm[keep_br], to[keep_br], b[keep_br], keep))
        expected = orc.solve_many(re, p[None, :])[0]
        assert np.abs(theta - expected).max() <= 1e-9 * max(1.0, np.abs(expected).max())
    # and two at a time (rank 2)
    theta = orc.outage_flows_smw(lambda c: orc.solve_many(chol, c[None, :])[0], keep.size, position, frm, to, b,
                                 [0, 5], base)
    keep_br = np.array([1, 2, 3, 4, 6])
    expected = orc.solve_many(host.cholesky(_bprime(nbus, frm[keep_br], to[keep_br], b[keep_br], keep)),
                              p[None, :])[0]
    assert np.abs(theta - expected).max() <= 1e-9 * max(1.0, np.abs(expected).max())
