"""Blocks built, solved and updated on the device (ybus_cuda/tests/gpu_pairs_test.rs), against
the oracle's CPU solves and the reference kernel's formulas on the host: pair solves and their
maxima, rank-one updates including a singular one, operator products with entries zeroed and
their maxima (the tie rule), and a single-row factor. The LU fixtures pivot, so right-hand-side
and solution orders differ. All calls go through the C ABI."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import Lcg, operator_matrix, pairs, random_spd, random_square
from ybus_b200 import ColumnMax, GpuFactor, Pair, PairUpdate, host

pytestmark = pytest.mark.gpu

BAR = 1e-12


def factors(n):
    return [("cholesky", host.cholesky(random_spd(n, 3, 21))), ("lu", host.lu(random_square(n, 4, 22)))]


def upload(gpu, f):
    return GpuFactor.from_cholesky(gpu, f) if isinstance(f, host.HostCholesky) else GpuFactor.from_lu(gpu, f)


def pair_vector(n, pair):
    c = np.zeros(n)
    if pair.plus is not None:
        c[pair.plus] = 1.0
    if pair.minus is not None:
        c[pair.minus] = -1.0
    return c


def max_difference(a, b):
    scale = max(1.0, float(np.abs(b).max()))
    return float(np.abs(a - b).max()) / scale


def host_update(f, base, update):
    """The update PairUpdate describes, on the host from the CPU's solve (gpu_pairs_test.rs:48-62)."""
    y = orc.solve_many(f, pair_vector(base.size, update.pair)[None, :])[0]
    p, m = update.pair.plus, update.pair.minus
    return orc.pair_update(base, y, p, m, update.alpha, update.inverse_weight)


def to_pairs(raw):
    return [Pair(p, m) for p, m in raw]


@pytest.mark.parametrize("name", ["cholesky", "lu"])
def test_pair_solves_and_their_maxima_match_the_host(gpu, name):
    n = 200
    f = dict(factors(n))[name]
    factor = upload(gpu, f)
    factor.set_block_width(32)
    ps = to_pairs(pairs(n, 29, 5))
    block = factor.pair_solves(ps)
    assert block.columns() == 29
    assert not any(block.singular())
    solutions = block.solutions()
    maxima = block.maxima()
    expected = orc.solve_many(f, np.array([pair_vector(n, p) for p in ps]))
    for pair, sol, mx, e in zip(ps, solutions, maxima, expected):
        assert max_difference(sol, e) < BAR
        largest = float(np.abs(e).max())
        assert abs(mx.value - largest) <= BAR * largest
        if mx.row is not None:
            assert abs(abs(sol[mx.row]) - mx.value) <= BAR * largest
        else:
            assert pair.plus is None and pair.minus is None  # an empty pair's solution is zero
        assert not mx.not_finite


@pytest.mark.parametrize("name", ["cholesky", "lu"])
def test_rank_one_updates_match_the_host_including_a_singular_one(gpu, name):
    n = 150
    rng = Lcg(9)
    base = np.array([rng.value() for _ in range(n)])
    f = dict(factors(n))[name]
    factor = upload(gpu, f)
    factor.set_block_width(16)
    updates = [PairUpdate(p, rng.value(), 2.0 + rng.value()) for p in to_pairs(pairs(n, 15, 6))]
    # an empty pair with a zero weight: w = 0 exactly, so singular
    updates.append(PairUpdate(Pair(None, None), 0.5, 0.0))
    block = factor.pair_updates(base, updates)
    solutions = block.solutions()
    singular = block.singular()
    for k, (u, sol) in enumerate(zip(updates, solutions)):
        expected, sing = host_update(f, base, u)
        assert singular[k] == sing, f"column {k}"
        assert max_difference(sol, expected) < BAR, f"column {k}"
    assert singular[15]
    # Given the GPU's own y, the device's update is the reference kernel's formula bit for bit
    ys = factor.pair_solves([u.pair for u in updates]).solutions()
    for k, (u, y) in enumerate(zip(updates, ys)):
        exact, _ = orc.pair_update(base, y, u.pair.plus, u.pair.minus, u.alpha, u.inverse_weight)
        assert np.array_equal(solutions[k].view(np.uint64), exact.view(np.uint64)), f"column {k}"


@pytest.mark.parametrize("name", ["cholesky", "lu"])
def test_operator_products_and_maxima_match_the_host(gpu, name):
    n, rows = 120, 90
    rng = Lcg(31)
    base = np.array([rng.value() for _ in range(n)])
    offset = np.array([rng.value() for _ in range(rows)])
    weights = np.array([0.0 if i % 4 == 0 else 1.0 + abs(rng.value()) for i in range(rows)])
    m = operator_matrix(rows, n, 32)
    mp, mi, mv = m.arrays()
    f = dict(factors(n))[name]
    factor = upload(gpu, f)
    factor.set_block_width(8)
    op = factor.operator(m)
    op.set_offset(offset)
    op.set_weights(weights)
    updates = [PairUpdate(p, 0.25, 3.0) for p in to_pairs(pairs(n, 7, 33))]
    zero = [k * 11 if k % 2 == 0 else None for k in range(7)]
    block = factor.pair_updates(base, updates)
    products = block.product(op, zero)
    maxima = block.product_maxima(op, zero)
    for k in range(7):
        theta, _ = host_update(f, base, updates[k])
        expected = orc.csr_mul_vec(mp, mi, mv, theta) + offset
        if zero[k] is not None:
            expected[zero[k]] = 0.0
            assert products[k][zero[k]] == 0.0
        assert max_difference(products[k], expected) < BAR, f"column {k}"
        # the host's maximum of |value| * weight over the downloaded products, smallest row on a tie
        row, value = None, 0.0
        for i, (e, w) in enumerate(zip(products[k], weights)):
            if abs(e) * w > value:
                row, value = i, abs(e) * w
        assert maxima[k] == ColumnMax(row, value, False), f"column {k}"
        assert (row, value, False) == orc.column_max(products[k], weights)


def test_column_maxima_flag_values_that_are_not_finite(gpu):
    chol = host.cholesky(random_spd(40, 10, 3))
    factor = GpuFactor.from_cholesky(gpu, chol)
    block = factor.pair_solves([Pair(1, None), Pair(None, None)])
    y = block.solutions()
    # row 0 is inf * theta[1]: inf for the first column (theta[1] > 0), NaN for the empty pair's zero
    op = factor.operator((2, np.array([0, 1, 2]), np.array([1, 2]), np.array([np.inf, 1.0])))
    mx = block.product_maxima(op)
    assert mx[0].not_finite and mx[0].value == abs(y[0][2]) and mx[0].row == (1 if y[0][2] != 0 else None)
    assert mx[1] == ColumnMax(None, 0.0, True)


def test_a_single_row_factor_keeps_its_blocks_narrow(gpu):
    one = host.lu(host.Matrix.from_triplets(1, 1, [0], [0], [4.0], by_rows=False))
    factor = GpuFactor.from_lu(gpu, one)
    factor.set_block_width(1024)
    assert factor.block_width() == 64
    solutions = factor.pair_solves([Pair(0, None)] * 64).solutions()
    assert (solutions == 0.25).all()


def test_contract_violations_are_errors_not_aborts(gpu):
    from ybus_b200 import CudaError
    chol = host.cholesky(random_spd(30, 10, 3))
    factor = GpuFactor.from_cholesky(gpu, chol)
    factor.set_block_width(4)
    with pytest.raises(CudaError):
        factor.pair_solves([Pair(1, None)] * 5)  # more than block_width
    with pytest.raises(CudaError):
        factor.pair_solves([Pair(3, 3)])  # the same unknown twice
    with pytest.raises(CudaError):
        factor.pair_solves([Pair(30, None)])  # past dim()
