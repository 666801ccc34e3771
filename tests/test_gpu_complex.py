"""Complex Ybus LU factors on the GPU (no ybus counterpart on the device; the oracle restates
ybus_sparse's generic complex LU solve, lu.rs:770-785): one network and a batch of networks of
uneven orders and right-hand-side counts in one launch, complex128 against the oracle at 1e-12,
complex64 with complex128 refinement to a 1e-10 relative residual."""
import numpy as np
import pytest

import oracle.oracle as orc
from fixtures import worst_relative_difference
from ybus_b200 import FP32, FP64, GpuFactor, grids, host, solve_batch_complex

pytestmark = pytest.mark.gpu


def ybus_factor(n_bus, seed):
    g = grids.make_complex_grid(n_bus, seed)
    r, c, v = grids.ybus_triplets(g)
    a = host.Matrix.from_triplets(n_bus, n_bus, r, c, v, by_rows=False)
    return a, host.lu(a, host.COLAMD)


def rhs(n, count, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((count, n)) + 1j * rng.standard_normal((count, n))


def run_batch(gpu, sizes, counts, precision, seed=1):
    import torch
    nets, bs, xs, ratios, factors = [], [], [], [], []
    for i, (n_bus, count) in enumerate(zip(sizes, counts)):
        a, lu = ybus_factor(n_bus, grids.SEED_BASE + 50 + i + seed)
        f = GpuFactor.from_lu_complex(gpu, lu)
        f.attach_matrix_complex(a)
        b = rhs(n_bus, count, seed + i)
        nets.append((a, lu, b))
        factors.append(f)
        bs.append(torch.from_numpy(b.view(np.float64).copy()).cuda())
        xs.append(torch.empty_like(bs[-1]))
        ratios.append(torch.empty(max(count, 1), dtype=torch.float64, device="cuda"))
    steps = solve_batch_complex(factors, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], counts, precision,
                                d_ratio=[r.data_ptr() for r in ratios])
    gpu.synchronize()
    out = []
    for (a, lu, b), x, r, count in zip(nets, xs, ratios, counts):
        sol = x.cpu().numpy().view(np.complex128).reshape(count, -1)
        out.append((a, lu, b, sol, r.cpu().numpy()[:count]))
    return out, steps


def test_one_complex_network_matches_the_oracle(gpu):
    out, _ = run_batch(gpu, [300], [16], FP64)
    a, lu, b, sol, ratio = out[0]
    cpu = orc.solve_many_lu(lu, b)
    assert worst_relative_difference(sol, cpu) < 1e-12
    assert ratio.max() < 1e-12


def test_a_batch_of_uneven_networks_in_complex128(gpu):
    out, _ = run_batch(gpu, [200, 1500, 600, 3000], [1, 5, 16, 33], FP64, seed=2)
    for a, lu, b, sol, ratio in out:
        assert worst_relative_difference(sol, orc.solve_many_lu(lu, b)) < 1e-12
        assert ratio.max() < 1e-12


def test_a_batch_in_complex64_with_refinement(gpu):
    out, steps = run_batch(gpu, [200, 1500, 600, 3000], [3, 7, 16, 20], FP32, seed=3)
    assert 1 <= steps[0] <= 3
    for a, lu, b, sol, ratio in out:
        assert ratio.max() <= 1e-10
        assert worst_relative_difference(sol, orc.solve_many_lu(lu, b)) < 1e-8
