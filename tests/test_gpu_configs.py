"""Parity at the sizes of the solve path's five configurations (the seeded workloads of
ybus_b200/configs.py, the same inputs the bench times), each through the C ABI against the oracle:

1. 2,000 buses, 256 unit right-hand sides, FP64: host-array and device-array solves within 1e-12
   of the oracle's `par_solve_many` (the reference's bar, ybus_cuda/tests/gpu_factor_test.rs:16).
3. 10,000 buses, 2,000 non-bridge outages with U[1, 64] injection scenarios each (65,046), in one
   captured launch in FP64 and with FP32 substitution and FP64 refinement: a seeded sample of 200
   cases against the oracle's rank-one SMW outage (ybus_powerflow/src/dc/outage.rs:126-241) and
   column maxima (ybus_cuda/src/kernels.cu:78-128).
4. 10,000 buses, 1,024 scenarios, the flow loss's gradients with respect to the injections and the
   branch susceptances against the CPU's transposed-solve gradient, and against FP64 central
   differences (h = 1e-6) at 200 seeded coordinates, each within 1e-6 of its own value (bridges'
   susceptances, whose gradient is zero to rounding, are checked to be zero instead).
5. The 16-network complex batch (500 to 70,000 buses, 128 right-hand sides each) in complex128
   against the oracle's complex LU solve (ybus_sparse/src/compressed_matrix/lu.rs:770-785) and in
   complex64 with complex128 refinement to a 1e-10 relative residual; and a network at the top of
   the range, 70,000 buses.

Configuration 2 (the 13,499-column PTDF block) is checked in test_gpu_factor.py."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle.oracle as orc
from dc_cases import cpu_model, oracle_screening
from fixtures import worst_relative_difference
from ybus_b200 import FP32, FP64, GpuFactor, configs, host, solve_batch_complex
from ybus_b200.dc import DcNetwork, FlowLoss

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps
# The complex128 solutions must match the oracle's to 1e-12; their relative residual
# |b - Ax|inf / |b|inf is set by the COLAMD LU factor's growth and conditioning (2.1e-12 on the
# worst network of the batch, whose solutions match the oracle's to 1e-12), so it gets a bound of
# its own.
RESIDUAL_C128 = 1e-11


def test_c1_unit_right_hand_sides_on_the_2k_grid(gpu):
    import torch
    g, rhs = configs.unit_rhs_2k()
    assert rhs.shape == (256, 1999) and (rhs.sum(axis=1) == 1.0).all()
    chol = host.cholesky(configs.bprime(g))
    factor = GpuFactor.from_cholesky(gpu, chol)
    cpu = orc.solve_many(chol, rhs, threads=8)
    host_x = factor.solve_many(rhs)
    assert worst_relative_difference(host_x, cpu) < 1e-12
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, None)
    gpu.synchronize()
    factor.check_error()
    assert worst_relative_difference(x.cpu().numpy(), cpu) < 1e-12
    assert np.array_equal(x.cpu().numpy(), host_x)  # the same kernels either way


@pytest.fixture(scope="module")
def grid10k():
    g = configs.grid_10k()
    _, chol, position = cpu_model(g)
    return g, chol, position


@pytest.mark.parametrize("precision,bar", [(FP64, 1e-10), (FP32, 1e-8)], ids=["fp64", "fp32_ir"])
def test_c3_n1_screening_of_2000_outages(gpu, grid10k, precision, bar):
    g, chol, position = grid10k
    net = DcNetwork.from_grid(gpu, g)
    cases = configs.n1_cases(g, net.bridges())
    sp = cases.scenario_ptr
    assert cases.outaged.size == 2000 and np.unique(cases.outaged).size == 2000
    counts = np.diff(sp)
    assert counts.min() >= 1 and counts.max() <= 64
    rows, values, bad, sing = net.outage_loadings_batch(cases.outaged, sp, cases.injections, cases.weights, precision)
    assert not bad.any() and not sing.any()
    if precision == FP64:  # the graph replays: the same bits
        again = net.outage_loadings_batch(cases.outaged, sp, cases.injections, cases.weights, precision)
        assert np.array_equal(again[0], rows) and np.array_equal(again[1], values)
    pick = np.sort(np.random.default_rng(7).choice(cases.outaged.size, 200, replace=False))
    cols = np.concatenate([np.arange(sp[c], sp[c + 1]) for c in pick])
    sub_sp = np.concatenate([[0], np.cumsum(counts[pick])])
    er, ev = oracle_screening(g, chol, position, cases.outaged[pick], sub_sp, cases.injections[cols], cases.weights)
    gv, gr = values[cols], rows[cols]
    assert np.abs(gv - ev).max() <= bar * np.abs(ev).max()
    # the same branch unless two loadings tie to within the bar
    for j in np.flatnonzero(gr != er):
        assert abs(gv[j] - ev[j]) <= bar * ev[j]
    assert np.count_nonzero(gr != er) <= 2


def _central_difference(f_minus, df, limits, step, margin=0.8):
    """(L(+) - L(-)) / 2 step for flows f_minus at the lower point and f_minus + df at the upper,
    the loss sum softplus(|f| - margin limit)^2 differenced term by term without cancellation:
    with u = |f| - margin limit and du = |f+| - |f-| (df times the flow's sign where both points
    share it), softplus(u + du) - softplus(u) = log1p(expm1(du) sigmoid(u)) and a term's change is
    ds (2 s + ds). Returns the quotient and an estimate of its error: 8 eps of the sum of the
    terms' absolute changes, plus every term whose flow changes sign between the two points (the
    kink of |f|, where a difference quotient is no derivative), over 2 step."""
    neg = np.signbit(f_minus)
    f_plus = f_minus + df
    kink = np.signbit(f_plus) != neg
    du = np.negative(df, where=neg, out=df.copy())
    du[kink] = np.abs(f_plus[kink]) - np.abs(f_minus[kink])
    u = np.abs(f_minus)
    u -= margin * limits
    e = np.exp(-np.abs(u))
    s = np.log1p(e)
    s += np.maximum(u, 0.0)
    sig = np.where(u >= 0, 1.0, e)
    sig /= 1.0 + e
    ds = np.expm1(du)
    ds *= sig
    np.log1p(ds, out=ds)
    dt = 2.0 * s
    dt += ds
    dt *= ds
    fd = dt.sum() / (2 * step)
    noise = (8 * EPS * np.abs(dt).sum() + np.abs(dt[kink]).sum()) / (2 * step)
    return fd, noise


def test_c4_adjoint_gradients_at_1024_scenarios(gpu, grid10k):
    g, chol, position = grid10k
    p, limits = configs.adjoint_scenarios(g)
    net = DcNetwork.from_grid(gpu, g)
    loss_fn = FlowLoss(net, p.shape[0])
    loss, flows = loss_fn.forward(p, limits, flows=True)
    gp, gb = loss_fn.backward()
    # against the CPU's gradient from the oracle's solve and transposed solve
    loss_c, gp_c, gb_c = orc.flow_loss_and_gradient(chol, g.n_bus, g.frm, g.to, g.susceptance, position, p, limits)
    assert abs(loss - loss_c) <= 1e-12 * abs(loss_c)
    assert np.abs(gp - gp_c).max() <= 1e-10 * np.abs(gp_c).max()
    assert np.abs(gb - gb_c).max() <= 1e-10 * np.abs(gb_c).max()
    assert (gp[:, 0] == 0.0).all()
    # a bridge's flow is its side's injection whatever its susceptance: dL/db is zero to rounding
    bridge = orc.bridges(g.n_bus, g.frm, g.to)
    assert np.abs(gb[bridge]).max() <= 1e-12 * np.abs(gb).max()

    # central differences at 200 seeded coordinates: 150 of dL/dp, 50 of dL/db over the branches
    # that are not bridges. Both points' flows are evaluated in FP64 from the oracle's solves, their
    # difference without cancellation: for p_ri, theta_r -+ h y with y = B'^-1 e_i; for b_k (step h
    # b_k), B' -+ step a a' (a = e_f - e_t) by the rank-one update of the kept factor's solutions,
    # theta(s) = theta - y (a'theta) s / (1 + s a'y), so theta(+) - theta(-) = -y (a'theta) 2 step /
    # (1 - step^2 (a'y)^2), and over the branches the angle differences move along dy = A y
    h = 1e-6
    unknown = position >= 0
    theta = orc.solve_many(chol, p[:, unknown], threads=8)

    def angles(th):  # (.., n_bus) with the slack at 0
        out = np.zeros(th.shape[:-1] + (g.n_bus,))
        out[..., unknown] = th[..., position[unknown]]
        return out

    b = g.susceptance
    tb = angles(theta)
    rng = np.random.default_rng(44)
    results = []  # (fd, gradient, noise)
    for _ in range(150):
        r, i = int(rng.integers(p.shape[0])), int(rng.integers(1, g.n_bus))
        e = np.zeros(chol.n)
        e[position[i]] = 1.0
        y = angles(orc.solve_many(chol, e[None, :])[0])
        t_m = tb[r] - h * y
        f_m = b * t_m[g.frm] + (-b) * t_m[g.to]
        df = b * (2 * h * y[g.frm]) + (-b) * (2 * h * y[g.to])
        fd, noise = _central_difference(f_m, df, limits, h)
        results.append((fd, gp[r, i], noise))
    d = tb[:, g.frm] - tb[:, g.to]  # every scenario's angle differences over the branches

    def susceptance_difference(k):
        step = h * b[k]
        a = np.zeros(chol.n)
        if unknown[g.frm[k]]:
            a[position[g.frm[k]]] += 1.0
        if unknown[g.to[k]]:
            a[position[g.to[k]]] -= 1.0
        y = angles(orc.solve_many(chol, a[None, :])[0])
        dy = y[g.frm] - y[g.to]
        at, ay = d[:, k], dy[k]  # a'theta and a'y
        d_m = d + np.outer(at * step / (1.0 - step * ay), dy)
        dd = np.outer(-at * (2 * step) / (1.0 - step * step * ay * ay), dy)
        bm = b.copy()
        bm[k] -= step
        f_m = bm * d_m
        df = b * dd
        df[:, k] = b[k] * dd[:, k] + step * (2 * d_m[:, k] + dd[:, k])  # (b+s)(d+dd) - (b-s)d
        return _central_difference(f_m, df, limits, step)

    ks = rng.choice(np.flatnonzero(~bridge), 50, replace=False)
    with ThreadPoolExecutor(8) as pool:  # numpy's array operations release the interpreter lock
        for k, (fd, noise) in zip(ks, pool.map(susceptance_difference, ks)):
            results.append((fd, gb[k], noise))
    res = np.array(results)
    fd, grad, noise = res[:, 0], res[:, 1], res[:, 2]
    # a coordinate is measurable when the difference quotient's error estimate is below 1e-7 of
    # the gradient's value; those must agree to 1e-6 relative, the rest to their estimate
    measurable = noise <= 1e-7 * np.abs(grad)
    assert measurable.mean() >= 0.95, f"{(~measurable).sum()} of 200 coordinates below the difference's resolution"
    rel = np.abs(fd - grad) / np.abs(grad)
    assert rel[measurable].max() <= 1e-6, rel[measurable].max()
    assert (np.abs(fd - grad) <= 1e-6 * np.abs(grad) + 10 * noise).all()


@pytest.fixture(scope="module")
def complex_batch():
    return [configs.complex_network(n, i) for i, n in enumerate(configs.complex_sizes())]


def _run_complex(gpu, nets, precision):
    import torch
    factors, bs, xs, rs = [], [], [], []
    for net in nets:
        f = GpuFactor.from_lu_complex(gpu, net.lu)
        f.attach_matrix_complex(net.ybus)
        factors.append(f)
        bs.append(torch.from_numpy(net.rhs.view(np.float64).copy()).cuda())
        xs.append(torch.empty_like(bs[-1]))
        rs.append(torch.empty(net.rhs.shape[0], dtype=torch.float64, device="cuda"))
    steps = solve_batch_complex(factors, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs],
                                [net.rhs.shape[0] for net in nets], precision, 3, 1e-10, [r.data_ptr() for r in rs])
    gpu.synchronize()
    for f in factors:
        f.check_error()
    sols = [x.cpu().numpy().view(np.complex128).reshape(net.rhs.shape) for x, net in zip(xs, nets)]
    return sols, [r.cpu().numpy() for r in rs], steps


@pytest.mark.parametrize("precision", [FP64, FP32], ids=["c128", "c64_ir"])
def test_c5_complex_batch_of_16_networks(gpu, complex_batch, precision):
    nets = complex_batch
    sizes = [net.n for net in nets]
    assert len(nets) == 16 and min(sizes) >= 500 and max(sizes) <= 70000
    sols, ratios, steps = _run_complex(gpu, nets, precision)
    for net, x, ratio in zip(nets, sols, ratios):
        cpu = orc.solve_many_lu(net.lu, net.rhs, threads=8)
        if precision == FP64:
            assert worst_relative_difference(x, cpu) < 1e-12, net.n
            assert ratio.max() <= RESIDUAL_C128, (net.n, ratio.max())
        else:
            assert ratio.max() <= 1e-10, (net.n, ratio.max())
            assert worst_relative_difference(x, cpu) < 1e-8, net.n
    if precision == FP32:
        assert all(1 <= s <= 3 for s in steps)


@pytest.mark.parametrize("precision", [FP64, FP32], ids=["c128", "c64_ir"])
def test_c5_a_network_at_the_top_of_the_range(gpu, precision):
    net = configs.complex_network(70000, 99, count=128)
    (x,), (ratio,), steps = _run_complex(gpu, [net], precision)
    # the oracle's residuals of the GPU's solutions, and the oracle's own solve
    p, i, v = net.ybus.to_csr().arrays()
    cpu = orc.solve_many_lu(net.lu, net.rhs, threads=8)
    if precision == FP64:
        assert worst_relative_difference(x, cpu) < 1e-12
    else:
        assert ratio.max() <= 1e-10
        assert worst_relative_difference(x, cpu) < 1e-8
    ax = np.stack([_csr_mul(p, i, v, xi) for xi in x[:8]])
    rel = np.abs(net.rhs[:8] - ax).max(axis=1) / np.abs(net.rhs[:8]).max(axis=1)
    assert rel.max() <= (RESIDUAL_C128 if precision == FP64 else 1e-10)


def _csr_mul(p, i, v, x):
    rows = np.repeat(np.arange(p.size - 1), np.diff(p))
    return np.bincount(rows, weights=(v * x[i]).real, minlength=p.size - 1) + \
        1j * np.bincount(rows, weights=(v * x[i]).imag, minlength=p.size - 1)
