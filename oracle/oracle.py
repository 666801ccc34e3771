"""ORACLE — test infrastructure only (tests, the smoke check and the bench's CPU baseline).

Python side of the oracle: loads liboracle.so (the C restatement of ybus's CPU solves in
oracle.c, built by oracle/Makefile) and adds the DC-domain formulas that sit on top of those
solves, each restating the reference function it names:

- `DcStudy::outage` rank-k Sherman–Morrison–Woodbury update (ybus_powerflow/src/dc/outage.rs:126-241)
- PTDF by branch and LODF (ybus_powerflow/src/dc/sensitivity.rs:199-381)
- bridges of a multigraph (ybus_powerflow/src/islands.rs:132-176)

Parity of this oracle is pinned by tests/test_oracle.py against the reference's own known-answer
tests and fixtures; the Rust reference cannot be built in this image.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None

vp, i64, dbl, i32 = C.c_void_p, C.c_int64, C.c_double, C.c_int


def build() -> Path:
    src = HERE / "oracle.c"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        h = C.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL)
        h.or_solve_many.restype = i32
        h.or_solve_many.argtypes = [i32, i64, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, vp, i32]
        h.or_pair_update.restype = i32
        h.or_pair_update.argtypes = [i64, vp, vp, i64, i64, dbl, dbl, vp]
        h.or_column_max.restype = None
        h.or_column_max.argtypes = [i64, vp, vp, C.POINTER(i64), C.POINTER(dbl), C.POINTER(i32)]
        h.or_csr_mul_vec.restype = None
        h.or_csr_mul_vec.argtypes = [i64, vp, vp, vp, vp, vp]
        h.or_relative_residual.restype = dbl
        h.or_relative_residual.argtypes = [i64, vp, vp, vp, vp, vp]
        _lib = h
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def _rhs(b, n, dtype=np.float64):
    b = _c(b, dtype)
    if b.ndim == 1:
        b = b.reshape(1, n)
    return b


def solve_many_cholesky(chol, rhs, threads: int = 1) -> np.ndarray:
    """`Factorization::par_solve_many` with `Cholesky::substitute` (factorization.rs:71-92,
    cholesky.rs:570-579). `chol` has .n, .l, .lt (ptr, idx, val) and .perm; rhs is (count, n)."""
    n = chol.n
    b = _rhs(rhs, n)
    out = np.empty_like(b)
    l, lt = chol.l, chol.lt
    arrs = [_c(l.ptr, np.int64), _c(l.idx, np.int64), _c(l.val, np.float64), _c(lt.ptr, np.int64),
            _c(lt.idx, np.int64), _c(lt.val, np.float64), _c(chol.perm, np.int64)]
    rc = lib().or_solve_many(1, n, *[_p(a) for a in arrs], _p(arrs[-1]), _p(b), b.shape[0], _p(out), threads)
    assert rc == 0
    return out


def _lu_arrays(f, dtype):
    return [_c(f.l.ptr, np.int64), _c(f.l.idx, np.int64), _c(f.l.val, dtype), _c(f.u.ptr, np.int64),
            _c(f.u.idx, np.int64), _c(f.u.val, dtype), _c(f.row_perm, np.int64), _c(f.col_perm, np.int64)]


def solve_many_lu(f, rhs, threads: int = 1, transpose: bool = False) -> np.ndarray:
    """`Lu::substitute` (lu.rs:770-785), or `Lu::solve_transpose` (lu.rs:506-533), per RHS."""
    n = f.n
    if f.is_complex:
        if transpose:
            raise NotImplementedError("complex transposed solve")
        b = _rhs(rhs, n, np.complex128)
        out = np.empty_like(b)
        a = _lu_arrays(f, np.complex128)
        rc = lib().or_solve_many(4, n, *[_p(x) for x in a], _p(b), b.shape[0], _p(out), threads)
    else:
        b = _rhs(rhs, n)
        out = np.empty_like(b)
        a = _lu_arrays(f, np.float64)
        rc = lib().or_solve_many(3 if transpose else 2, n, *[_p(x) for x in a], _p(b), b.shape[0], _p(out), threads)
    assert rc == 0
    return out


def solve_many(f, rhs, threads: int = 1) -> np.ndarray:
    return solve_many_cholesky(f, rhs, threads) if hasattr(f, "lt") else solve_many_lu(f, rhs, threads)


def pair_update(base, y, plus, minus, alpha, inverse_weight):
    """The rank-one update formula of ybus_cuda/src/kernels.cu:24-58 (and the test's host
    re-derivation, ybus_cuda/tests/gpu_pairs_test.rs:48-62). Returns (result, singular)."""
    base = _c(base, np.float64)
    y = _c(y, np.float64)
    out = np.empty_like(base)
    s = lib().or_pair_update(base.size, _p(base), _p(y), -1 if plus is None else plus, -1 if minus is None else minus,
                             float(alpha), float(inverse_weight), _p(out))
    return out, bool(s)


def column_max(v, weight=None):
    """column_max (ybus_cuda/src/kernels.cu:78-128): (row or None, value, not_finite)."""
    v = _c(v, np.float64)
    w = None if weight is None else _c(weight, np.float64)
    row, value, bad = C.c_int64(), C.c_double(), C.c_int()
    lib().or_column_max(v.size, _p(v), _p(w), C.byref(row), C.byref(value), C.byref(bad))
    return (None if row.value < 0 else row.value), value.value, bool(bad.value)


def csr_mul_vec(ptr, idx, val, x) -> np.ndarray:
    """CsrMatrix::mul_vec (ybus_sparse/src/compressed_matrix/product.rs:17-27)."""
    ptr, idx, val, x = _c(ptr, np.int64), _c(idx, np.int64), _c(val, np.float64), _c(x, np.float64)
    out = np.empty(ptr.size - 1)
    lib().or_csr_mul_vec(ptr.size - 1, _p(ptr), _p(idx), _p(val), _p(x), _p(out))
    return out


def relative_residual(ptr, idx, val, x, b) -> float:
    """relative_residual (ybus_sparse/src/compressed_matrix/accuracy.rs:58-79)."""
    ptr, idx, val = _c(ptr, np.int64), _c(idx, np.int64), _c(val, np.float64)
    x, b = _c(x, np.float64), _c(b, np.float64)
    return lib().or_relative_residual(ptr.size - 1, _p(ptr), _p(idx), _p(val), _p(x), _p(b))


def refine_normwise(ptr, idx, val, b, max_steps, tolerance, solve):
    """`refine_normwise` (ybus_sparse/src/compressed_matrix/accuracy.rs:93-118): x = solve(b), then
    while the relative residual ||b - A x||inf / ||b||inf (accuracy.rs:58-79) is above the tolerance,
    at most max_steps corrections x += solve(b - A x), keeping the iterate with the smallest ratio,
    stopping on a NaN ratio or one above half the ratio before. A is CSR (ptr, idx, val). Returns
    (best x, its correction count, its ratio, every ratio in order, the smallest relative margin of
    the comparisons the decisions took)."""
    b = _c(b, np.float64)

    def residual(x):
        r = b - csr_mul_vec(ptr, idx, val, x)
        rn, bn = np.abs(r).max(initial=0.0), np.abs(b).max(initial=0.0)
        ratio = rn / bn if bn > 0 else (np.inf if rn > 0 else 0.0)
        return ratio, r

    def margin(lhs, rhs):
        return abs(lhs - rhs) / max(abs(rhs), 1e-300) if np.isfinite(lhs) and np.isfinite(rhs) else np.inf

    x = solve(b)
    ratio, r = residual(x)
    best = (x.copy(), 0, ratio)
    ratios, margins = [ratio], []
    for step in range(1, max_steps + 1):
        margins.append(margin(ratio, tolerance))
        if ratio <= tolerance:
            break
        x = x + solve(r)
        previous = ratio
        ratio, r = residual(x)
        ratios.append(ratio)
        margins.append(margin(ratio, best[2]))
        if ratio < best[2]:
            best = (x.copy(), step, ratio)
        margins.append(margin(ratio, 0.5 * previous))
        if np.isnan(ratio) or ratio > 0.5 * previous:
            break
    return best[0], best[1], best[2], ratios, min(margins, default=np.inf)


# ---- factor checks (independent of how the factor was made) -------------------------------

def dense_from_csr(n_rows, n_cols, ptr, idx, val, by_rows=True):
    out = np.zeros((n_rows, n_cols), dtype=np.result_type(val.dtype, np.float64))
    for major in range(len(ptr) - 1):
        for p in range(ptr[major], ptr[major + 1]):
            if by_rows:
                out[major, idx[p]] += val[p]
            else:
                out[idx[p], major] += val[p]
    return out


def cholesky_reconstruction_error(chol, a_dense) -> float:
    """max |P A Pᵀ − L Lᵀ| / max |A| for a small factor."""
    n = chol.n
    L = dense_from_csr(n, n, chol.l.ptr, chol.l.idx, chol.l.val)
    p = chol.perm
    pap = a_dense[np.ix_(p, p)]
    return float(np.abs(pap - L @ L.T).max() / max(np.abs(a_dense).max(), 1e-300))


def lu_reconstruction_error(f, a_dense) -> float:
    """max |P A Q − L U| / max |A| for a small factor."""
    n = f.n
    L = dense_from_csr(n, n, f.l.ptr, f.l.idx, f.l.val, by_rows=False)
    U = dense_from_csr(n, n, f.u.ptr, f.u.idx, f.u.val, by_rows=False)
    paq = a_dense[np.ix_(f.row_perm, f.col_perm)]
    return float(np.abs(paq - L @ U).max() / max(np.abs(a_dense).max(), 1e-300))


# ---- DC domain -----------------------------------------------------------------------------

def bridges(n_bus: int, frm, to) -> np.ndarray:
    """Which branches are bridges of the multigraph (ybus_powerflow/src/islands.rs:132-176):
    parallel branches are separate edges, so neither of a parallel pair is a bridge; a
    self-loop is never a bridge."""
    frm = np.asarray(frm)
    to = np.asarray(to)
    adj = [[] for _ in range(n_bus)]
    for k, (a, b) in enumerate(zip(frm, to)):
        if a != b:
            adj[a].append((b, k))
            adj[b].append((a, k))
    disc = [-1] * n_bus
    low = [0] * n_bus
    is_bridge = np.zeros(frm.size, dtype=bool)
    timer = 0
    for root in range(n_bus):
        if disc[root] >= 0:
            continue
        disc[root] = low[root] = timer
        timer += 1
        stack = [(root, -1, iter(adj[root]))]
        while stack:
            node, via, it = stack[-1]
            advanced = False
            for nxt, k in it:
                if k == via:
                    continue
                if disc[nxt] < 0:
                    disc[nxt] = low[nxt] = timer
                    timer += 1
                    stack.append((nxt, k, iter(adj[nxt])))
                    advanced = True
                    break
                low[node] = min(low[node], disc[nxt])
            if not advanced:
                stack.pop()
                if stack:
                    parent = stack[-1][0]
                    low[parent] = min(low[parent], low[node])
                    if low[node] > disc[parent]:
                        is_bridge[via] = True
    return is_bridge


def outage_flows_smw(solve, n_unknown, position, frm, to, b, outaged, theta_base, alpha=None):
    """`DcStudy::outage` (ybus_powerflow/src/dc/outage.rs:126-241) for outaged branches `outaged`:
    Y = A⁻¹ C, x = base + Σ α_k Y_k, W = D⁻¹ − Cᵀ Y, θ' = x + Y W⁻¹ Cᵀ x. `solve(rhs)` solves with
    the kept factor; `position[bus]` is the unknown of a bus or -1 (slack). Returns θ' over the
    unknowns. `alpha` defaults to zeros (no phase shifters, a zero-angle slack)."""
    columns = []
    for j, k in enumerate(outaged):
        entries = []
        pf, pt = position[frm[k]], position[to[k]]
        if pf >= 0:
            entries.append((pf, 1.0))
        if pt >= 0:
            entries.append((pt, -1.0))
        if frm[k] == to[k] or not entries:
            continue
        entries.sort()
        columns.append((entries, b[k], 0.0 if alpha is None else alpha[j]))
    x = np.array(theta_base, dtype=np.float64)
    ys = []
    for entries, _, _ in columns:
        c = np.zeros(n_unknown)
        for p, v in entries:
            c[p] = v
        ys.append(solve(c))
    for (_, _, a), y in zip(columns, ys):
        x = x + a * y

    def dot(entries, v):
        s = 0.0
        for p, sign in entries:
            s += sign * v[p]
        return s

    m = len(columns)
    if m:
        w = np.zeros((m, m))
        for i, (entries, bk, _) in enumerate(columns):
            for j, y in enumerate(ys):
                w[i, j] = -dot(entries, y)
                if i == j:
                    w[i, j] += 1.0 / bk
        ctx = np.array([dot(e, x) for e, _, _ in columns])
        z = np.linalg.solve(w, ctx)
        for zj, y in zip(z, ys):
            x = x + zj * y
    return x


def flow_loss_and_gradient(chol, n_bus, frm, to, susceptance, position, injections, limits, margin=0.8):
    """The flow loss Σ softplus(|f| − margin·limit)², f = diag(b) A θ, θ = B′⁻¹ p, and its gradients
    on the CPU from the oracle's solves: λ = B′⁻ᵀ (Bfᵀ dL/df) by the transposed solve (the same
    solve for a Cholesky factor, `Cholesky::substitute`, cholesky.rs:570-579), dL/dp = λ (0 at the
    slack), dL/db_k = Σ_scenarios dL/df_k d_k − (λ_f − λ_t) d_k with d_k = θ_f − θ_t.
    Returns (loss, dL/dp (count, n_bus), dL/db (n_branch))."""
    p = np.atleast_2d(np.asarray(injections, np.float64))
    frm, to = np.asarray(frm), np.asarray(to)
    b = np.asarray(susceptance, np.float64)
    unknown = position >= 0
    theta = solve_many(chol, p[:, unknown])

    def over_buses(v):
        out = np.zeros((v.shape[0], n_bus))
        out[:, unknown] = v[:, position[unknown]]
        return out

    tb = over_buses(theta)
    d = tb[:, frm] - tb[:, to]
    f = b * tb[:, frm] + (-b) * tb[:, to]
    u = np.abs(f) - margin * np.asarray(limits)
    s = np.maximum(u, 0.0) + np.log1p(np.exp(-np.abs(u)))
    loss = float((s * s).sum())
    sig = np.where(u >= 0, 1.0 / (1.0 + np.exp(-np.where(u >= 0, u, 0.0))),
                   np.exp(np.where(u < 0, u, 0.0)) / (1.0 + np.exp(np.where(u < 0, u, 0.0))))
    g = 2.0 * s * sig * np.sign(f)
    q_bus = np.zeros((p.shape[0], n_bus))
    np.add.at(q_bus.T, frm, (b * g).T)
    np.add.at(q_bus.T, to, (-b * g).T)
    q = np.zeros((p.shape[0], int(unknown.sum())))
    q[:, position[unknown]] = q_bus[:, unknown]
    lam = solve_many(chol, q)
    lb = over_buses(lam)
    e = lb[:, frm] - lb[:, to]
    grad_b = (g * d - e * d).sum(axis=0)
    return loss, lb, grad_b
