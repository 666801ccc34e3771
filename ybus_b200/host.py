"""The host-side factor producer: sparse matrices and their Cholesky and LU factors.

These are the ybus_sparse calls whose results ybus_cuda uploads (`CsrMatrix::cholesky`,
`CscMatrix::analyze_lu(..).factor(..)`, ybus_sparse/src/compressed_matrix/{cholesky,lu}.rs),
computed in FP64 (or complex128) by libybhost.so's C++ code; the layout diagnostics at the end
call libybgpu.so's host-side layout builders.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, ptr
from ._lib import host_lib as lib

NATURAL = _lib.YB_ORDER_NATURAL
AMD = _lib.YB_ORDER_AMD
COLAMD = _lib.YB_ORDER_COLAMD


class Matrix:
    """A compressed sparse matrix (CSR when `by_rows`, else CSC), real or complex."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_matrix_free(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def from_triplets(cls, rows: int, cols: int, r, c, v, by_rows: bool = True) -> "Matrix":
        r = np.ascontiguousarray(r, dtype=np.int64)
        c = np.ascontiguousarray(c, dtype=np.int64)
        is_complex = np.iscomplexobj(v)
        v = np.ascontiguousarray(v, dtype=np.complex128 if is_complex else np.float64)
        if not (r.size == c.size == v.size):
            raise ValueError("triplet arrays differ in length")
        out = C.c_void_p()
        check(lib().yb_matrix_from_triplets(rows, cols, r.size, ptr(r), ptr(c), ptr(v), int(by_rows),
                                            int(is_complex), C.byref(out)))
        return cls(out.value)

    def info(self):
        rows, cols, stored = C.c_int64(), C.c_int64(), C.c_int64()
        by_rows, cplx = C.c_int32(), C.c_int32()
        check(lib().yb_matrix_info(self._h, C.byref(rows), C.byref(cols), C.byref(stored), C.byref(by_rows),
                                   C.byref(cplx)))
        return rows.value, cols.value, stored.value, bool(by_rows.value), bool(cplx.value)

    @property
    def shape(self):
        r, c, *_ = self.info()
        return r, c

    @property
    def by_rows(self) -> bool:
        return self.info()[3]

    @property
    def is_complex(self) -> bool:
        return self.info()[4]

    def arrays(self):
        """(ptr, idx, values) as numpy arrays."""
        rows, cols, stored, by_rows, cplx = self.info()
        major = rows if by_rows else cols
        p = np.zeros(major + 1, np.int64)
        i = np.zeros(stored, np.int64)
        v = np.zeros(stored, np.complex128 if cplx else np.float64)
        check(lib().yb_matrix_export(self._h, ptr(p), ptr(i), ptr(v)))
        return p, i, v

    def select(self, rows, cols) -> "Matrix":
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        out = C.c_void_p()
        check(lib().yb_matrix_select(self._h, rows.size, ptr(rows), cols.size, ptr(cols), C.byref(out)))
        return Matrix(out.value)

    def reoriented(self) -> "Matrix":
        out = C.c_void_p()
        check(lib().yb_matrix_reorient(self._h, C.byref(out)))
        return Matrix(out.value)

    def to_csc(self) -> "Matrix":
        return self if not self.by_rows else self.reoriented()

    def to_csr(self) -> "Matrix":
        return self if self.by_rows else self.reoriented()

    def ordering(self, kind: int = AMD) -> np.ndarray:
        n = self.shape[1]
        perm = np.zeros(n, np.int64)
        check(lib().yb_ordering(self._h, kind, ptr(perm)))
        return perm

    def to_dense(self) -> np.ndarray:
        rows, cols, _, by_rows, cplx = self.info()
        p, i, v = self.arrays()
        out = np.zeros((rows, cols), np.complex128 if cplx else np.float64)
        for major in range(p.size - 1):
            for q in range(p[major], p[major + 1]):
                if by_rows:
                    out[major, i[q]] += v[q]
                else:
                    out[i[q], major] += v[q]
        return out


@dataclass
class Triangle:
    ptr: np.ndarray
    idx: np.ndarray
    val: np.ndarray


@dataclass
class HostCholesky:
    """P A Pᵀ = L Lᵀ: `l` in CSR (diagonal last per row), `lt` = Lᵀ in CSR (diagonal first)."""
    n: int
    l: Triangle
    lt: Triangle
    perm: np.ndarray
    parent: np.ndarray


@dataclass
class HostLu:
    """P A Q = L U: `l` unit lower in CSC (diagonal first), `u` upper in CSC (diagonal last)."""
    n: int
    l: Triangle
    u: Triangle
    row_perm: np.ndarray
    col_perm: np.ndarray
    is_complex: bool


def _export(handle) -> tuple:
    kind, cplx, n, lo, up = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
    check(lib().yb_host_factor_info(handle, C.byref(kind), C.byref(cplx), C.byref(n), C.byref(lo), C.byref(up)))
    n_, lo_, up_ = n.value, lo.value, up.value
    dt = np.complex128 if cplx.value else np.float64
    lp, li, lv = np.zeros(n_ + 1, np.int64), np.zeros(lo_, np.int64), np.zeros(lo_, dt)
    up_p, ui, uv = np.zeros(n_ + 1, np.int64), np.zeros(up_, np.int64), np.zeros(up_, dt)
    rp, cp = np.zeros(n_, np.int64), np.zeros(n_, np.int64)
    check(lib().yb_host_factor_export(handle, ptr(lp), ptr(li), ptr(lv), ptr(up_p), ptr(ui), ptr(uv), ptr(rp), ptr(cp)))
    return kind.value, bool(cplx.value), n_, Triangle(lp, li, lv), Triangle(up_p, ui, uv), rp, cp


def cholesky(a: Matrix, ordering: int = AMD) -> HostCholesky:
    """`CsrMatrix::analyze_cholesky(ordering)` then `factor` (cholesky.rs:50-311)."""
    h = C.c_void_p()
    check(lib().yb_host_cholesky(a._h, ordering, C.byref(h)))
    try:
        _, _, n, l, lt, perm, _ = _export(h)
        parent = np.zeros(n, np.int64)
        check(lib().yb_host_etree(h, ptr(parent)))
    finally:
        lib().yb_host_factor_free(h)
    return HostCholesky(n=n, l=l, lt=lt, perm=perm, parent=parent)


def lu(a: Matrix, ordering: int = AMD, pivot_threshold: float = 0.1) -> HostLu:
    """`CscMatrix::analyze_lu(ordering)` then `factor` (lu.rs:142-247); A must be CSC."""
    h = C.c_void_p()
    check(lib().yb_host_lu(a._h, ordering, pivot_threshold, C.byref(h)))
    try:
        _, cplx, n, l, u, rp, cp = _export(h)
    finally:
        lib().yb_host_factor_free(h)
    return HostLu(n=n, l=l, u=u, row_perm=rp, col_perm=cp, is_complex=cplx)


def domain_layout(chol: HostCholesky, value_bytes: int = 8, warps: int = 16, page_bytes: int = 2048,
                  cut: int = -1) -> dict:
    """The domain solve's records for a Cholesky factor, built on the host (no GPU): the per-warp
    pages the kernel streams, with the cut and the top block's rows (diagnostics and tests)."""
    info = np.zeros(8, np.int64)
    l = chol.l
    val = np.ascontiguousarray(l.val, dtype=np.float64)
    args = (chol.n, ptr(l.ptr), ptr(l.idx), ptr(val), ptr(chol.perm), value_bytes, warps, page_bytes, cut)
    check(_lib.lib().yb_domain_layout_cholesky(*args, ptr(info), None, None, None, None))
    cut_, top, stages, w, pages, records, entries, pb = (int(v) for v in info)
    blob = np.zeros(pages * pb, np.uint8)
    warp_page = np.zeros(w + 1, np.int32)
    top_slot = np.zeros(max(top, 1), np.int32)
    cond = C.c_double()
    check(_lib.lib().yb_domain_layout_cholesky(*args, ptr(info), ptr(blob), ptr(warp_page), ptr(top_slot),
                                               C.byref(cond)))
    return {"cut": cut_, "top": top, "stages": stages, "warps": w, "pages": pages, "records": records,
            "entries": entries, "page_bytes": pb, "blob": blob, "warp_page": warp_page, "top_slot": top_slot[:top],
            "value_bytes": value_bytes, "top_condition": cond.value}


def lane_layout(factor: "HostCholesky | HostLu", value_bytes: int = 8, page_bytes: int = 2048,
                max_slots: int = 1 << 20, warps: int = 1, rpl: int = 1) -> dict:
    """The lane solve's records for a Cholesky or a real LU factor, built on the host (no GPU):
    every warp's pages and each row's position in the work array (diagnostics and tests); `rpl`
    right-hand sides per lane (1 or 2)."""
    info = np.zeros(12, np.int64)
    n = factor.n
    if isinstance(factor, HostLu):
        if factor.is_complex:
            raise ValueError("a real LU factor only")
        lv = np.ascontiguousarray(factor.l.val, dtype=np.float64)
        uv = np.ascontiguousarray(factor.u.val, dtype=np.float64)
        fn = _lib.lib().yb_lane_layout_lu
        args = (n, ptr(factor.l.ptr), ptr(factor.l.idx), ptr(lv), ptr(factor.u.ptr), ptr(factor.u.idx), ptr(uv),
                ptr(factor.row_perm), ptr(factor.col_perm), value_bytes, page_bytes, max_slots, warps, rpl)
    else:
        l = factor.l
        val = np.ascontiguousarray(l.val, dtype=np.float64)
        fn = _lib.lib().yb_lane_layout_cholesky
        args = (n, ptr(l.ptr), ptr(l.idx), ptr(val), ptr(factor.perm), value_bytes, page_bytes, max_slots, warps, rpl)
    check(fn(*args, ptr(info), None, None, None, None))
    slots, pages, pb, fwd_live, bwd_live, fwd_entries, bwd_entries, w, domains, top, partials, r = (int(v) for v in info)
    blob = np.zeros(pages * pb, np.uint8)
    warp_page = np.zeros(w + 1, np.int32)
    in_pos = np.zeros(n, np.int32)
    out_pos = np.zeros(n, np.int32)
    check(fn(*args, ptr(info), ptr(blob), ptr(warp_page), ptr(in_pos), ptr(out_pos)))
    return {"slots": slots, "pages": pages, "page_bytes": pb, "fwd_live": fwd_live, "bwd_live": bwd_live,
            "fwd_entries": fwd_entries, "bwd_entries": bwd_entries, "warps": w, "domains": domains, "top": top,
            "partials": partials, "blob": blob, "warp_page": warp_page, "in_pos": in_pos, "out_pos": out_pos,
            "value_bytes": value_bytes, "rpl": r}
