"""The GPU path's host API, mirroring ybus_cuda (ybus_cuda/src/lib.rs, factor.rs, pairs.rs).

`Gpu.new()` is `Gpu::new()`: a device, or None where there is none. `GpuFactor` is an uploaded
factorization whose `solve_many` solves many right-hand sides at once on the device. Every call
goes through libybgpu's C ABI; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import YbError, check, lib, ptr
from .host import HostCholesky, HostLu

FP64 = _lib.YB_FP64
FP32 = _lib.YB_FP32


class CudaError(YbError):
    """An error from the GPU path (ybus_cuda's `CudaError`, ybus_cuda/src/lib.rs:89-124)."""


class ShapeMismatch(CudaError):
    """A right-hand side doesn't have one entry per row (`CudaError::ShapeMismatch`)."""

    def __init__(self, expected: int, found: int):
        super().__init__(_lib.YB_ERROR_SHAPE_MISMATCH,
                         f"a right-hand side has {found} entries, but the factorization has {expected} rows")
        self.expected = expected
        self.found = found


def _check(status: int) -> None:
    if status != _lib.YB_OK:
        raise CudaError(status, _lib.last_error())


@dataclass
class Timings:
    """Time spent by `GpuFactor.solve_many`, by stage (ybus_cuda/src/factor.rs:22-31), seconds."""
    upload: float = 0.0
    solve: float = 0.0
    download: float = 0.0
    blocks: int = 0


class Gpu:
    """A CUDA device and its stream (ybus_cuda's `Gpu`)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def new(cls, device: int = 0) -> "Gpu | None":
        out = C.c_void_p()
        status = lib().yb_gpu_new(device, C.byref(out))
        if status == _lib.YB_NO_DEVICE:
            return None
        _check(status)
        return cls(out.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_gpu_free(h)
            except Exception:
                pass
            self._h = None

    def name(self) -> str:
        buf = C.create_string_buffer(256)
        _check(lib().yb_gpu_name(self._h, buf, len(buf)))
        return buf.value.decode()

    def memory(self) -> tuple[int, int]:
        free, total = C.c_uint64(), C.c_uint64()
        _check(lib().yb_gpu_memory(self._h, C.byref(free), C.byref(total)))
        return free.value, total.value

    def properties(self) -> dict:
        sm, major, minor, l2 = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int64()
        _check(lib().yb_gpu_properties(self._h, C.byref(sm), C.byref(major), C.byref(minor), C.byref(l2)))
        return {"sm_count": sm.value, "cc": (major.value, minor.value), "l2_bytes": l2.value}

    def synchronize(self, stream: int | None = None) -> None:
        _check(lib().yb_gpu_synchronize(self._h, stream))

    @property
    def stream(self) -> int:
        return lib().yb_gpu_stream(self._h) or 0


def _rhs_array(rhs, n: int) -> np.ndarray:
    """Right-hand sides as a C-contiguous (count, n) array (column-major n x count)."""
    if isinstance(rhs, np.ndarray):
        if rhs.ndim != 2:
            raise ValueError("right-hand sides are a (count, n) array")
        if rhs.shape[1] != n and rhs.shape[0] > 0:
            raise ShapeMismatch(n, rhs.shape[1])
        return np.ascontiguousarray(rhs, dtype=np.float64)
    rows = list(rhs)
    for b in rows:
        if len(b) != n:
            raise ShapeMismatch(n, len(b))
    if not rows:
        return np.zeros((0, n))
    return np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(len(rows), n))


class GpuFactor:
    """A factorization uploaded once, solving blocks of right-hand sides (ybus_cuda's `GpuFactor`)."""

    def __init__(self, gpu: Gpu, handle: int):
        self.gpu = gpu
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_factor_free(h)
            except Exception:
                pass
            self._h = None

    @classmethod
    def from_cholesky(cls, gpu: Gpu, chol: HostCholesky) -> "GpuFactor":
        out = C.c_void_p()
        l = chol.l
        _check(lib().yb_factor_from_cholesky(gpu._h, chol.n, ptr(l.ptr), ptr(l.idx), ptr(np.ascontiguousarray(l.val)),
                                             ptr(chol.perm), C.byref(out)))
        return cls(gpu, out.value)

    @classmethod
    def from_lu(cls, gpu: Gpu, f: HostLu) -> "GpuFactor":
        if f.is_complex:
            raise CudaError(_lib.YB_ERROR_INVALID_ARGUMENT, "a complex factor uploads with from_lu_complex")
        out = C.c_void_p()
        _check(lib().yb_factor_from_lu(gpu._h, f.n, ptr(f.l.ptr), ptr(f.l.idx), ptr(f.l.val), ptr(f.u.ptr),
                                       ptr(f.u.idx), ptr(f.u.val), ptr(f.row_perm), ptr(f.col_perm), C.byref(out)))
        return cls(gpu, out.value)

    @classmethod
    def from_lu_transposed(cls, gpu: Gpu, f: HostLu) -> "GpuFactor":
        """The factor of Aᵀ from A's LU (`Lu::solve_transpose`, lu.rs:506-533): its solves solve Aᵀ x = b."""
        if f.is_complex:
            raise CudaError(_lib.YB_ERROR_INVALID_ARGUMENT, "a real LU factor only")
        out = C.c_void_p()
        _check(lib().yb_factor_from_lu_transposed(gpu._h, f.n, ptr(f.l.ptr), ptr(f.l.idx), ptr(f.l.val), ptr(f.u.ptr),
                                                  ptr(f.u.idx), ptr(f.u.val), ptr(f.row_perm), ptr(f.col_perm),
                                                  C.byref(out)))
        return cls(gpu, out.value)

    @classmethod
    def from_lu_complex(cls, gpu: Gpu, f: HostLu) -> "GpuFactor":
        """A complex128 LU factor (P A Q = L U of a Ybus), kept in complex128 and complex64."""
        if not f.is_complex:
            raise CudaError(_lib.YB_ERROR_INVALID_ARGUMENT, "a real factor uploads with from_lu")
        lv = np.ascontiguousarray(f.l.val, np.complex128)
        uv = np.ascontiguousarray(f.u.val, np.complex128)
        out = C.c_void_p()
        _check(lib().yb_factor_from_lu_complex(gpu._h, f.n, ptr(f.l.ptr), ptr(f.l.idx), ptr(lv), ptr(f.u.ptr),
                                               ptr(f.u.idx), ptr(uv), ptr(f.row_perm), ptr(f.col_perm),
                                               C.byref(out)))
        factor = cls(gpu, out.value)
        factor._keep = (lv, uv)
        return factor

    def attach_matrix_complex(self, a) -> None:
        """Attaches the complex A (a host.Matrix) for refinement and residuals."""
        p, i, v = a.to_csr().arrays()
        v = np.ascontiguousarray(v, np.complex128)
        self._cmatrix = (p, i, v)
        _check(lib().yb_factor_attach_matrix_complex(self._h, ptr(p), ptr(i), ptr(v)))

    def dim(self) -> int:
        return lib().yb_factor_dim(self._h)

    def block_width(self) -> int:
        return lib().yb_factor_block_width(self._h)

    def set_block_width(self, width: int) -> None:
        _check(lib().yb_factor_set_block_width(self._h, width))

    def timings(self) -> Timings:
        u, s, d, b = C.c_double(), C.c_double(), C.c_double(), C.c_int64()
        _check(lib().yb_factor_timings(self._h, C.byref(u), C.byref(s), C.byref(d), C.byref(b)))
        return Timings(u.value, s.value, d.value, b.value)

    def reset_timings(self) -> None:
        _check(lib().yb_factor_reset_timings(self._h))

    def plan_info(self) -> dict:
        fl, bl, fe, be, fw, bw = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64(), C.c_int32(), C.c_int32()
        _check(lib().yb_factor_plan_info(self._h, C.byref(fl), C.byref(bl), C.byref(fe), C.byref(be), C.byref(fw),
                                         C.byref(bw)))
        return {"fwd_levels": fl.value, "bwd_levels": bl.value, "fwd_entries": fe.value, "bwd_entries": be.value,
                "fwd_widest": fw.value, "bwd_widest": bw.value}

    def set_tile(self, precision: int, width: int, threads: int = 512, blocks_per_sm: int = 1) -> None:
        _check(lib().yb_factor_set_tile(self._h, precision, width, threads, blocks_per_sm))

    def set_tile_kind(self, precision: int, kind: int) -> None:
        """0 automatic, 1 shared-memory, 2 global-scratch, 3 streamed, 4 domain tile, 5 lane solve."""
        _check(lib().yb_factor_set_tile_kind(self._h, precision, kind))

    def set_stream(self, precision: int, warps: int = 8, ring: int = 4, page_bytes: int = 2048,
                   narrow_rows: int = 0) -> None:
        _check(lib().yb_factor_set_stream(self._h, precision, warps, ring, page_bytes, narrow_rows))

    def stream_info(self, precision: int) -> dict:
        w, st, nf, nb, nr = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        rec, by = C.c_int64(), C.c_int64()
        _check(lib().yb_factor_stream_info(self._h, precision, C.byref(w), C.byref(st), C.byref(rec), C.byref(by),
                                           C.byref(nf), C.byref(nb), C.byref(nr)))
        return {"tile": w.value, "stages": st.value, "records": rec.value, "bytes": by.value,
                "fwd_wide_levels": nf.value, "bwd_wide_levels": nb.value, "narrow_rows": nr.value}

    def set_tail_level(self, precision: int, level: int) -> None:
        """-1: chosen from the factor, 0: no dense tail, else the first forward level of the tail."""
        _check(lib().yb_factor_set_tail_level(self._h, precision, level))

    def set_domain(self, precision: int, warps: int = 16, ring: int = 2, page_bytes: int = 2048, cut: int = -1) -> None:
        """The domain solve's shape: warps per block, pages in flight per warp, page bytes, cut
        (-1: chosen by the layout's cost model)."""
        _check(lib().yb_factor_set_domain(self._h, precision, warps, ring, page_bytes, cut))

    def domain_info(self, precision: int) -> dict:
        w, cut, top = C.c_int32(), C.c_int32(), C.c_int32()
        rec, by, sm, cyc = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        _check(lib().yb_factor_domain_info(self._h, precision, C.byref(w), C.byref(cut), C.byref(top), C.byref(rec),
                                           C.byref(by), C.byref(sm), C.byref(cyc)))
        return {"tile": w.value, "cut": cut.value, "top": top.value, "records": rec.value, "bytes": by.value,
                "smem": sm.value, "model_cycles": cyc.value}

    def set_lane_rhs_per_lane(self, precision: int, rhs_per_lane: int) -> None:
        """How many right-hand sides each lane of the plain lane solve carries (1 or 2)."""
        _check(lib().yb_factor_set_lane_rhs_per_lane(self._h, precision, rhs_per_lane))

    def lane_info(self, precision: int = FP64) -> dict:
        """The lane solve's layout: slots, pages, peaks of live values, shared memory per block,
        warps per block, domains, top rows and partial values per block."""
        v = np.zeros(12, np.int64)
        _check(lib().yb_factor_lane_info(self._h, precision, ptr(v)))
        keys = ("slots", "pages", "page_bytes", "fwd_live", "bwd_live", "entries", "smem", "warps", "domains", "top",
                "partials", "rpl")
        return dict(zip(keys, (int(a) for a in v)))

    def set_lane(self, precision: int, warps: int, page_bytes: int = 0) -> None:
        """The lane solve's warps per block (1..16) and page bytes (0: the automatic choice)."""
        _check(lib().yb_factor_set_lane(self._h, precision, warps, page_bytes))

    def set_lane_min_count(self, precision: int, min_count: int) -> None:
        """The number of right-hand sides from which the automatic choice takes the lane solve
        (-1: the automatic threshold, by the factor's domain tiles)."""
        _check(lib().yb_factor_set_lane_min_count(self._h, precision, min_count))

    def set_refine_lane_min_count(self, min_count: int) -> None:
        """The number of right-hand sides from which the refined solve takes the FP32 lane solve."""
        _check(lib().yb_factor_set_refine_lane_min_count(self._h, min_count))

    def lane_min_count(self, precision: int = FP64) -> int:
        """The number of right-hand sides from which the automatic choice takes the lane solve."""
        v = C.c_int64()
        _check(lib().yb_factor_lane_min_counts(self._h, precision, C.byref(v), None))
        return v.value

    def refine_lane_min_count(self) -> int:
        """The refined solve's own lane threshold."""
        v = C.c_int64()
        _check(lib().yb_factor_lane_min_counts(self._h, FP32, None, C.byref(v)))
        return v.value

    def time_lane(self, on: bool = True) -> None:
        """Records CUDA events around the gather, solve and scatter of every lane-solve launch
        (on), or stops; either way clears the record."""
        _check(lib().yb_factor_time_lane(self._h, 1 if on else 0))

    def lane_times(self) -> dict:
        """Total device milliseconds of the recorded lane launches' gathers, solves and scatters
        and their count (waits for them); clears the record."""
        g, s_, o, k = C.c_double(), C.c_double(), C.c_double(), C.c_int64()
        _check(lib().yb_factor_lane_times(self._h, C.byref(g), C.byref(s_), C.byref(o), C.byref(k)))
        return {"gather_ms": g.value, "solve_ms": s_.value, "scatter_ms": o.value, "launches": k.value}

    def autotune(self, precision: int = FP64, count: int = 2048) -> dict:
        """Times the domain and lane solves' shapes on `count` right-hand sides and keeps the fastest."""
        cfg = np.zeros(5, np.int32)
        ms = C.c_double()
        _check(lib().yb_factor_autotune(self._h, precision, count, ptr(cfg), C.byref(ms)))
        return {"kind": int(cfg[0]), "tile": int(cfg[1]), "warps": int(cfg[2]), "ring": int(cfg[3]),
                "page_bytes": int(cfg[4]), "ms": ms.value}

    def set_phase_clock(self, d_clock: int | None) -> None:
        """Diagnostics: a device buffer of 512 int64 for phase clocks (None to stop)."""
        _check(lib().yb_factor_set_phase_clock(self._h, d_clock))

    def check_error(self) -> None:
        _check(lib().yb_factor_check_error(self._h))

    def tile(self, precision: int) -> tuple[int, int, int]:
        w, t, b = C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().yb_factor_get_tile(self._h, precision, C.byref(w), C.byref(t), C.byref(b)))
        return w.value, t.value, b.value

    def solve_many(self, rhs) -> np.ndarray:
        """Solves A x = b for each right-hand side (a (count, n) array or a list of vectors) and
        returns the solutions as a (count, n) array, in order (factor.rs:234-289)."""
        n = self.dim()
        b = _rhs_array(rhs, n)
        out = np.empty_like(b)
        if b.shape[0] == 0 or n == 0:
            return out
        _check(lib().yb_solve_many(self._h, ptr(b), b.shape[0], ptr(out)))
        return out

    def solve_many_transpose(self, rhs) -> np.ndarray:
        """Solves A' x = b for each right-hand side (`Lu::solve_transpose`, lu.rs:506-533)."""
        n = self.dim()
        b = _rhs_array(rhs, n)
        out = np.empty_like(b)
        if b.shape[0] == 0 or n == 0:
            return out
        _check(lib().yb_solve_many_transpose(self._h, ptr(b), b.shape[0], ptr(out)))
        return out

    def solve_many_mixed(self, rhs, max_steps: int = 3, tolerance: float = 1e-10):
        """FP32 substitution with FP64 refinement against the attached matrix, host arrays in and
        out: returns (x, corrections per column, relative residual per column)."""
        n = self.dim()
        b = _rhs_array(rhs, n)
        out = np.empty_like(b)
        steps = np.zeros(b.shape[0], np.int32)
        ratio = np.zeros(b.shape[0])
        if b.shape[0] == 0 or n == 0:
            return out, steps, ratio
        _check(lib().yb_solve_many_mixed(self._h, ptr(b), b.shape[0], ptr(out), max_steps, tolerance, ptr(steps),
                                         ptr(ratio)))
        return out, steps, ratio

    def solve_many_into(self, b: np.ndarray, out: np.ndarray) -> None:
        """`solve_many` into a caller's (count, n) buffer (pinned buffers are copied directly)."""
        _check(lib().yb_solve_many(self._h, b.ctypes.data, b.shape[0], out.ctypes.data))

    def attach_matrix(self, a) -> None:
        """Attaches A (a host.Matrix, or (ptr, idx, val) CSR arrays in natural order) for refinement."""
        if hasattr(a, "arrays"):
            a = a.to_csr().arrays()
        p, i, v = (np.ascontiguousarray(a[0], dtype=np.int64), np.ascontiguousarray(a[1], dtype=np.int64),
                   np.ascontiguousarray(a[2], dtype=np.float64))
        self._matrix = (p, i, v)
        _check(lib().yb_factor_attach_matrix(self._h, ptr(p), ptr(i), ptr(v)))

    def solve_many_refined_device(self, d_rhs: int, d_out: int, count: int, max_steps: int = 3,
                                  tolerance: float = 1e-10, d_ratio: int | None = None, d_steps: int | None = None,
                                  stream: int | None = None, ldb: int | None = None, ldx: int | None = None) -> None:
        """FP32 substitution with FP64 refinement on device pointers (accuracy.rs:83-122)."""
        n = self.dim()
        _check(lib().yb_solve_many_refined_device(self._h, d_rhs, ldb or n, d_out, ldx or n, count, max_steps,
                                                  float(tolerance), d_ratio, d_steps, stream))

    def operator(self, matrix) -> "GpuOperator":
        """`GpuFactor::operator` (pairs.rs:112-149): a CSR matrix (host.Matrix or (rows, ptr, idx, val))
        with one column per unknown."""
        if hasattr(matrix, "arrays"):
            m = matrix.to_csr()
            rows = m.shape[0]
            p, i, v = m.arrays()
        else:
            rows, p, i, v = matrix
        p, i, v = np.ascontiguousarray(p, np.int64), np.ascontiguousarray(i, np.int64), np.ascontiguousarray(v, np.float64)
        out = C.c_void_p()
        _check(lib().yb_operator_new(self._h, rows, ptr(p), ptr(i), ptr(v), C.byref(out)))
        return GpuOperator(self, out.value)


    def pair_solves(self, pairs) -> "GpuBlock":
        """`GpuFactor::pair_solves` (pairs.rs:194-202)."""
        plus, minus = _pair_arrays(pairs)
        out = C.c_void_p()
        _check(lib().yb_pair_solves(self._h, plus.size, ptr(plus), ptr(minus), C.byref(out)))
        return GpuBlock(self, out.value)


    def pair_updates(self, base, updates) -> "GpuBlock":
        """`GpuFactor::pair_updates` (pairs.rs:209-253)."""
        base = np.ascontiguousarray(base, dtype=np.float64)
        if base.size != self.dim():
            raise ValueError("one base value per unknown")
        plus, minus = _pair_arrays([u.pair for u in updates])
        alpha = np.array([u.alpha for u in updates], np.float64)
        inv = np.array([u.inverse_weight for u in updates], np.float64)
        out = C.c_void_p()
        _check(lib().yb_pair_updates(self._h, ptr(base), plus.size, ptr(plus), ptr(minus), ptr(alpha), ptr(inv),
                                     C.byref(out)))
        return GpuBlock(self, out.value)

    def solve_many_device(self, d_rhs: int, d_out: int, count: int, precision: int = FP64, stream: int | None = None,
                          ldb: int | None = None, ldx: int | None = None) -> None:
        """The solve on device pointers (column-major n x count), asynchronous on `stream`."""
        n = self.dim()
        _check(lib().yb_solve_many_device(self._h, d_rhs, ldb or n, d_out, ldx or n, count, precision, stream))


# ---- blocks solved on the device (ybus_cuda/src/pairs.rs) ----------------------------------------

@dataclass(frozen=True)
class Pair:
    """A right-hand side e_plus − e_minus over the unknowns (None for no entry) (pairs.rs:17)."""
    plus: int | None
    minus: int | None


@dataclass(frozen=True)
class PairUpdate:
    """One column of `pair_updates` (pairs.rs:30): x = base + alpha y, w = inverse_weight − cᵀy,
    z = cᵀx / w, result x + z y."""
    pair: Pair
    alpha: float
    inverse_weight: float


@dataclass(frozen=True)
class ColumnMax:
    """A column's largest |value| · weight (pairs.rs:42): its row (None if all are zero), the value,
    and whether any value isn't finite."""
    row: int | None
    value: float
    not_finite: bool


def _pair_arrays(pairs):
    plus = np.array([-1 if p.plus is None else p.plus for p in pairs], np.int64)
    minus = np.array([-1 if p.minus is None else p.minus for p in pairs], np.int64)
    return plus, minus


def _maxima(rows, values, bad):
    return [ColumnMax(None if r < 0 else int(r), float(v), bool(b)) for r, v, b in zip(rows, values, bad)]


class GpuOperator:
    """A sparse matrix over a factor's unknowns, applied to a block's columns (pairs.rs:55-86)."""

    def __init__(self, factor: "GpuFactor", handle: int):
        self.factor = factor
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_operator_free(h)
            except Exception:
                pass
            self._h = None

    def rows(self) -> int:
        return lib().yb_operator_rows(self._h)

    def set_offset(self, offset) -> None:
        offset = np.ascontiguousarray(offset, dtype=np.float64)
        if offset.size != self.rows():
            raise ValueError("one offset per row")
        _check(lib().yb_operator_set_offset(self._h, ptr(offset)))

    def set_weights(self, weights) -> None:
        weights = np.ascontiguousarray(weights, dtype=np.float64)
        if weights.size != self.rows():
            raise ValueError("one weight per row")
        _check(lib().yb_operator_set_weights(self._h, ptr(weights)))


class GpuBlock:
    """Solutions kept on the device, one column per pair (pairs.rs:90-110)."""

    def __init__(self, factor: "GpuFactor", handle: int):
        self.factor = factor
        self._h = C.c_void_p(handle)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_block_free(h)
            except Exception:
                pass
            self._h = None

    def columns(self) -> int:
        return lib().yb_block_columns(self._h)

    def singular(self) -> list[bool]:
        out = np.zeros(max(self.columns(), 1), np.int32)
        _check(lib().yb_block_singular(self._h, ptr(out)))
        return [bool(v) for v in out[: self.columns()]]

    def solutions(self) -> np.ndarray:
        out = np.zeros((self.columns(), self.factor.dim()))
        _check(lib().yb_block_solutions(self._h, ptr(out)))
        return out

    def maxima(self) -> list[ColumnMax]:
        k = self.columns()
        rows, values, bad = np.zeros(max(k, 1), np.int64), np.zeros(max(k, 1)), np.zeros(max(k, 1), np.int32)
        _check(lib().yb_block_maxima(self._h, ptr(rows), ptr(values), ptr(bad)))
        return _maxima(rows[:k], values[:k], bad[:k])

    @staticmethod
    def _zero(zero, k):
        return np.array([-1 if z is None else z for z in zero], np.int64) if zero is not None else np.full(k, -1, np.int64)

    def product(self, op: GpuOperator, zero=None) -> np.ndarray:
        k = self.columns()
        z = self._zero(zero, k)
        out = np.zeros((k, op.rows()))
        _check(lib().yb_block_product(self._h, op._h, ptr(z), ptr(out)))
        return out

    def product_maxima(self, op: GpuOperator, zero=None) -> list[ColumnMax]:
        k = self.columns()
        z = self._zero(zero, k)
        rows, values, bad = np.zeros(max(k, 1), np.int64), np.zeros(max(k, 1)), np.zeros(max(k, 1), np.int32)
        _check(lib().yb_block_product_maxima(self._h, op._h, ptr(z), ptr(rows), ptr(values), ptr(bad)))
        return _maxima(rows[:k], values[:k], bad[:k])




def solve_batch_complex(factors, d_rhs, d_out, counts, precision: int = FP64, max_steps: int = 3,
                        tolerance: float = 1e-10, d_ratio=None, stream: int | None = None) -> list[int]:
    """Solves many complex factors' right-hand sides in one launch (device pointers per network,
    complex128 column-major n x count). FP64: complex128 substitution; FP32: complex64 substitution
    with complex128 refinement. Returns the corrections taken per network."""
    k = len(factors)
    hs = (C.c_void_p * k)(*[f._h.value for f in factors])
    rhs = (C.c_void_p * k)(*d_rhs)
    out = (C.c_void_p * k)(*d_out)
    cnt = np.ascontiguousarray(counts, np.int64)
    ratio = (C.c_void_p * k)(*d_ratio) if d_ratio is not None else None
    steps = np.zeros(k, np.int32)
    _check(lib().yb_solve_batch_complex(k, hs, rhs, out, ptr(cnt), precision, max_steps, float(tolerance), ratio,
                                        ptr(steps), stream))
    return steps.tolist()
