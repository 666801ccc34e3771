"""The DC callers of the solve path (ybus_powerflow/src/dc/gpu.rs `DcGpuStudy`,
`DcGpuSensitivity`), over libybgpu's C ABI: a network from its branch list, PTDF and LODF columns,
bridges, and the batched N-1 screening of injection scenarios."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import lib, ptr
from .gpu import FP64, Gpu, _check


# The flags of a screened or solved scenario
FLOW_NOT_FINITE = 1  # a branch flow is not finite
ANGLE_SUSPECT = 2    # an angle is not finite or above 1e5 in magnitude


class DcNetwork:
    """B′ and Bf of a network (bus indices `frm`, `to`, reactances `x`, a slack bus), B′ factored
    on the host and uploaded, Bf kept on the device as an operator on the solutions."""

    def __init__(self, gpu: Gpu, n_bus: int, frm, to, x, slack: int = 0):
        self.gpu = gpu
        self.n_bus = int(n_bus)
        self.frm = np.ascontiguousarray(frm, np.int64)
        self.to = np.ascontiguousarray(to, np.int64)
        self.x = np.ascontiguousarray(x, np.float64)
        self.slack = int(slack)
        out = C.c_void_p()
        _check(lib().yb_dc_network_new(gpu._h, self.n_bus, self.frm.size, ptr(self.frm), ptr(self.to), ptr(self.x),
                                       self.slack, C.byref(out)))
        self._h = out

    @classmethod
    def from_grid(cls, gpu: Gpu, grid, slack: int = 0) -> "DcNetwork":
        return cls(gpu, grid.n_bus, grid.frm, grid.to, grid.x, slack)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_dc_network_free(h)
            except Exception:
                pass
            self._h = None

    @property
    def n_branch(self) -> int:
        return int(self.frm.size)

    def bridges(self) -> np.ndarray:
        out = np.zeros(self.n_branch, np.uint8)
        _check(lib().yb_dc_bridges(self._h, ptr(out)))
        return out.astype(bool)

    def ptdf_columns(self, buses) -> np.ndarray:
        """(count, n_branch): each bus's PTDF column (injection there, withdrawal at the slack)."""
        buses = np.ascontiguousarray(buses, np.int64)
        out = np.zeros((buses.size, self.n_branch))
        _check(lib().yb_dc_ptdf_columns(self._h, buses.size, ptr(buses), ptr(out)))
        return out

    def ptdf_transfers(self, from_bus, to_bus) -> np.ndarray:
        f = np.ascontiguousarray(from_bus, np.int64)
        t = np.ascontiguousarray(to_bus, np.int64)
        out = np.zeros((f.size, self.n_branch))
        _check(lib().yb_dc_ptdf_transfers(self._h, f.size, ptr(f), ptr(t), ptr(out)))
        return out

    def lodf_columns(self, branches) -> np.ndarray:
        """(count, n_branch): each outaged branch's LODF column (NaN for a bridge)."""
        br = np.ascontiguousarray(branches, np.int64)
        out = np.zeros((br.size, self.n_branch))
        _check(lib().yb_dc_lodf_columns(self._h, br.size, ptr(br), ptr(out)))
        return out

    def outage_loadings_batch(self, outaged, scenario_ptr, injections, weights=None, precision: int = FP64):
        """N-1 screening: case c takes out branch outaged[c] under the scenarios
        injections[scenario_ptr[c]:scenario_ptr[c+1]] (each a vector over the buses). Returns
        (branch, loading, flags) per scenario (flags: FLOW_NOT_FINITE | ANGLE_SUSPECT bits) and
        singular per case."""
        outaged = np.ascontiguousarray(outaged, np.int64)
        sp = np.ascontiguousarray(scenario_ptr, np.int64)
        inj = np.ascontiguousarray(injections, np.float64)
        total = int(sp[-1]) if sp.size else 0
        if inj.shape != (total, self.n_bus):
            raise ValueError("one injection vector over the buses per scenario")
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        row = np.zeros(max(total, 1), np.int64)
        val = np.zeros(max(total, 1))
        bad = np.zeros(max(total, 1), np.int32)
        sing = np.zeros(max(outaged.size, 1), np.int32)
        _check(lib().yb_dc_outage_loadings_batch(self._h, outaged.size, ptr(outaged), ptr(sp), ptr(inj), ptr(w),
                                                 precision, ptr(row), ptr(val), ptr(bad), ptr(sing)))
        return row[:total], val[:total], bad[:total], sing[: outaged.size].astype(bool)

    def set_slack_weights(self, weights=None) -> None:
        """A distributed slack for PTDF columns (weights per bus, normalized to sum to 1), or the
        single slack again (None)."""
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        if w is not None and w.shape != (self.n_bus,):
            raise ValueError("one weight per bus")
        _check(lib().yb_dc_set_slack_weights(self._h, ptr(w)))

    def solve_many(self, injections):
        """Angles over the buses (slack 0), branch flows and flags per scenario (each row of
        `injections` a vector over the buses)."""
        inj = np.ascontiguousarray(np.atleast_2d(injections), np.float64)
        if inj.shape[1] != self.n_bus:
            raise ValueError("one injection vector over the buses per scenario")
        count = inj.shape[0]
        theta = np.zeros((count, self.n_bus))
        flows = np.zeros((count, self.n_branch))
        flags = np.zeros(max(count, 1), np.int32)
        _check(lib().yb_dc_solve_many(self._h, count, ptr(inj), ptr(theta), ptr(flows), ptr(flags)))
        return theta, flows, flags[:count]

    def outage_solutions(self, outages, scenario_ptr, injections):
        """Whole solutions of outages of one or more branches each: case c takes out the branches
        outages[c] (a sequence) under the scenarios injections[scenario_ptr[c]:scenario_ptr[c+1]].
        Returns (theta over the buses, flows, flags) per scenario and singular per case."""
        cases = len(outages)
        bp = np.zeros(cases + 1, np.int64)
        for c, rows in enumerate(outages):
            bp[c + 1] = bp[c] + len(rows)
        br = np.ascontiguousarray([k for rows in outages for k in rows] or [0], np.int64)
        sp = np.ascontiguousarray(scenario_ptr, np.int64)
        inj = np.ascontiguousarray(np.atleast_2d(injections), np.float64)
        total = int(sp[-1]) if sp.size else 0
        if inj.shape != (total, self.n_bus):
            raise ValueError("one injection vector over the buses per scenario")
        theta = np.zeros((total, self.n_bus))
        flows = np.zeros((total, self.n_branch))
        flags = np.zeros(max(total, 1), np.int32)
        sing = np.zeros(max(cases, 1), np.int32)
        _check(lib().yb_dc_outage_solutions(self._h, cases, ptr(bp), ptr(br), ptr(sp), ptr(inj), ptr(theta), ptr(flows),
                                            ptr(flags), ptr(sing)))
        return theta, flows, flags[:total], sing[:cases].astype(bool)

    def solve_branch_outages(self, injection, branches):
        """`DcGpuStudy::solve_branch_outages`: each branch taken out alone under one injection
        vector over the buses. Returns (theta, flows, flags) per branch and singular per branch."""
        branches = [int(k) for k in branches]
        inj = np.repeat(np.ascontiguousarray(injection, np.float64)[None, :], len(branches), axis=0)
        return self.outage_solutions([[k] for k in branches], np.arange(len(branches) + 1), inj)


class FlowLoss:
    """The adjoint of Σ softplus(|f| − margin·limit)² over a DC network's flows f = diag(b) A θ,
    θ = B′⁻¹ p: `forward(p, limits)` gives the loss (and optionally the flows) and keeps θ and
    dL/df on the device; `backward()` gives dL/dp (per scenario and bus, 0 at the slack) and dL/db
    (per branch, b = 1/x) from one transposed solve with the same factor."""

    def __init__(self, net: DcNetwork, count: int):
        self.net = net
        self.count = int(count)
        out = C.c_void_p()
        _check(lib().yb_dc_adjoint_new(net._h, self.count, C.byref(out)))
        self._h = out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().yb_dc_adjoint_free(h)
            except Exception:
                pass
            self._h = None

    def forward(self, injections, limits, margin: float = 0.8, flows: bool = False):
        p = np.ascontiguousarray(injections, np.float64)
        if p.shape != (self.count, self.net.n_bus):
            raise ValueError("one injection vector over the buses per scenario")
        lim = np.ascontiguousarray(limits, np.float64)
        loss = C.c_double()
        f = np.zeros((self.count, self.net.n_branch)) if flows else None
        _check(lib().yb_dc_adjoint_forward(self._h, ptr(p), ptr(lim), float(margin), C.byref(loss), ptr(f)))
        return (loss.value, f) if flows else loss.value

    def backward(self, grad_injections=None, grad_susceptance=None):
        """(dL/dp, dL/db); either may be given as a caller's float64 array of the right shape
        (pinned host memory, for instance) to receive it."""
        gp = np.zeros((self.count, self.net.n_bus)) if grad_injections is None else grad_injections
        gb = np.zeros(self.net.n_branch) if grad_susceptance is None else grad_susceptance
        if gp.shape != (self.count, self.net.n_bus) or gp.dtype != np.float64 or not gp.flags.c_contiguous:
            raise ValueError("dL/dp is a contiguous float64 (count, n_bus) array")
        if gb.shape != (self.net.n_branch,) or gb.dtype != np.float64:
            raise ValueError("dL/db is a float64 array over the branches")
        _check(lib().yb_dc_adjoint_backward(self._h, ptr(gp), ptr(gb)))
        return gp, gb
