#!/usr/bin/env python
"""Benchmark: the full PTDF block of the 10,000-bus synthetic grid, solved on the GPU.

Workload (synthetic, seeded): 10,000 buses uniform in the unit square, a random spanning tree of
the k=4 nearest-neighbour graph plus 3,500 further neighbour edges (13,499 branches), reactance
log-uniform in [0.005, 0.5]; B' (9,999 x 9,999) factored once by AMD-ordered Cholesky on the host.
A step solves all 13,499 branch right-hand sides A'diag(1/x)e_k (restricted to the non-slack buses)
with that factor. The right-hand sides (1.08 GB) are larger than L2, so no flush is needed.

Our arm times, on the device with CUDA events, K steps of the solve with inputs resident in HBM
(`value`), and separately the same solve through the host-array C ABI call with pinned host
buffers, copies included (`e2e`). `--impl reference` times the reference's CPU solve path (the
oracle's restatement of ybus_sparse's `par_solve_many`) on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RHS solved/s @1e-10 resid, 10k buses: batched FP32+IR vs FP64 GPU; HBM GB/s"
UNIT = "RHS/s"
WORKLOAD = "10k-bus PTDF block: B' 9,999 x 9,999 AMD Cholesky, 13,499 branch RHS"
N_BUS, EXTRA = 10000, 3500
FALLBACK_HBM_GBS = 6650.0
IR_TOLERANCE, IR_MAX_STEPS = 1e-10, 3
LANE_MIN_COUNT, LANE_AUTO_SLOTS = 3072, 64
LANE_REFINE_MIN_COUNT = 5120  # the refined solve's own threshold for the lane solve  # the library's automatic choice of the lane solve


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default="auto", choices=["auto", "fp64", "fp32_ir"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--rhs", type=int, default=0, help="solve only the first RHS (a smaller case for profiling)")
    p.add_argument("--workload", default="ptdf", choices=["ptdf", "n1", "adjoint", "complex"],
                   help="ptdf: the headline PTDF block; n1, adjoint, complex: the N-1 screening batch, the flow-loss "
                        "adjoint and the complex multi-network batch, each timed on its own (one GPU)")
    return p.parse_args()


def workload():
    from ybus_b200 import grids, host
    g = grids.make_grid(N_BUS, EXTRA, grids.SEED_BASE + 2)
    r, c, v = grids.bbus_triplets(g)
    keep = np.arange(1, N_BUS)
    bp = host.Matrix.from_triplets(N_BUS, N_BUS, r, c, v).select(keep, keep)
    chol = host.cholesky(bp)
    rhs = np.zeros((g.n_branch, N_BUS))
    k = np.arange(g.n_branch)
    rhs[k, g.frm] += g.susceptance
    rhs[k, g.to] -= g.susceptance
    rhs = np.ascontiguousarray(rhs[:, 1:])
    return g, bp, chol, rhs


def measured_peak():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(n: int, count: int, info: dict, mode: str, steps: float = 0.0, a_nnz: int = 0) -> int:
    """The per-launch byte model of the solve path (per RHS, plus the factor once):
    FP64: read b (8n), write and read the intermediate y (16n), write x (8n): 32 n.
    FP32 + m refinement steps: 24 n for the first solve, 48 n per step (residual reads x and b and
    writes r, the substitution writes and reads y, the update reads d and reads and writes x),
    plus the FP64 matrix once. The factor: values and int32 indices of both sweeps, row pointers."""
    entries = info["fwd_entries"] + info["bwd_entries"]
    if mode == "fp64":
        return int(count * 32 * n + entries * 12 + 8 * (n + 1))
    a_bytes = a_nnz * 12 + 4 * (n + 1)
    return int(count * (24 * n + steps * 48 * n) + entries * 8 + 8 * (n + 1) + a_bytes)


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one lane_solve_kernel<double> launch on
# the 10,000-bus block of 13,499 right-hand sides, from one ncu capture of this kernel (2.176 GB read,
# 2.115 GB written); other kernels and workloads report none
LANE_FP64_TRAFFIC = {(9999, 13499): 4.290592e9}


def traffic_of(result: dict, count: int, n: int):
    if result.get("kernel") == "lane_solve_kernel<double>":
        return LANE_FP64_TRAFFIC.get((n, count))
    return None


def cpu_baseline(chol, rhs, seconds_target: float = 10.0) -> dict:
    from oracle import oracle as orc
    cores = os.cpu_count() or 1
    # bounded sample: enough RHS for ~1-3 s per pass on all cores
    sample = rhs[: min(rhs.shape[0], 13499)]
    orc.solve_many(chol, sample[:256], threads=cores)  # warm-up
    times = []
    t_total = 0.0
    while len(times) < 5 and t_total < seconds_target:
        t0 = time.perf_counter()
        orc.solve_many(chol, sample, threads=cores)
        dt = time.perf_counter() - t0
        times.append(dt)
        t_total += dt
    med = statistics.median(times)
    return {"value": sample.shape[0] / med, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{sample.shape[0]} PTDF RHS of the 10k-bus B' factor, median of {len(times)} passes, "
                      f"oracle par_solve_many on {cores} threads"}


def run_reference(a):
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    g, bp, chol, rhs = workload()
    from oracle import oracle as orc
    cores = os.cpu_count() or 1
    for _ in range(a.warmup):
        orc.solve_many(chol, rhs[:512], threads=cores)
    per_step = min(rhs.shape[0], 13499)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        orc.solve_many(chol, rhs[:per_step], threads=cores)
    dt = time.perf_counter() - t0
    value = per_step * a.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rhs_per_step": per_step, "n": chol.n, "flush": "inputs > L2"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{per_step} PTDF RHS per step, oracle par_solve_many (restating "
                                       f"ybus_sparse factorization.rs:71-92) on {cores} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_workload(a) -> int:
    """The other workloads of the solve path, one GPU, one JSON line each: the N-1 screening batch
    (10,000-bus grid, 2,000 non-bridge outages with U[1, 64] injection scenarios each), the
    flow-loss adjoint (1,024 scenarios, forward and backward), and the complex multi-network batch
    (16 Ybus networks of 500 to 70,000 buses, 128 right-hand sides each, complex128 and complex64
    with complex128 refinement). Pinned host arrays in and out for the first two (their API takes
    host arrays, so the copies are inside the time); device arrays for the third."""
    import torch

    from ybus_b200 import FP32, FP64, Gpu, GpuFactor, grids, host, solve_batch_complex
    from ybus_b200.dc import DcNetwork, FlowLoss

    if int(os.environ.get("WORLD_SIZE", 1)) > 1:
        if int(os.environ.get("RANK", 0)) == 0:
            print(json.dumps({"workload": a.workload, "unavailable": "the extra workloads run on one GPU"}))
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    gpu = Gpu.new(int(os.environ.get("LOCAL_RANK", 0)))
    steps, warm = max(a.steps, 1), max(a.warmup, 1)
    line = {"workload": a.workload, "n_gpus": 1, "steps": steps, "warmup": warm, "data": "synthetic"}

    def wall(fn):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", 0))).start()
        t0 = time.perf_counter()
        for _ in range(steps):
            out = fn()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / steps
        return dt, out, clocks.stop()

    if a.workload == "n1":
        g = grids.make_grid(N_BUS, EXTRA, grids.SEED_BASE + 2)
        net = DcNetwork.from_grid(gpu, g)
        rng = np.random.default_rng(grids.SEED_BASE + 3)
        outaged = rng.choice(np.flatnonzero(~net.bridges()), 2000, replace=False)
        counts = rng.integers(1, 65, outaged.size)
        sp = np.concatenate([[0], np.cumsum(counts)])
        inj = rng.normal(0.0, 0.1, (int(sp[-1]), g.n_bus))
        inj[:, 0] = -inj[:, 1:].sum(axis=1)
        inj = torch.from_numpy(inj).pin_memory().numpy()  # pinned, as the headline's e2e
        weights = 1.0 / rng.uniform(0.5, 2.0, g.n_branch)
        modes = {}
        for name, prec in (("fp64", FP64), ("fp32_ir", FP32)):
            dt, (rows, vals, bad, sing), ck = wall(lambda: net.outage_loadings_batch(outaged, sp, inj, weights, prec))
            modes[name] = {"scenarios_s": sp[-1] / dt, "ms_per_step": dt * 1e3, "not_finite": int(bad.sum()),
                           "singular": int(sing.sum()), "clocks": ck}
        best = max(modes, key=lambda m: modes[m]["scenarios_s"])
        line.update({"metric": "N-1 scenarios screened/s (largest loading per scenario), pinned host arrays in and out",
                     "value": modes[best]["scenarios_s"], "unit": "scenarios/s", "higher_is_better": True,
                     "config": {"n_bus": N_BUS, "outages": int(outaged.size), "scenarios": int(sp[-1]),
                                "h2d_bytes_per_step": int(inj.nbytes), "mode": best}, "modes": modes})
    elif a.workload == "adjoint":
        g = grids.make_grid(N_BUS, EXTRA, grids.SEED_BASE + 2)
        net = DcNetwork.from_grid(gpu, g)
        rng = np.random.default_rng(grids.SEED_BASE + 4)
        count = 1024
        p = rng.normal(0.0, 0.1, (count, g.n_bus))
        p[:, 0] = -p[:, 1:].sum(axis=1)
        p = torch.from_numpy(p).pin_memory().numpy()  # pinned host arrays in and out
        gp_out = torch.zeros((count, g.n_bus), dtype=torch.float64).pin_memory().numpy()
        limits = rng.uniform(0.5, 2.0, g.n_branch)
        loss_fn = FlowLoss(net, count)

        def step():
            loss = loss_fn.forward(p, limits)
            return loss, loss_fn.backward(gp_out)
        dt, (loss, (gp, gb)), ck = wall(step)
        line.update({"metric": "flow-loss forward + backward scenarios/s (dL/dp and dL/db), pinned host arrays in and out",
                     "value": count / dt, "unit": "scenarios/s", "higher_is_better": True, "ms_per_step": dt * 1e3,
                     "config": {"n_bus": N_BUS, "scenarios": count, "loss": loss,
                                "finite": bool(np.isfinite(gp).all() and np.isfinite(gb).all())}, "clocks": ck})
    else:
        rng = np.random.default_rng(grids.SEED_BASE + 5)
        sizes = np.sort(np.exp(rng.uniform(np.log(500), np.log(70000), 16)).astype(int))[::-1]
        factors, bs, xs, rs = [], [], [], []
        for i, n_bus in enumerate(sizes):
            gc = grids.make_complex_grid(int(n_bus), grids.SEED_BASE + 60 + i)
            r, c, v = grids.ybus_triplets(gc)
            m = host.Matrix.from_triplets(int(n_bus), int(n_bus), r, c, v, by_rows=False)
            f = GpuFactor.from_lu_complex(gpu, host.lu(m, host.COLAMD))
            f.attach_matrix_complex(m)
            factors.append(f)
            b = rng.standard_normal((128, int(n_bus))) + 1j * rng.standard_normal((128, int(n_bus)))
            bs.append(torch.from_numpy(b.view(np.float64).copy()).cuda())
            xs.append(torch.empty_like(bs[-1]))
            rs.append(torch.empty(128, dtype=torch.float64, device="cuda"))
        total = 128 * len(sizes)
        modes = {}
        for name, prec in (("c128", FP64), ("c64_ir", FP32)):
            dt, st, ck = wall(lambda: solve_batch_complex(factors, [b.data_ptr() for b in bs],
                                                          [x.data_ptr() for x in xs], [128] * len(sizes), prec,
                                                          3, 1e-10, [r.data_ptr() for r in rs]))
            worst = max(float(r.max()) for r in rs) if prec == FP32 else None
            modes[name] = {"rhs_s": total / dt, "ms_per_step": dt * 1e3, "corrections": st,
                           "max_rel_residual": worst, "clocks": ck}
        passing = [m for m in modes if m == "c128" or (modes[m]["max_rel_residual"] or 1) <= 1e-10]
        best = max(passing, key=lambda m: modes[m]["rhs_s"])
        line.update({"metric": "complex RHS solved/s over a 16-network Ybus batch, one launch",
                     "value": modes[best]["rhs_s"], "unit": "RHS/s", "higher_is_better": True,
                     "config": {"networks": [int(v) for v in sizes], "rhs_per_network": 128, "mode": best},
                     "modes": modes})
    print(json.dumps(line), flush=True)
    return 0


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload != "ptdf":
        return run_workload(a)
    import torch
    import torch.distributed as dist

    from ybus_b200 import FP32, FP64, Gpu, GpuFactor, replicas

    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    g, bp, chol, rhs = workload()
    if a.rhs > 0:
        rhs = np.ascontiguousarray(rhs[: a.rhs])
    n, count = chol.n, rhs.shape[0]
    gpu = Gpu.new(local)
    factor = GpuFactor.from_cholesky(gpu, chol)
    info = factor.plan_info()
    factor.attach_matrix(bp)

    d_b = torch.from_numpy(rhs).cuda()
    d_x = torch.empty_like(d_b)
    d_ratio = torch.empty(count, dtype=torch.float64, device="cuda")
    d_steps = torch.empty(count, dtype=torch.int32, device="cuda")
    # A stream of our own: the current (legacy default) stream's handle is 0, which the C ABI
    # reads as the library's own stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream

    # each mode: one launch per step over the whole block
    runs = {
        "fp64": lambda: factor.solve_many_device(d_b.data_ptr(), d_x.data_ptr(), count, FP64, sh),
        "fp32_ir": lambda: factor.solve_many_refined_device(d_b.data_ptr(), d_x.data_ptr(), count, IR_MAX_STEPS,
                                                            IR_TOLERANCE, d_ratio.data_ptr(), d_steps.data_ptr(), sh),
    }
    modes = ["fp64", "fp32_ir"] if a.mode == "auto" else [a.mode]

    def timed(run, lane_timing=False):
        for _ in range(max(a.warmup, 3)):
            run()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        if lane_timing:  # events around each launch's gather, solve and scatter kernels
            factor.time_lane(True)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for e0, e1 in evs:
            e0.record(stream)
            run()
            e1.record(stream)
        end.record(stream)
        torch.cuda.synchronize()
        elapsed_ms = start.elapsed_time(end)
        launch_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in evs)
        kernels = None
        if lane_timing:
            t = factor.lane_times()
            factor.time_lane(False)
            k = max(t["launches"], 1)
            kernels = {"gather_ms": t["gather_ms"] / k, "solve_ms": t["solve_ms"] / k, "scatter_ms": t["scatter_ms"] / k,
                       "launches": t["launches"]}
        replicas.barrier()
        return replicas.max_over_ranks(elapsed_ms), launch_ms, kernels

    # which solve each mode runs: from the lane threshold on, the plain FP64 solve takes the lane
    # solve (three launches: gather, solve, scatter), and from its own higher threshold the refined
    # solve takes FP32 lane passes with an FP64 update and residual between them; below them, the
    # domain solve (the refined one with its refinement fused into one launch)
    lane = None
    try:
        lane = factor.lane_info(FP64)
    except Exception:
        pass
    use_lane = lane is not None and count >= LANE_MIN_COUNT and lane["slots"] <= LANE_AUTO_SLOTS

    lane32 = None
    try:
        lane32 = factor.lane_info(FP32)
    except Exception:
        pass
    use_lane32 = lane32 is not None and count >= LANE_REFINE_MIN_COUNT and lane32["slots"] <= LANE_AUTO_SLOTS

    def solver_of(mode):
        if mode == "fp64" and use_lane:
            return {"solver": "lane", "kernel": "lane_solve_kernel<double>", "launches_per_step": 3,
                    "lane": {k: lane[k] for k in ("warps", "slots", "domains", "top", "pages", "smem")}}
        if mode == "fp32_ir" and use_lane32:
            # an initialisation and two gathers, per pass a solve, an update, a residual and a
            # decision (passes after every group has stopped return at once), then the scatter
            return {"solver": "lane", "kernel": "lane_solve_kernel<float>", "launches_per_step": 4 + 4 * (IR_MAX_STEPS + 1),
                    "lane": {k: lane32[k] for k in ("warps", "slots", "domains", "top", "pages", "smem")}}
        prec = FP64 if mode == "fp64" else FP32
        return {"solver": "domain", "kernel": "domain_tile_kernel", "launches_per_step": 1,
                "tile": factor.domain_info(prec)["tile"]}

    from oracle import oracle as orc  # the checker, outside the timed regions
    p, i, v = bp.arrays()
    sample = np.arange(0, count, max(1, count // 64))
    cpu = orc.solve_many(chol, rhs[sample], threads=os.cpu_count() or 1)
    peak, peak_kind = measured_peak()
    clocks = ClockSampler(local).start()
    time.sleep(0.3)
    results = {}
    for mode in modes:
        on_lane = mode == "fp64" and use_lane
        elapsed_ms, launch_ms, kernels = timed(runs[mode], lane_timing=on_lane)
        # check the timed results: relative residual of every 13th column, the oracle on a sample
        xs = d_x.cpu().numpy()
        resid = max(orc.relative_residual(p, i, v, xs[k], rhs[k]) for k in range(0, count, 13))
        err = float(max(np.abs(xs[k] - c).max() / np.abs(c).max() for k, c in zip(sample, cpu)))
        r = {"rhs_s": world * count * a.steps / (elapsed_ms / 1e3), "ms_per_step": elapsed_ms / a.steps,
             "launch_ms": launch_ms, "max_rel_residual": resid, "max_rel_err_vs_oracle": err}
        if mode == "fp32_ir":
            ratios, steps = d_ratio.cpu().numpy(), d_steps.cpu().numpy()
            r.update({"device_max_ratio": float(ratios.max()), "mean_corrections": float(steps.mean()),
                      "max_corrections": int(steps.max()), "tolerance": IR_TOLERANCE, "max_steps": IR_MAX_STEPS})
            r["algorithmic_bytes_per_launch"] = algorithmic_bytes(n, count, info, "fp32_ir", float(steps.mean()), len(i))
        else:
            r["algorithmic_bytes_per_launch"] = algorithmic_bytes(n, count, info, "fp64")
        r.update(solver_of(mode))
        # the dominant kernel's own launch time: the lane solve kernel (events around it in every
        # launch), else the one launch of the step
        r["kernel_ms"] = launch_ms
        if kernels:
            r["kernels"] = kernels
            r["kernel_ms"] = kernels["solve_ms"]
            io_bytes = count * 16 * n  # each of the gather and the scatter reads and writes 8 n per RHS
            r["kernels"]["gather_gbs"] = io_bytes / (kernels["gather_ms"] / 1e3) / 1e9
            r["kernels"]["scatter_gbs"] = io_bytes / (kernels["scatter_ms"] / 1e3) / 1e9
        results[mode] = r
    clock_info = clocks.stop()

    # the headline: the fastest mode whose every checked column meets the 1e-10 relative residual
    passing = [m for m in modes if results[m]["max_rel_residual"] <= 1e-10]
    mode = max(passing, key=lambda m: results[m]["rhs_s"]) if passing else modes[0]
    best = results[mode]
    achieved = best["algorithmic_bytes_per_launch"] / (best["kernel_ms"] / 1e3) / 1e9
    compulsory = count * 16 * n / (best["launch_ms"] / 1e3) / 1e9
    if "fp64" in results and "fp32_ir" in results:
        results["fp32_ir_over_fp64"] = results["fp32_ir"]["rhs_s"] / results["fp64"]["rhs_s"]

    line = {"metric": METRIC, "value": best["rhs_s"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": best["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if mode == "fp64" else "f32 substitution, f64 refinement",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "rhs_per_step": count, "n": n, "mode": mode,
                       "nnz_factor_per_sweep": info["fwd_entries"] + n, "levels": [info["fwd_levels"], info["bwd_levels"]],
                       "solver": best["solver"], "flush": "inputs (1.08 GB) > L2", "parallelism": f"replicas x{world}"},
            "accuracy": {"max_rel_residual": best["max_rel_residual"], "max_rel_err_vs_oracle": best["max_rel_err_vs_oracle"]},
            "modes": results,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_of(best, count, n), "peak_source": peak_kind, "kernel": best["kernel"],
                         "algorithmic_bytes_per_launch": best["algorithmic_bytes_per_launch"],
                         "kernel_ms": best["kernel_ms"], "launch_ms": best["launch_ms"], "compulsory_gbs": compulsory,
                         "compulsory_frac": compulsory / peak},
            "clocks": clock_info, "gpu_launches": a.steps * sum(results[m]["launches_per_step"] for m in modes)}

    if not a.no_e2e:
        # every rank through the host-array call on its own GPU; the step time is the max over ranks
        b_pin = torch.from_numpy(rhs).pin_memory()
        x_pin = torch.empty_like(b_pin).pin_memory()
        bn, xn = b_pin.numpy(), x_pin.numpy()
        factor.set_block_width(count)
        for _ in range(max(a.warmup, 1)):
            factor.solve_many_into(bn, xn)
        reps = max(3, min(a.steps, 10))
        factor.reset_timings()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            factor.solve_many_into(bn, xn)
        dt = replicas.max_over_ranks(time.perf_counter() - t0)
        t = factor.timings()
        e2e_err = float(max(np.abs(xn[k] - c).max() / np.abs(c).max() for k, c in zip(sample, cpu)))
        line["e2e"] = {"value": world * count * reps / dt, "unit": UNIT, "h2d_bytes_per_step": int(rhs.nbytes),
                       "d2h_bytes_per_step": int(rhs.nbytes), "ms_per_step": dt / reps * 1e3,
                       "api": "yb_solve_many (pinned host arrays, chunks overlapped over both copy engines)",
                       "max_rel_err_vs_oracle": e2e_err, "chunks_per_step": t.blocks // reps,
                       "stage_ms_per_step": {"upload": t.upload / reps * 1e3, "solve": t.solve / reps * 1e3,
                                             "download": t.download / reps * 1e3}}
    if world == 1 and not a.no_e2e:
        # for comparison: ybus_cuda's own route to the solve (cuSPARSE SpSM, lower then upper, in
        # blocks), on the same factor and device arrays; its best block width of 64, 256 and 1024
        spsm = {}
        for width in (64, 256, 1024):
            factor.reference_spsm_solve_device(d_b.data_ptr(), d_x.data_ptr(), count, width)
            spsm[width] = factor.reference_spsm_solve_device(d_b.data_ptr(), d_x.data_ptr(), count, width)
        width = min(spsm, key=spsm.get)
        line["reference_gpu_spsm"] = {"value": count / (spsm[width] / 1e3), "unit": UNIT, "ms_per_step": spsm[width],
                                      "width": width, "ms_by_width": spsm,
                                      "route": "cuSPARSE SpSM lower + upper on CSR triangles (ybus_cuda's Block::solve)"}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(chol, rhs)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
