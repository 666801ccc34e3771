#!/usr/bin/env python
"""Benchmark of the factor-once / solve-many path on the synthetic 10,000-bus grid.

Headline workload (seeded; ybus_b200/configs.py): 10,000 buses uniform in the unit square, a random
spanning tree of the k=4 nearest-neighbour graph plus 3,500 further neighbour edges (13,499
branches), reactance log-uniform in [0.005, 0.5]; B' (9,999 x 9,999) factored once by AMD-ordered
Cholesky on the host. A step solves all 13,499 branch right-hand sides A'diag(1/x)e_k (restricted
to the non-slack buses) with that factor; on N GPUs the columns are split over the ranks. The
right-hand sides (1.08 GB) are larger than L2, so no flush is needed.

Our arm times, on the device with CUDA events, K steps of the solve with inputs resident in HBM
(`value`: FP64, and FP32 substitution with FP64 refinement to 1e-10, the faster passing mode as the
headline), the same block in blocks of 64, 256 and 1,024 columns (`modes_by_width`), the solve
through the host-array C ABI call with pinned host buffers, copies included (`e2e`), and the
other configurations of the path (`workloads`: the N-1 screening batch, the flow-loss adjoint, the
complex multi-network batch, the Newton-Raphson Jacobian's LU solve). `--impl reference` times the reference's CPU solve path (the
oracle's restatement of ybus_sparse's `par_solve_many`) on all host cores, loading no GPU library.
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
FALLBACK_HBM_GBS = 6650.0
IR_TOLERANCE, IR_MAX_STEPS = 1e-10, 3
WIDTHS = (64, 256, 1024)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default="auto", choices=["auto", "fp64", "fp32_ir"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="time the headline modes only (no block widths, workloads or comparison): for profiling")
    p.add_argument("--rhs", type=int, default=0, help="solve only the first RHS (a smaller case for profiling)")
    p.add_argument("--lane-warps", type=int, default=0,
                   help="jacobian: the lane solve at this many warps per block instead of the autotuner's pick "
                        "(a fixed kernel for profiling)")
    p.add_argument("--workload", default="ptdf", choices=["ptdf", "n1", "adjoint", "complex", "jacobian"],
                   help="ptdf: the headline PTDF block with the other workloads as extra keys; n1, adjoint, complex, jacobian: "
                        "one of the other workloads alone, one JSON line")
    return p.parse_args()


def headline_config(count: int, n: int, world: int) -> dict:
    """The workload's description, the same for both arms."""
    return {"workload": WORKLOAD, "rhs_per_step": count, "n": n, "flush": "inputs (1.08 GB) > L2",
            "parallelism": f"RHS columns split over {world} GPU(s)"}


def workload():
    from ybus_b200 import configs, host
    g = configs.grid_10k()
    bp = configs.bprime(g)
    chol = host.cholesky(bp)
    return g, bp, chol, configs.branch_rhs(g)


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


def _time_oracle(chol, rhs, threads: int, passes: int, seconds: float) -> tuple[float, int]:
    """Median seconds of `passes` oracle solves of `rhs` on `threads` threads (fewer if the time
    budget runs out), after one warm-up on a slice."""
    from oracle import oracle as orc
    orc.solve_many(chol, rhs[: min(64, rhs.shape[0])], threads=threads)
    times, total = [], 0.0
    while len(times) < passes and total < seconds:
        t0 = time.perf_counter()
        orc.solve_many(chol, rhs, threads=threads)
        times.append(time.perf_counter() - t0)
        total += times[-1]
    return statistics.median(times), len(times)


def cpu_baseline(chol, rhs) -> dict:
    """The oracle's par_solve_many on every host core (13,499 RHS, median of up to 5 passes) and on
    one thread (a 1,000-RHS sample, median of up to 3 passes)."""
    cores = os.cpu_count() or 1
    med, passes = _time_oracle(chol, rhs, cores, 5, 10.0)
    one = rhs[:1000]
    med1, passes1 = _time_oracle(chol, one, 1, 3, 10.0)
    return {"value": rhs.shape[0] / med, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{rhs.shape[0]} PTDF RHS of the 10k-bus B' factor, median of {passes} passes, oracle "
                      f"par_solve_many on {cores} threads",
            "value_1thread": one.shape[0] / med1,
            "sample_1thread": f"the first {one.shape[0]} of those RHS, median of {passes1} passes on 1 thread"}


def run_reference(a):
    """The reference's CPU path: the oracle's restatement of ybus_sparse's par_solve_many on every
    host core, on the factor the host producer (libybhost.so alone) makes. Rank 0 only."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    g, bp, chol, rhs = workload()
    from oracle import oracle as orc
    cores = os.cpu_count() or 1
    if a.rhs > 0:
        rhs = np.ascontiguousarray(rhs[: a.rhs])
    for _ in range(max(a.warmup, 1)):
        orc.solve_many(chol, rhs[:512], threads=cores)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        orc.solve_many(chol, rhs, threads=cores)
    dt = time.perf_counter() - t0
    value = rhs.shape[0] * a.steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": dt / a.steps * 1e3, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(rhs.shape[0], chol.n, a.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{rhs.shape[0]} PTDF RHS per step, oracle par_solve_many (restating "
                                       f"ybus_sparse factorization.rs:71-92) on {cores} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    maps = Path("/proc/self/maps")
    if maps.exists():
        text = maps.read_text()
        line["native_libraries"] = sorted({n for n in ("libybhost.so", "libybgpu.so", "liboracle.so") if n in text})
    print(json.dumps(line), flush=True)
    return 0


# ---- the other workloads of the path ------------------------------------------------------------

def _timed_wall(fn, steps: int, warm: int, device: int):
    """Wall time per step of `fn` (it synchronises before returning: its API takes host arrays),
    the max over ranks, with the clocks sampled meanwhile."""
    import torch

    from ybus_b200 import replicas
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    replicas.barrier()
    clocks = ClockSampler(device).start()
    t0 = time.perf_counter()
    for _ in range(steps):
        out = fn()
    torch.cuda.synchronize()
    dt = replicas.max_over_ranks((time.perf_counter() - t0) / steps)
    return dt, out, clocks.stop()


def workload_n1(gpu, steps: int, warm: int, rank: int, world: int, device: int) -> dict:
    """Configuration 3: 2,000 non-bridge outages of the 10,000-bus grid with U[1, 64] injection
    scenarios each, screened for their largest loading in one captured launch per rank (cases split
    over the ranks by LPT on their scenario counts), pinned host arrays in and out."""
    import torch

    from ybus_b200 import FP32, FP64, configs, replicas
    from ybus_b200.dc import DcNetwork
    g = configs.grid_10k()
    net = DcNetwork.from_grid(gpu, g)
    cases = configs.n1_cases(g, net.bridges())
    counts = np.diff(cases.scenario_ptr)
    mine = replicas.lpt(counts + 1, world)[rank]
    sp = np.concatenate([[0], np.cumsum(counts[mine])]).astype(np.int64)
    cols = np.concatenate([np.arange(cases.scenario_ptr[c], cases.scenario_ptr[c + 1]) for c in mine])
    inj = torch.from_numpy(np.ascontiguousarray(cases.injections[cols])).pin_memory().numpy()
    outaged = cases.outaged[mine]
    modes = {}
    for name, prec in (("fp64", FP64), ("fp32_ir", FP32)):
        dt, (rows, vals, bad, sing), ck = _timed_wall(
            lambda: net.outage_loadings_batch(outaged, sp, inj, cases.weights, prec), steps, warm, device)
        modes[name] = {"scenarios_s": int(cases.scenario_ptr[-1]) / dt, "ms_per_step": dt * 1e3,
                       "not_finite": int(((bad & 1) != 0).sum()), "suspect_angles": int(((bad & 2) != 0).sum()),
                       "singular": int(sing.sum()), "clocks": ck}
    best = max(modes, key=lambda m: modes[m]["scenarios_s"])
    return {"metric": "N-1 scenarios screened/s (largest loading per scenario), pinned host arrays in and out",
            "value": modes[best]["scenarios_s"], "unit": "scenarios/s", "higher_is_better": True,
            "config": {"n_bus": configs.N_BUS, "outages": int(cases.outaged.size),
                       "scenarios": int(cases.scenario_ptr[-1]), "h2d_bytes_per_step": int(inj.nbytes),
                       "mode": best, "split": f"cases by LPT over {world} GPU(s)"}, "modes": modes}


def workload_adjoint(gpu, steps: int, warm: int, rank: int, world: int, device: int) -> dict:
    """Configuration 4: the flow-loss forward and backward over 1,024 scenarios of the 10,000-bus
    grid (dL/dp and dL/db), pinned host arrays in and out; on N GPUs the scenarios are split and
    dL/db and the loss are summed over the ranks in rank order."""
    import torch

    from ybus_b200 import configs, replicas
    from ybus_b200.dc import DcNetwork, FlowLoss
    g = configs.grid_10k()
    net = DcNetwork.from_grid(gpu, g)
    p, limits = configs.adjoint_scenarios(g)
    share = replicas.shard(p.shape[0], rank, world)
    pm = torch.from_numpy(np.ascontiguousarray(p[share.start:share.stop])).pin_memory().numpy()
    gp_out = torch.zeros(pm.shape, dtype=torch.float64).pin_memory().numpy()
    gb_out = np.zeros(g.n_branch)
    loss_fn = FlowLoss(net, pm.shape[0])

    def step():
        loss = loss_fn.forward(pm, limits)
        gp, gb = loss_fn.backward(gp_out, gb_out)
        total = replicas.sum_in_rank_order(np.append(gb, loss))
        return total[-1], gp, total[:-1]

    dt, (loss, gp, gb), ck = _timed_wall(step, steps, warm, device)
    return {"metric": "flow-loss forward + backward scenarios/s (dL/dp and dL/db), pinned host arrays in and out",
            "value": p.shape[0] / dt, "unit": "scenarios/s", "higher_is_better": True, "ms_per_step": dt * 1e3,
            "config": {"n_bus": configs.N_BUS, "scenarios": int(p.shape[0]), "loss": float(loss),
                       "finite": bool(np.isfinite(gp).all() and np.isfinite(gb).all()),
                       "split": f"scenarios over {world} GPU(s), dL/db summed in rank order"}, "clocks": ck}


def workload_complex(gpu, steps: int, warm: int, rank: int, world: int, device: int) -> dict:
    """Configuration 5: 16 complex Ybus networks of 500 to 70,000 buses, 128 right-hand sides each,
    in one launch per rank (networks split over the ranks by LPT on factor entries x right-hand
    sides), device arrays, complex128 and complex64 with complex128 refinement."""
    import torch

    from ybus_b200 import FP32, FP64, GpuFactor, configs, replicas, solve_batch_complex
    sizes = configs.complex_sizes()
    nets = [configs.complex_network(int(n), i) for i, n in enumerate(sizes)]
    work = [(net.lu.l.idx.size + net.lu.u.idx.size) * net.rhs.shape[0] for net in nets]
    mine = replicas.lpt(work, world)[rank]
    factors, bs, xs, rs = [], [], [], []
    for i in mine:
        net = nets[i]
        f = GpuFactor.from_lu_complex(gpu, net.lu)
        f.attach_matrix_complex(net.ybus)
        factors.append(f)
        bs.append(torch.from_numpy(net.rhs.view(np.float64).copy()).cuda())
        xs.append(torch.empty_like(bs[-1]))
        rs.append(torch.empty(net.rhs.shape[0], dtype=torch.float64, device="cuda"))
    total = sum(net.rhs.shape[0] for net in nets)
    modes = {}
    for name, prec in (("c128", FP64), ("c64_ir", FP32)):
        def run():
            st = solve_batch_complex(factors, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs],
                                     [nets[i].rhs.shape[0] for i in mine], prec, 3, 1e-10, [r.data_ptr() for r in rs])
            torch.cuda.synchronize()
            return st
        dt, st, ck = _timed_wall(run, steps, warm, device)
        worst = replicas.max_over_ranks(max((float(r.max()) for r in rs), default=0.0))
        modes[name] = {"rhs_s": total / dt, "ms_per_step": dt * 1e3, "corrections": st, "max_rel_residual": worst,
                       "clocks": ck}
    passing = [m for m in modes if modes[m]["max_rel_residual"] <= 1e-10]
    best = max(passing or list(modes), key=lambda m: modes[m]["rhs_s"])
    return {"metric": "complex RHS solved/s over a 16-network Ybus batch, one launch",
            "value": modes[best]["rhs_s"], "unit": "RHS/s", "higher_is_better": True,
            "config": {"networks": [int(v) for v in sizes], "rhs_per_network": configs.COMPLEX_RHS, "mode": best,
                       "split": f"networks by LPT over {world} GPU(s)"}, "modes": modes}


def workload_jacobian(gpu, steps: int, warm: int, rank: int, world: int, device: int, lane_warps: int = 0) -> dict:
    """The Newton-Raphson Jacobian of the 10,000-bus complex network (order 17,998, AMD LU on the
    host; the reference's other matrix for its GPU survey): 4,096 right-hand sides, device arrays,
    FP64, split over the ranks by columns; the autotuner picks the solve, or `lane_warps` fixes the
    lane solve's blocks."""
    import torch

    from ybus_b200 import FP64, GpuFactor, configs, replicas
    sysj = configs.jacobian_system()
    mine = replicas.shard(sysj.rhs.shape[0], rank, world)
    rhs = np.ascontiguousarray(sysj.rhs[mine.start:mine.stop])
    factor = GpuFactor.from_lu(gpu, sysj.lu)
    if lane_warps:
        factor.set_tile_kind(FP64, 5)
        factor.set_lane(FP64, lane_warps)
        tuned = {"kind": 5, "tile": 0, "warps": lane_warps, "fixed": True}
    else:
        tuned = factor.autotune(FP64, rhs.shape[0])  # as a caller would, once per factor
    b = torch.from_numpy(rhs).cuda()
    x = torch.empty_like(b)
    # a stream of our own: the legacy default stream's handle is 0, which the C ABI reads as the
    # library's own stream, and the events must be on the stream the solves run on
    stream = torch.cuda.Stream()

    def run():
        factor.solve_many_device(b.data_ptr(), x.data_ptr(), rhs.shape[0], FP64, stream.cuda_stream)

    for _ in range(warm):
        run()
    torch.cuda.synchronize()
    replicas.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        run()
    e1.record(stream)
    torch.cuda.synchronize()
    factor.check_error()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1) / steps)
    return {"metric": "Newton-Raphson Jacobian RHS solved/s, device arrays", "value": sysj.rhs.shape[0] / (ms / 1e3),
            "unit": "RHS/s", "higher_is_better": True, "ms_per_step": ms,
            "config": {"n_bus": sysj.n_bus, "order": int(sysj.lu.n), "lu_entries": int(sysj.lu.l.idx.size + sysj.lu.u.idx.size),
                       "rhs": int(sysj.rhs.shape[0]), "split": f"columns over {world} GPU(s)",
                       "autotuned": {k: v for k, v in tuned.items() if k != "ms"}}}


WORKLOADS = {"n1": workload_n1, "adjoint": workload_adjoint, "complex": workload_complex, "jacobian": workload_jacobian}


def init_ranks():
    import datetime

    import torch
    import torch.distributed as dist

    from ybus_b200 import replicas
    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def run_workload(a) -> int:
    """One of the other workloads alone: one JSON line (rank 0)."""
    from ybus_b200 import Gpu
    rank, world, local = init_ranks()
    gpu = Gpu.new(local)
    line = {"workload": a.workload, "n_gpus": world, "steps": max(a.steps, 1), "warmup": max(a.warmup, 1),
            "data": "synthetic"}
    extra = {"lane_warps": a.lane_warps} if a.workload == "jacobian" and a.lane_warps else {}
    line.update(WORKLOADS[a.workload](gpu, max(a.steps, 1), max(a.warmup, 1), rank, world, local, **extra))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# ---- the headline ---------------------------------------------------------------------------------

def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload != "ptdf":
        return run_workload(a)
    import torch
    import torch.distributed as dist

    from ybus_b200 import FP32, FP64, Gpu, GpuFactor, replicas

    rank, world, local = init_ranks()
    g, bp, chol, rhs_all = workload()
    if a.rhs > 0:
        rhs_all = np.ascontiguousarray(rhs_all[: a.rhs])
    total = rhs_all.shape[0]
    mine = replicas.shard(total, rank, world)
    rhs = np.ascontiguousarray(rhs_all[mine.start:mine.stop])
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

    def solve(mode, cols=None, off=0):
        c = count if cols is None else cols
        b, x = d_b.data_ptr() + off * n * 8, d_x.data_ptr() + off * n * 8
        if mode == "fp64":
            factor.solve_many_device(b, x, c, FP64, sh)
        else:
            factor.solve_many_refined_device(b, x, c, IR_MAX_STEPS, IR_TOLERANCE, d_ratio.data_ptr() + off * 8,
                                             d_steps.data_ptr() + off * 4, sh)

    def blocks(mode, width):  # the block solved in blocks of `width` columns, one launch each
        for k0 in range(0, count, width):
            solve(mode, min(width, count - k0), k0)

    modes = ["fp64", "fp32_ir"] if a.mode == "auto" else [a.mode]

    def timed(run, lane_timing=False, steps=None):
        steps = a.steps if steps is None else steps
        for _ in range(max(a.warmup, 3)):
            run()
        torch.cuda.synchronize()
        replicas.barrier()
        torch.cuda.synchronize()
        if lane_timing:  # events around each launch's gather, solve and scatter kernels
            factor.time_lane(True)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
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

    # which solve each mode runs (the library's automatic choice, read back from its settings)
    lane = lane32 = None
    try:
        lane = factor.lane_info(FP64)
    except Exception:
        pass
    try:
        lane32 = factor.lane_info(FP32)
    except Exception:
        pass
    lane_min, refine_min = factor.lane_min_count(FP64), factor.refine_lane_min_count()
    use_lane = lane is not None and count >= lane_min and lane["slots"] <= 64
    use_lane32 = lane32 is not None and count >= max(refine_min, factor.lane_min_count(FP32)) and lane32["slots"] <= 64

    def solver_of(mode):
        if mode == "fp64" and use_lane:
            return {"solver": "lane", "kernel": "lane_solve_kernel<double>", "launches_per_step": 3,
                    "lane": {k: lane[k] for k in ("warps", "slots", "domains", "top", "pages", "smem")}}
        if mode == "fp32_ir" and use_lane32:
            # an initialisation and the gather, per pass a solve, a residual (the update folded
            # in), a decision and the restore of columns a pass made no better, and between passes
            # the FP64 carry of x (kernels of groups that have stopped return at once)
            return {"solver": "lane", "kernel": "lane_solve_kernel<float>",
                    "launches_per_step": 2 + 4 * (IR_MAX_STEPS + 1) + max(0, IR_MAX_STEPS - 1),
                    "lane": {k: lane32[k] for k in ("warps", "slots", "domains", "top", "pages", "smem")}}
        prec = FP64 if mode == "fp64" else FP32
        return {"solver": "domain", "kernel": "domain_tile_kernel", "launches_per_step": 1,
                "tile": factor.domain_info(prec)["tile"]}

    from oracle import oracle as orc  # the checker, outside the timed regions
    p, i, v = bp.arrays()
    sample = np.arange(0, count, max(1, count // 64))
    cpu = orc.solve_many(chol, rhs[sample], threads=os.cpu_count() or 1)
    peak, peak_kind = measured_peak()

    def check(mode, r):
        xs = d_x.cpu().numpy()
        r["max_rel_residual"] = max(orc.relative_residual(p, i, v, xs[k], rhs[k]) for k in range(0, count, 13))
        r["max_rel_err_vs_oracle"] = float(max(np.abs(xs[k] - c).max() / np.abs(c).max() for k, c in zip(sample, cpu)))
        if mode == "fp32_ir":
            ratios, steps = d_ratio.cpu().numpy(), d_steps.cpu().numpy()
            r.update({"device_max_ratio": float(ratios.max()), "mean_corrections": float(steps.mean()),
                      "max_corrections": int(steps.max()), "tolerance": IR_TOLERANCE, "max_steps": IR_MAX_STEPS})
        return r

    clocks = ClockSampler(local).start()
    time.sleep(0.3)
    results = {}
    for mode in modes:
        on_lane = mode == "fp64" and use_lane
        elapsed_ms, launch_ms, kernels = timed(lambda: solve(mode), lane_timing=on_lane)
        r = check(mode, {"rhs_s": total * a.steps / (elapsed_ms / 1e3), "ms_per_step": elapsed_ms / a.steps,
                         "launch_ms": launch_ms})
        steps_mean = r.get("mean_corrections", 0.0)
        r["algorithmic_bytes_per_launch"] = algorithmic_bytes(n, count, info, mode, steps_mean, len(i))
        r.update(solver_of(mode))
        # the dominant kernel's own launch time where the library records it (the lane solve), else
        # the step's launches
        r["kernel_ms"] = launch_ms
        if kernels:
            r["kernels"] = kernels
            r["kernel_ms"] = kernels["solve_ms"]
            io_bytes = count * 16 * n  # each of the gather and the scatter reads and writes 8 n per RHS
            r["kernels"]["gather_gbs"] = io_bytes / (kernels["gather_ms"] / 1e3) / 1e9
            r["kernels"]["scatter_gbs"] = io_bytes / (kernels["scatter_ms"] / 1e3) / 1e9
        # the mode's roofline over its whole step (every launch of it): the mode's algorithmic bytes
        # over the step's time, against the measured copy bandwidth
        step_gbs = r["algorithmic_bytes_per_launch"] / (launch_ms / 1e3) / 1e9
        r["step_roofline"] = {"achieved": step_gbs, "peak": peak, "unit": "GB/s", "frac": step_gbs / peak}
        results[mode] = r
    if "fp64" in results and "fp32_ir" in results:
        results["fp32_ir_over_fp64"] = results["fp32_ir"]["rhs_s"] / results["fp64"]["rhs_s"]

    # the same block in blocks of 64, 256 and 1,024 columns (configuration 2's block widths)
    by_width = {}
    if not a.no_extras:
        for width in WIDTHS:
            by_width[str(width)] = {}
            for mode in modes:
                steps_w = max(3, min(a.steps, 10))
                elapsed_ms, launch_ms, _ = timed(lambda: blocks(mode, width), steps=steps_w)
                r = check(mode, {"rhs_s": total * steps_w / (elapsed_ms / 1e3), "ms_per_step": elapsed_ms / steps_w,
                                 "launches_per_step": -(-count // width)})
                r["solver"] = solver_of(mode)["solver"] if width >= (lane_min if mode == "fp64" else refine_min) \
                    else "domain"
                by_width[str(width)][mode] = r
    clock_info = clocks.stop()

    # the headline: the fastest mode whose every checked column meets the 1e-10 relative residual
    passing = [m for m in modes if results[m]["max_rel_residual"] <= 1e-10]
    mode = max(passing, key=lambda m: results[m]["rhs_s"]) if passing else modes[0]
    best = results[mode]
    achieved = best["algorithmic_bytes_per_launch"] / (best["kernel_ms"] / 1e3) / 1e9
    compulsory = count * 16 * n / (best["launch_ms"] / 1e3) / 1e9
    launches = a.steps * sum(results[m]["launches_per_step"] for m in modes)
    launches += sum(max(3, min(a.steps, 10)) * r["launches_per_step"] for w in by_width.values() for r in w.values())

    line = {"metric": METRIC, "value": best["rhs_s"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": best["ms_per_step"], "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64" if mode == "fp64" else "f32 substitution, f64 refinement",
            "data": "synthetic", "config": headline_config(total, n, world),
            "mode": mode, "solver": best["solver"], "nnz_factor_per_sweep": info["fwd_entries"] + n,
            "levels": [info["fwd_levels"], info["bwd_levels"]],
            "accuracy": {"max_rel_residual": best["max_rel_residual"], "max_rel_err_vs_oracle": best["max_rel_err_vs_oracle"]},
            "modes": results, "modes_by_width": by_width,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic_of(best, count, n), "peak_source": peak_kind, "kernel": best["kernel"],
                         "algorithmic_bytes_per_launch": best["algorithmic_bytes_per_launch"],
                         "kernel_ms": best["kernel_ms"], "launch_ms": best["launch_ms"], "compulsory_gbs": compulsory,
                         "compulsory_frac": compulsory / peak},
            "clocks": clock_info, "gpu_launches": launches}

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
        replicas.barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            factor.solve_many_into(bn, xn)
        dt = replicas.max_over_ranks(time.perf_counter() - t0)
        t = factor.timings()
        e2e_err = float(max(np.abs(xn[k] - c).max() / np.abs(c).max() for k, c in zip(sample, cpu)))
        line["e2e"] = {"value": total * reps / dt, "unit": UNIT, "h2d_bytes_per_step": int(rhs.nbytes),
                       "d2h_bytes_per_step": int(rhs.nbytes), "ms_per_step": dt / reps * 1e3,
                       "api": "yb_solve_many (pinned host arrays, chunks overlapped over both copy engines)",
                       "max_rel_err_vs_oracle": e2e_err, "chunks_per_step": t.blocks // reps,
                       "stage_ms_per_step": {"upload": t.upload / reps * 1e3, "solve": t.solve / reps * 1e3,
                                             "download": t.download / reps * 1e3}}
    if world == 1 and not a.no_extras:
        # for comparison: ybus_cuda's own route to the solve (cuSPARSE SpSM, lower then upper, in
        # blocks; libybcompare.so), on the same factor and device arrays; its best block width
        from ybus_b200 import compare
        spsm = {}
        for width in WIDTHS:
            compare.spsm_solve(chol, d_b.data_ptr(), d_x.data_ptr(), count, width)
            spsm[width] = compare.spsm_solve(chol, d_b.data_ptr(), d_x.data_ptr(), count, width)
        width = min(spsm, key=spsm.get)
        line["reference_gpu_spsm"] = {"value": count / (spsm[width] / 1e3), "unit": UNIT, "ms_per_step": spsm[width],
                                      "width": width, "ms_by_width": spsm,
                                      "route": "cuSPARSE SpSM lower + upper on CSR triangles (ybus_cuda's Block::solve)"}
    if not a.no_extras:
        steps_w, warm_w = max(3, min(a.steps, 5)), max(1, min(a.warmup, 2))
        line["workloads"] = {name: fn(gpu, steps_w, warm_w, rank, world, local) for name, fn in WORKLOADS.items()}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(chol, rhs)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
