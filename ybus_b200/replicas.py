"""One process per GPU for the solve path, which shards with no data-path exchange: right-hand
sides, outage cases and networks are independent, so every rank solves its own share on its own GPU
and the processes meet only to start timing together and to take the slowest rank's time. The one
exchange is the adjoint's: the gradient with respect to the branch susceptances is a sum over
scenarios, so ranks that split the scenarios add their partial sums (in rank order, so the result
does not depend on timing). These helpers hold that logic apart from the GPU so that it runs (and
is tested) on any torch.distributed backend, gloo on the CPU included."""
from __future__ import annotations

import os

import torch
import torch.distributed as dist


def rank_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment (1 process when unset)."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def _device() -> torch.device:
    return torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier() -> None:
    """All ranks meet (a no-op for one process)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(value: float) -> float:
    """The largest of every rank's `value` (its own for one process): a step's time is the slowest
    rank's."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(units: int, rank: int, world: int) -> range:
    """Rank `rank`'s contiguous share of `units` independent units, the shares differing by at most
    one and covering every unit once."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank outside the world")
    base, extra = divmod(int(units), world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def lpt(weights, world: int) -> list[list[int]]:
    """Longest processing time first: units in decreasing weight (ties by index), each to the rank
    with the least weight so far (ties to the lowest rank). Returns each rank's units in increasing
    index order; every unit once. Used for outage cases (weighted by their right-hand sides) and
    networks (weighted by factor entries times right-hand sides)."""
    if world < 1:
        raise ValueError("a world of at least one rank")
    w = [float(x) for x in weights]
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    share: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += w[i]
        share[r].append(i)
    return [sorted(s) for s in share]


def sum_in_rank_order(values):
    """The sum over ranks of every rank's float64 array `values` (its own for one process), added
    in rank order on every rank, so all ranks get the same bits whatever the backend's reduction
    order: an all-gather, then rank 0's + rank 1's + ..."""
    import numpy as np
    v = np.ascontiguousarray(values, np.float64)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return v.copy()
    t = torch.from_numpy(v).to(_device())
    parts = [torch.empty_like(t) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    total = parts[0].cpu().numpy().copy()
    for q in parts[1:]:
        total += q.cpu().numpy()
    return total


def whole_job_rate(units_per_rank: int, world: int, seconds: float) -> float:
    """Units per second over all ranks when every rank processed `units_per_rank` units and the
    slowest took `seconds`."""
    return units_per_rank * world / seconds
