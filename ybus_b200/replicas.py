"""One process per GPU for the solve path, which shards with no data-path exchange: right-hand
sides, outage cases and networks are independent, so every rank solves its own share on its own GPU
and the processes meet only to start timing together and to take the slowest rank's time. These
helpers hold that logic apart from the GPU so that it runs (and is tested) on any torch.distributed
backend, gloo on the CPU included."""
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


def whole_job_rate(units_per_rank: int, world: int, seconds: float) -> float:
    """Units per second over all ranks when every rank processed `units_per_rank` units and the
    slowest took `seconds`."""
    return units_per_rank * world / seconds
