"""The multi-process path of the solve (one process per GPU, no data-path exchange), on the CPU:
two gloo ranks meet at a barrier, agree on the slowest rank's time, and split independent units
(right-hand sides, outage cases, networks) into shares that cover every unit once."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from ybus_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = replicas.rank_info()
        replicas.barrier()
        slowest = replicas.max_over_ranks(1.0 + r)  # rank 1 is the slow one
        mine = replicas.shard(13499, r, w)
        out.put((r, w, local, slowest, mine.start, mine.stop))
        replicas.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_disjoint_shares():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in results] == [(0, 2, 0), (1, 2, 1)]
    assert all(r[3] == 2.0 for r in results)
    shares = [range(r[4], r[5]) for r in results]
    assert shares[0].start == 0 and shares[0].stop == shares[1].start and shares[1].stop == 13499
    assert abs(len(shares[0]) - len(shares[1])) <= 1


@pytest.mark.parametrize("units,world", [(0, 3), (7, 3), (13499, 8), (5, 8)])
def test_shares_cover_every_unit_once(units, world):
    covered = [u for r in range(world) for u in replicas.shard(units, r, world)]
    assert covered == list(range(units))
    sizes = [len(replicas.shard(units, r, world)) for r in range(world)]
    assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(units, world, world)


def test_one_process_needs_no_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    replicas.barrier()
    assert replicas.whole_job_rate(13499, 4, 2.0) == 13499 * 4 / 2.0
