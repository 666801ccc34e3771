"""The multi-process path of the solve (one process per GPU, no data-path exchange but the
adjoint's), on the CPU: two gloo ranks meet at a barrier, agree on the slowest rank's time, and
split independent units (right-hand sides, outage cases by LPT, networks) into shares that cover
every unit once; ranks that split the adjoint's scenarios reduce dL/db and the loss in rank order
to the single process's gradient, every rank with the same bits."""
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


def _adjoint_rank(rank: int, world: int, port: int, out) -> None:
    # the sharded adjoint on the CPU: this rank's scenarios through the oracle's gradient, then the
    # one exchange of the path, dL/db and the loss summed over the ranks in rank order
    import datetime

    import numpy as np
    import torch.distributed as dist

    import oracle.oracle as orc
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g, p, limits, chol, position = _adjoint_case()
        mine = replicas.shard(p.shape[0], rank, world)
        loss, gp, gb = orc.flow_loss_and_gradient(chol, g.n_bus, g.frm, g.to, g.susceptance, position,
                                                  p[mine.start:mine.stop], limits)
        total = replicas.sum_in_rank_order(np.append(gb, loss))
        out.put((rank, mine.start, mine.stop, gp, total))
    finally:
        dist.destroy_process_group()


def _adjoint_case():
    import numpy as np

    from dc_cases import cpu_model
    from ybus_b200 import grids
    g = grids.make_grid(300, 100, grids.SEED_BASE + 7)
    _, chol, position = cpu_model(g)
    rng = np.random.default_rng(8)
    p = rng.normal(0.0, 0.1, (37, g.n_bus))
    p[:, 0] = -p[:, 1:].sum(axis=1)
    limits = rng.uniform(0.5, 2.0, g.n_branch)
    return g, p, limits, chol, position


def test_sharded_adjoint_gradients_reduce_to_the_single_process_gradient():
    import numpy as np

    import oracle.oracle as orc
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_adjoint_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted((out.get(timeout=180) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g, p, limits, chol, position = _adjoint_case()
    loss, gp, gb = orc.flow_loss_and_gradient(chol, g.n_bus, g.frm, g.to, g.susceptance, position, p, limits)
    # every rank holds the same bits of the reduced dL/db and loss (summed in rank order)
    assert np.array_equal(results[0][4], results[1][4])
    total = results[0][4]
    assert np.abs(total[:-1] - gb).max() <= 1e-12 * np.abs(gb).max()
    assert abs(total[-1] - loss) <= 1e-12 * abs(loss)
    # dL/dp needs no exchange: each rank's rows are the single process's rows, bit for bit
    for rank, start, stop, gp_rank, _ in results:
        assert np.array_equal(gp_rank, gp[start:stop]), rank


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_lpt_covers_every_unit_once_and_balances(world):
    import numpy as np
    w = np.random.default_rng(9).integers(1, 65, 2000)  # outage cases weighted by scenario counts
    share = replicas.lpt(w, world)
    assert sorted(u for s in share for u in s) == list(range(w.size))
    loads = [int(w[s].sum()) for s in share]
    assert max(loads) - min(loads) <= w.max()  # LPT's bound: within one unit's weight
