"""CPU, two gloo ranks: the multi-GPU plumbing of the reconstruction path —
max over ranks of a time, the y-slab partition of one series, the replicas'
distinct seeded series, and the whole-job rate."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from aretomo3_b200 import ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, lr = ranks.rank_env()
        ranks.barrier()
        slowest = ranks.max_over_ranks(10.0 * (r + 1))
        y0, y1 = ranks.rows_of_rank(101, r, w)
        from aretomo3_b200 import synth
        c = synth.wbp_small(seed=1 + r)
        frames = synth.make_tilt_series(64, 4, c["tilts"][:5], 16, c["phantom"])
        out.put((r, w, lr, slowest, (y0, y1), float(frames.sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[0] for x in res] == [0, 1] and all(x[1] == 2 and x[2] == x[0] for x in res)
    assert all(x[3] == 20.0 for x in res)                       # both ranks see the slowest time
    assert res[0][4] == (0, 51) and res[1][4] == (51, 101)      # the slabs tile the series
    assert res[0][5] != res[1][5]                               # replicas reconstruct distinct series


@pytest.mark.parametrize("ny,world", [(1, 1), (7, 3), (1024, 8), (5, 8)])
def test_rows_partition(ny, world):
    covered = []
    for r in range(world):
        y0, y1 = ranks.rows_of_rank(ny, r, world)
        assert 0 <= y0 <= y1 <= ny
        covered += list(range(y0, y1))
    assert covered == list(range(ny))


def test_aggregate_rate():
    assert ranks.aggregate_rate(1e9, 5, 4, 1000.0) == pytest.approx(2e10)
    assert ranks.max_over_ranks(3.5) == 3.5   # single process: no process group
