"""bench.py's replica bookkeeping with two gloo ranks on CPU: the job time is
the maximum over ranks and the value counts every replica's steps."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        ws, r = bench._dist()
        t = bench.max_over_ranks(100.0 + 50.0 * rank, dist, "cpu")
        q.put((r, ws, t, bench.replica_value(t, 3, ws)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_value():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, ws, t, v in out:
        assert ws == 2
        assert t == 150.0
        assert v == pytest.approx(150.0 / 1e3 / 6)
