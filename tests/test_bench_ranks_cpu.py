"""The benchmark's multi-rank logic on two gloo ranks (CPU): each rank renders its own replica
of the frame (weak scaling, no collective on the data path), and the line's value is all
ranks' path solves over the slowest rank's device time.  bench.barrier / bench.reduce are the
calls bench.py makes between and after the timed frames under torchrun."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = [120.0, 135.5][rank]         # the slower rank sets the time
        paths = [1.28e9, 1.30e9][rank]    # every rank's replica counts
        bench.barrier(world)
        t_max = bench.reduce(world, ms, "max")
        total = bench.reduce(world, paths, "sum")
        bench.barrier(world)
        out[rank] = (t_max, total, total / (t_max / 1e3))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_reduce_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]
    t_max, total, value = res[0]
    assert t_max == 135.5 and total == 1.28e9 + 1.30e9
    assert abs(value - (2.58e9 / 0.1355)) < 1.0
