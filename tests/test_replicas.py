"""Multi-GPU path of the benchmark on CPU: replicas only.

One solve is a sequential V-cycle, so N GPUs run N independent replicas, each
solving its own geometries with no collective in the data path; the job time
is the slowest rank's time (an all-reduce MAX once, outside the timed
region).  Two gloo ranks on 127.0.0.1 check that reduction, the barrier and
that the ranks' geometry seeds are disjoint.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        import bench
        bench.barrier(world)
        t = bench.max_over_ranks(1.0 + rank, world)
        seeds = bench.rank_seeds(rank, 7)
        out.put((rank, t, seeds))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_disjoint_geometries():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [2.0, 2.0]
    assert not set(res[0][2]) & set(res[1][2])
