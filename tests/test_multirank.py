"""The multi-rank path of the benchmark on CPU (world size 2, gloo): disjoint specimen shards per rank, the step time
is the slowest rank's, the job throughput counts every rank's systems.  The solves themselves need no collective."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = bench.shard_seeds(rank, 3)
        ms = bench.max_over_ranks(10.0 * (rank + 1), world, torch.device("cpu"))
        out.put((rank, seeds, ms, bench.job_throughput(world, 18, 2, ms)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, ms0, v0), (r1, s1, ms1, v1) = res
    assert s0 == [0, 1, 2] and s1 == [3, 4, 5]            # disjoint shards
    assert ms0 == ms1 == 20.0                              # slowest rank
    assert v0 == v1 == pytest.approx(2 * 18 * 2 / 0.020)   # whole-job systems per second
