"""The multi-rank path of the benchmark on CPU (world size 2, gloo): disjoint specimen shards per rank, the step time
is the slowest rank's, the job throughput counts every rank's systems.  The solves themselves need no collective: in
the second test every rank solves its own shard (6^3 specimens, the CPU oracle's FP64 PCG standing in for the GPU
solve), rank 0 gathers the shards, and the gathered results equal a single-process run of all specimens."""
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


def _specimen(seed):
    import numpy as np
    from lpm_b200 import geom as G
    from lpm_b200 import micro as M
    n = 6
    lat = G.LatticeGeom(n, n, n, 1.0)
    ph, _ = M.spheres(n, n, n, 0.25, 1.5, np.random.default_rng(seed), rjit=0.0)
    C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    return lat, Kn, Tv


def _solve_shard(seeds):
    """FP64 block-Jacobi PCG (the oracle) of loads k_xx and k_xy of every specimen of a shard, one thread."""
    import numpy as np
    import oracle as O
    from lpm_b200 import geom as G
    O.set_threads(1)
    out = {}
    for sd in seeds:
        lat, Kn, Tv = _specimen(sd)
        us = []
        for ld in ("k_xx", "k_xy"):
            fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk, (6,) * 3, 1)
            u, _ = O.solve_pcg(lat, Kn, Tv, fixed, np.where(fixed[:, None], up, 0.0), tol=1e-10)
            us.append(u)
        out[sd] = np.stack(us)
    return out


def _rank_solve(rank, world, port, out):
    import sys
    import time
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    sys.path.insert(0, os.path.join(root, "tests"))
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = bench.shard_seeds(rank, 2)
        t0 = time.perf_counter()
        res = _solve_shard(seeds)
        ms = bench.max_over_ranks(1e3 * (time.perf_counter() - t0), world, torch.device("cpu"))
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            out.put((ms, merged, bench.job_throughput(world, 2 * len(seeds), 1, ms)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_solve_their_shards():
    import sys
    import numpy as np
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "oracle"))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_solve, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ms, merged, value = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == [0, 1, 2, 3]                  # every specimen solved once, on its own rank
    single = _solve_shard([0, 1, 2, 3])
    for sd in range(4):
        assert np.array_equal(merged[sd], single[sd])
    assert ms > 0 and value == pytest.approx(2 * 4 / (ms / 1e3))
