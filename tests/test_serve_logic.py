"""Host logic of the serving loop (no GPU): bucket placement within the HBM budget, continuous admission into free
slots between rounds, retirement, release of idle buckets, validation.  Buckets are replaced by a fake that converges
each request after a set number of rounds."""
import collections
import threading
import time

import numpy as np
import pytest

from lpm_b200 import serve


class FakeBucket:
    log = []
    lock = threading.Lock()

    def __init__(self, key, slots, rmax):
        self.key, self.S, self.R = key, slots, rmax
        self.slots = [None] * slots
        self.queue = collections.deque()
        self.idle_since = time.perf_counter()
        self.rounds = 0

    @property
    def occupied(self):
        return sum(r is not None for r in self.slots)

    @property
    def free_slots(self):
        return [s for s in range(self.S) if self.slots[s] is None]

    def admit(self, req, s):
        self.slots[s] = req
        req.admitted = time.perf_counter()
        with FakeBucket.lock:
            FakeBucket.log.append(("admit", req.rid, self.key, s, self.rounds))

    def round(self):
        time.sleep(0.005)
        rel = np.ones(self.S * self.R)
        for s, req in enumerate(self.slots):
            if req is not None and req.rounds + 1 >= req.need:
                rel[s * self.R:(s + 1) * self.R] = 0.0
        self.rounds += 1
        return rel, np.zeros(self.S * self.R, np.int32), np.full(self.S * self.R, 7, np.int32)

    def retire(self, s, status):
        req = self.slots[s]
        req.status, req.done = status, time.perf_counter()
        self.slots[s] = None
        if self.occupied == 0:
            self.idle_since = time.perf_counter()
        with FakeBucket.lock:
            FakeBucket.log.append(("retire", req.rid, self.key, s, self.rounds))
        return req


def req(dim, n, loads, need):
    N = n ** dim
    d = dim
    NN = 18 if dim == 3 else 8
    r = serve.Request(dim, (n,) * dim, np.zeros((N, NN)), np.zeros((N, NN)), np.ones((loads, N, d), bool),
                      np.zeros((loads, N, d)))
    r.need = need
    return r


def bytes_fn(key, slots, rmax):
    return slots * 100


def make_server(budget, max_slots=2):
    FakeBucket.log = []
    return serve.Server(device="cpu", budget_bytes=budget, rmax=4, max_slots=max_slots, bytes_fn=bytes_fn,
                        bucket_factory=lambda k, s, r: FakeBucket(k, s, r), idle_release_s=0.02)


def test_continuous_admission_into_running_bucket():
    """A request that arrives while its bucket is busy is admitted as soon as a slot frees, while the other slot's
    long request is still running."""
    srv = make_server(budget=1000, max_slots=2)
    try:
        long_, short = req(3, 8, 2, need=30), req(3, 8, 1, need=2)
        srv.submit(long_)
        srv.submit(short)
        time.sleep(0.05)
        late = req(3, 8, 3, need=2)
        srv.submit(late)
        done = srv.wait_all(3, timeout=20)
        assert len(done) == 3 and all(r.status == 0 for r in done)
        assert late.admitted < long_.done, "the late request waited for the whole batch"
        admits = [e for e in FakeBucket.log if e[0] == "admit"]
        assert [e[1] for e in admits][:2] == [long_.rid, short.rid]
        assert admits[2][4] > 0            # admitted between rounds of a running bucket
    finally:
        srv.close()


def test_budget_limits_buckets_and_idle_release():
    """With room for one bucket only, a second size waits until the first bucket is idle and released."""
    srv = make_server(budget=250, max_slots=2)
    try:
        a1, a2 = req(3, 8, 1, need=3), req(3, 8, 1, need=3)
        b1 = req(2, 16, 2, need=2)
        for r in (a1, a2, b1):
            srv.submit(r)
        done = srv.wait_all(3, timeout=20)
        assert len(done) == 3
        assert b1.admitted >= max(a1.done, a2.done)
        assert srv.used_bytes() <= 250
    finally:
        srv.close()


def test_slots_follow_budget_and_validation():
    srv = make_server(budget=150, max_slots=4)
    try:
        assert srv._slots_for((3, 8, 8, 8)) == 1
        with pytest.raises(ValueError):
            srv.submit(req(3, 8, 5, need=1))       # more load cases than the bucket's systems
        assert serve.bucket_bytes((3, 48, 48, 48), 2, 9) > serve.bucket_bytes((3, 48, 48, 48), 1, 9)
    finally:
        srv.close()


def test_latency_stats():
    rs = [req(2, 4, 1, 1) for _ in range(4)]
    for k, r in enumerate(rs):
        r.arrival, r.done = 0.0, 0.01 * (k + 1)
    st = serve.latency_stats(rs)
    assert abs(st["p50_ms"] - 25.0) < 1e-6 and st["max_ms"] == pytest.approx(40.0)


def std_req(n, loads, need=1):
    """A 3D request whose load cases use the reference's standard boundary boxes (geom.prescribed)."""
    from lpm_b200 import geom as G
    lat = G.LatticeGeom(n, n, n, 1.0)
    free, up = [], []
    for ld in loads:
        fixed, u, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        free.append(np.repeat(~fixed[:, None], 3, 1))
        up.append(np.where(fixed[:, None], u, 0.0))
    r = serve.Request(3, (n,) * 3, np.zeros((lat.N, 18)), np.zeros((lat.N, 18)), np.array(free), np.array(up))
    r.need = need
    return r


def test_amg_bucket_routing_and_slots():
    """3D requests on the standard load boxes are keyed to AMG buckets, one slot per load type (the six KUBC loads
    share the ring mask, the two plate loads the z-plate mask); any other mask keeps the plain key; 2D never uses AMG."""
    from lpm_b200 import geom as G
    srv = make_server(budget=1000)
    try:
        r = std_req(9, ["tb_sx", "k_xx", "lr_tx", "k_yz", "tb_tz"])
        assert srv.bucket_key(r) == (3, 9, 9, 9, "amg")
        slots = serve.amg_slots(r)
        masks = serve.standard_masks((9, 9, 9))
        assert len(set(slots)) == 5
        for l, j in enumerate(slots):
            assert np.array_equal(masks[j], r.free[l][:, 0])
        assert slots[1] == G.LOADS.index("k_xx") and slots[2] == G.LOADS.index("lr_tx")
        assert srv._rmax(srv.bucket_key(r)) == len(G.LOADS)
        all_ring = std_req(9, G.LOADS[:6])
        assert sorted(serve.amg_slots(all_ring)) == list(range(6))
        assert srv.bucket_key(req(3, 8, 2, need=1)) == (3, 8, 8, 8)     # all-free masks: not a standard box
        assert srv.bucket_key(req(2, 16, 2, need=1)) == (2, 16, 16, 1)
        srv.amg3d = False
        assert srv.bucket_key(r) == (3, 9, 9, 9)
        key = (3, 9, 9, 9, "amg")
        assert serve.bucket_bytes(key, 2, 9) > serve.bucket_bytes(key[:4], 2, 9)
    finally:
        srv.close()


def test_reference_sample_walks_the_batch():
    """The reference arm's bounded sample takes consecutive (specimen, load) pairs of the whole batch, wrapping."""
    import bench
    assert bench.reference_picks(16, 6, 0, 1) == [(0, 0)]
    assert bench.reference_picks(16, 6, 7, 1) == [(1, 1)]
    seen = {bench.reference_picks(16, 6, k, 1)[0] for k in range(96)}
    assert len(seen) == 96
    assert bench.reference_picks(2, 3, 2, 2) == [(1, 1), (1, 2)]
