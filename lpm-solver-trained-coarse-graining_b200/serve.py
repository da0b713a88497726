"""Continuous-batching serving of LPM solves (mixed precision) on one GPU.

A request is one specimen: a full 2D square or 3D simple-cubic box of any size, its per-bond Kn, Tv, and 1-9 load
cases (DOF masks and prescribed displacements).  Requests are grouped into size buckets:

* A bucket is a persistent batch on the device: S specimen slots x R system slots (R = the most load cases a request
  may bring), with its own CUDA stream, coefficient / preconditioner / vector state and solver workspace.
* A worker thread per bucket runs rounds.  One round is one refinement step of the mixed-precision solver over the
  whole bucket (FP64 true residual; FP32 block-Jacobi PCG on every unconverged system, each system frozen at its own
  convergence; FP64 correction).  Empty slots and converged systems cost no operator work (per-system activity masks
  inside the kernels).
* Between rounds the worker retires the slots whose load cases all converged and admits waiting requests into free
  slots.  A request that arrives while others are on the GPU therefore joins the running batch at the next refinement
  step; rounds of different buckets overlap on the device.
* Buckets are created on demand while the HBM budget allows and released when idle, so waiting requests of a new
  size are admitted as memory frees up.
* 3D buckets autotune the z-chunking of their operator when created; blocks of CG iterations replay CUDA graphs that
  the library captures per bucket (its workspace and buffers are fixed for the bucket's lifetime).
* 3D requests whose load cases all use the standard boundary boxes of the reference's load set (KUBC ring, z plates,
  x plates: geom.LOADS) go to AMG buckets: the inner solver is the aggregation-AMG PCG (timing/t3d/amg3d.py) instead
  of block Jacobi.  Such a bucket has one system slot per load of geom.LOADS, so slot j always carries load type j's
  DOF mask and the hierarchy's aggregation (one per free box) is built once, with the bucket; a request's load cases
  take the free slots of their mask.  The numeric hierarchies are set up again after every round that admitted a
  specimen.  Other 3D requests (any other boundary masks) use block-Jacobi buckets.

The solution of a request does not depend on the other requests of its bucket: systems are independent in every
kernel, reductions are per system in a fixed order, and the bucket's launch geometry is fixed by its capacity.
"""
import collections
import ctypes
import threading
import time

import numpy as np
import torch

from . import _lib as L
from . import amg as GA
from . import core
from . import geom as G

_F64, _F32 = torch.float64, torch.float32


class Request:
    """One specimen to solve.  dim 2 (square) or 3 (SC); shape (nx, ny) or (nx, ny, nz); Kn, Tv (N, NN) FP64 arrays;
    free (L, N, d) bool per-DOF free masks and up (L, N, d) prescribed displacements of its L load cases."""

    _ids = iter(range(1 << 62))

    def __init__(self, dim, shape, Kn, Tv, free, up, arrival=None):
        self.rid = next(Request._ids)
        self.dim = int(dim)
        self.shape = tuple(int(v) for v in shape)
        self.Kn = np.ascontiguousarray(Kn, dtype=np.float64)
        self.Tv = np.ascontiguousarray(Tv, dtype=np.float64)
        self.free = np.ascontiguousarray(free, dtype=bool)
        self.up = np.ascontiguousarray(up, dtype=np.float64)
        self.nloads = self.free.shape[0]
        self.arrival = arrival
        self.admitted = None
        self.done = None
        self.u = None
        self.relres = None
        self.status = None
        self.iters = 0
        self.rounds = 0
        self.slot_map = None  # AMG buckets: the system slot of each load case

    @property
    def key(self):
        nz = self.shape[2] if self.dim == 3 else 1
        return (self.dim, self.shape[0], self.shape[1], nz)

    @property
    def latency(self):
        return None if self.done is None or self.arrival is None else self.done - self.arrival


def bucket_bytes(key, slots, rmax):
    """Device bytes a bucket of `slots` specimens x `rmax` systems holds (state + solver workspace), estimated."""
    dim, nx, ny, nz = key[:4]
    N = nx * ny * nz
    NN, d = (18, 3) if dim == 3 else (8, 2)
    nsys = slots * rmax
    per_set = N * NN * (8 * 2 + 4 * 2) + N * d * d * 4           # FP64 + FP32 coefficients, FP32 preconditioner
    per_sys = N * d * (8 * 3 + 1)                                 # b, x, up (FP64) + mask
    work = nsys * N * d * (8 * 3 + 4 * 2 * 4)                     # IR vectors (FP64) + FP32 engine (pair layout)
    if len(key) > 4 and key[4] == "amg":
        # AMG handle: level-1 operators of three free boxes (36 floats per fine particle each), dense coarsest
        # inverses (FP64 + FP32, at most 1024 unknowns per box), cycle vectors
        per_set += N * 36 * 4 * 3 + 3 * (1024 ** 2) * 12
        work += nsys * N * d * 4 * 8
    return slots * per_set + nsys * per_sys + work + (64 << 20)


_STD_MASKS = {}
_STD_LOCK = threading.Lock()


def standard_masks(shape):
    """Particle free masks (len(geom.LOADS), N) of the reference's 3D load set on an nx x ny x nz box (cached)."""
    shape = tuple(int(v) for v in shape)
    with _STD_LOCK:
        m = _STD_MASKS.get(shape)
        if m is None:
            lat = G.LatticeGeom(*shape, 1.0)
            m = np.array([~G.prescribed(ld, lat.x, lat.ijk, shape, 1)[0] for ld in G.LOADS])
            _STD_MASKS[shape] = m
        return m


def amg_slots(req):
    """Slot (index into geom.LOADS) of each load case of a 3D request whose DOF masks are all standard boxes, each
    load on its own slot of that mask; None if some load case has another mask."""
    if req.dim != 3:
        return None
    masks = standard_masks(req.shape)
    used, out = set(), []
    for l in range(req.nloads):
        f = req.free[l]
        if not (f == f[:, :1]).all():               # not a particle mask
            return None
        fp = f[:, 0]
        j = next((j for j in range(len(masks)) if j not in used and np.array_equal(masks[j], fp)), None)
        if j is None:
            return None
        used.add(j)
        out.append(j)
    return out


class Bucket:
    """Persistent device batch of one lattice size.  A key with a trailing "amg" makes an AMG bucket (3D only): one
    system slot per load type of geom.LOADS, the aggregation-AMG PCG as the inner solver."""

    def __init__(self, key, slots, rmax, device, tol=1e-8, inner_tol=1e-3, maxit=50000, autotune=True,
                 amg_inner_tol=1e-4):
        self.use_amg = len(key) > 4 and key[4] == "amg"
        if self.use_amg:
            rmax = len(G.LOADS)
            inner_tol = amg_inner_tol
        self.key, self.S, self.R = key, int(slots), int(rmax)
        self.device = torch.device(device)
        self.tol, self.inner_tol, self.maxit = tol, inner_tol, maxit
        dim, nx, ny, nz = key[:4]
        self.lat = G.LatticeGeom(nx, ny, nz, 1.0) if dim == 3 else G.SquareLattice(nx, ny, 1.0)
        self.dl = core.DeviceLattice(self.lat, self.device)
        N, NN, d = self.lat.N, self.lat.NN, dim
        self.N, self.NN, self.d = N, NN, d
        S, R = self.S, self.R
        self.nsys = S * R
        dv = self.device
        self.stream = torch.cuda.Stream(dv)
        with torch.cuda.stream(self.stream):
            # FP64 coefficients packed (S, NN, N): the refinement's FP64 residuals and the right-hand sides run on the
            # packed operators (TMA-fed in 3D, shared-memory tiles in 2D)
            self.K64 = torch.zeros((S, NN, N), dtype=_F64, device=dv)
            self.T64 = torch.zeros((S, NN, N), dtype=_F64, device=dv)
            self.K32 = torch.zeros((S, NN, N), dtype=_F32, device=dv)
            self.T32 = torch.zeros((S, NN, N), dtype=_F32, device=dv)
            self.M32 = torch.zeros((S, N, d, d), dtype=_F32, device=dv)
            self.mask = torch.ones((self.nsys, N, d), dtype=torch.uint8, device=dv)
            self.b = torch.zeros((self.nsys, N, d), dtype=_F64, device=dv)
            self.x = torch.zeros((self.nsys, N, d), dtype=_F64, device=dv)
            self.up = torch.zeros((self.nsys, N, d), dtype=_F64, device=dv)
            lib = L.load()
            self._batch = L.Batch(self.nsys, R, self.nsys, 0)
            self.amgb = None
            if self.use_amg:
                # slot j of every specimen carries load type j's mask; every set starts as a homogeneous solid so
                # that the hierarchies of empty slots are well defined
                std = standard_masks((nx, ny, nz))
                self.amgb = GA.AmgBatch(self.dl, self.nsys, R, std, **GA.AMG_CFG)
                self._batch = L.Batch(self.nsys, R, R, 0)
                self.mask = self.amgb.mask              # (R, N, 3): system s uses mask s % R
                Kh, Th = G.bond_params_two_end_mean(self.lat, G.sc_params_from_C(G.iso_C(np.ones(N), 0.2), 0.5))
                Kr = torch.as_tensor(Kh, device=dv)[None]
                Tr = torch.as_tensor(Th, device=dv)[None]
                self.K64[:] = core.pack(Kr, _F64)
                self.T64[:] = core.pack(Tr, _F64)
                self.K32[:] = core.pack(Kr, _F32)
                self.T32[:] = core.pack(Tr, _F32)
                self.M32[:] = core.block_jacobi(self.dl, Kr, Tr, _F32)
                self._setup_due = True
            nbytes = lib.lpm_ir_workspace_bytes(self.dl.ref, ctypes.byref(self._batch), 0 if self.use_amg else 1)
            L.check(nbytes if nbytes < 0 else 0, "lpm_ir_workspace_bytes")
            self.ws = torch.empty(int(nbytes), dtype=torch.uint8, device=dv)
            self.it = torch.zeros(self.nsys, dtype=torch.int32, device=dv)
            self.rel = torch.zeros(self.nsys, dtype=_F64, device=dv)
            self.st = torch.zeros(self.nsys, dtype=torch.int32, device=dv)
            self.zchunk = None
            if autotune and dim == 3 and nx % 4 == 0:
                self.zchunk = core.autotune(self.dl, self.K32, self.T32, self.nsys, R)
        self.stream.synchronize()
        self.slots = [None] * S
        self.queue = collections.deque()
        self.rounds = 0
        self.busy_s = 0.0
        self.admit_s = 0.0
        self.inner_iters = 0
        self.idle_since = time.perf_counter()

    # ------------------------------------------------------------------------------------------------ state
    @property
    def occupied(self):
        return sum(r is not None for r in self.slots)

    @property
    def free_slots(self):
        return [s for s in range(self.S) if self.slots[s] is None]

    def nbytes(self):
        ts = (self.K64, self.T64, self.K32, self.T32, self.M32, self.mask, self.b, self.x, self.up, self.ws)
        return sum(t.numel() * t.element_size() for t in ts)

    def admit(self, req, s):
        """Copy a request into slot s: coefficients (FP64 and packed FP32), block-Jacobi inverse, DOF masks,
        right-hand sides b = -K u_p (FP64), x = 0."""
        if req.key != self.key[:4] or req.nloads > self.R:
            raise ValueError("request %s with %d loads does not fit bucket %s x %d" % (req.key, req.nloads, self.key,
                                                                                      self.R))
        if self.use_amg:
            if req.slot_map is None:
                req.slot_map = amg_slots(req)
            if req.slot_map is None:
                raise ValueError("request %s has boundary masks outside the AMG bucket's load set" % (req.key,))
        R, d, N = self.R, self.d, self.N
        sl = slice(s * R, (s + 1) * R)
        t_adm = time.perf_counter()
        with torch.cuda.stream(self.stream):
            dv = self.device
            Kr = torch.as_tensor(req.Kn).to(dv)[None]          # reference layout (1, N, NN), FP64
            Tr = torch.as_tensor(req.Tv).to(dv)[None]
            self.K64[s:s + 1] = core.pack(Kr, _F64)
            self.T64[s:s + 1] = core.pack(Tr, _F64)
            self.K32[s:s + 1] = core.pack(Kr, _F32)
            self.T32[s:s + 1] = core.pack(Tr, _F32)
            self.M32[s:s + 1] = core.block_jacobi(self.dl, Kr, Tr, _F32)
            rows = self.rows(s, req) - s * R          # the request's system slots within the specimen slot
            rows_t = torch.as_tensor(rows, device=dv)
            # DOF masks and prescribed displacements of the slot's R systems, built on the device (only the
            # request's own arrays cross from the host)
            fr = self.mask.clone() if self.use_amg else torch.ones((R, N, d), dtype=torch.uint8, device=dv)
            fr[rows_t] = torch.as_tensor(req.free.reshape(req.nloads, N, d)).to(dv, torch.uint8)
            up = torch.zeros((R, N, d), dtype=torch.float64, device=dv)
            up[rows_t] = torch.as_tensor(req.up.reshape(req.nloads, N, d)).to(dv)
            if not self.use_amg:
                self.mask[sl].copy_(fr)
            self.up[sl].copy_(up * (1 - fr.double()))
            Ku = core.kmv(self.dl, self.up[sl], self.K64[s:s + 1], self.T64[s:s + 1], layout=L.LAYOUT_SOA,
                          rhs_per_set=R)
            used = torch.zeros(R, dtype=_F64, device=dv)
            used[torch.as_tensor(rows, device=dv)] = 1.0
            self.b[sl] = -Ku * fr * used[:, None, None]
            self.x[sl] = 0.0
            if self.use_amg:
                self._setup_due = True
        self.slots[s] = req
        req.admitted = time.perf_counter()
        self.admit_s += req.admitted - t_adm

    def rows(self, s, req):
        """System indices of request req in specimen slot s."""
        if self.use_amg:
            return s * self.R + np.asarray(req.slot_map, dtype=np.int64)
        return s * self.R + np.arange(req.nloads)

    def round(self):
        """One refinement step over the bucket.  Returns the per-system (relres, status) on the host."""
        lib = L.load()
        opts = L.IrOpts(float(self.tol), float(self.inner_tol), int(self.maxit), 1, 1, 10, None)
        outer = ctypes.c_int32(0)
        t0 = time.perf_counter()
        with torch.cuda.stream(self.stream):
            if self.use_amg:
                if self._setup_due:                     # new specimens since the last round: numeric hierarchies
                    self.amgb.setup(self.K32, self.T32, self.M32)
                    self._setup_due = False
                L.check(lib.lpm_ir_amg(self.dl.ref, L.ptr(self.K64), L.ptr(self.T64), L.LAYOUT_SOA, self.amgb._h,
                                       ctypes.byref(self._batch), L.ptr(self.mask), L.ptr(self.b), L.ptr(self.x),
                                       ctypes.byref(opts), L.ptr(self.ws), self.ws.numel(), L.ptr(self.it),
                                       L.ptr(self.rel), L.ptr(self.st), ctypes.byref(outer), self.stream.cuda_stream),
                        "lpm_ir_amg")
            else:
                L.check(lib.lpm_ir_batched(self.dl.ref, L.ptr(self.K64), L.ptr(self.T64), L.LAYOUT_SOA,
                                           L.ptr(self.K32), L.ptr(self.T32), L.ptr(self.M32), ctypes.byref(self._batch),
                                           L.ptr(self.mask), L.ptr(self.b), L.ptr(self.x), ctypes.byref(opts),
                                           L.ptr(self.ws), self.ws.numel(), L.ptr(self.it), L.ptr(self.rel),
                                           L.ptr(self.st), ctypes.byref(outer), self.stream.cuda_stream),
                        "lpm_ir_batched")
            rel = self.rel.cpu().numpy()
            st = self.st.cpu().numpy()
            its = self.it.cpu().numpy()
        self.rounds += 1
        self.busy_s += time.perf_counter() - t0
        self.inner_iters += int(its.max())
        return rel, st, its

    def retire(self, s, status):
        """Copy slot s's solution u = u_p + x to the host and free the slot."""
        req = self.slots[s]
        n = req.nloads
        rows = torch.as_tensor(self.rows(s, req), device=self.device)
        with torch.cuda.stream(self.stream):
            u = (self.up[rows] + self.x[rows]).cpu().numpy()
            rel = self.rel[rows].cpu().numpy()
        req.u = u.reshape((n,) + (self.N, self.d))
        req.relres = rel
        req.status = status
        req.done = time.perf_counter()
        self.slots[s] = None
        if self.occupied == 0:
            self.idle_since = time.perf_counter()
        return req


class Server:
    """Request loop: buckets per lattice size within an HBM budget, one worker thread per bucket.

    submit(req) hands a request to its bucket (created on demand); results are collected with wait_all().  A request
    whose bucket cannot be created yet (budget) waits in a pending list and is placed as soon as idle buckets are
    released.  `bucket_factory(key, slots, rmax)` builds buckets (the CUDA `Bucket` by default)."""

    def __init__(self, device="cuda", budget_bytes=None, rmax=9, max_slots=8, tol=1e-8, inner_tol=1e-3,
                 max_rounds=40, idle_release_s=0.5, bucket_factory=None, bytes_fn=bucket_bytes, rmax2d=None,
                 amg3d=True, amg_inner_tol=1e-4):
        self.device = torch.device(device)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(0.6 * free)
        self.budget = int(budget_bytes)
        self.rmax, self.max_slots = rmax, max_slots
        self.rmax2d = rmax if rmax2d is None else rmax2d   # system slots per specimen of 2D buckets
        self.amg3d = amg3d                                 # 3D requests on standard boxes go to AMG buckets
        self.tol, self.inner_tol, self.max_rounds = tol, inner_tol, max_rounds
        self.idle_release_s = idle_release_s
        self.bytes_fn = bytes_fn
        self.factory = bucket_factory or (lambda key, slots, rmax: Bucket(key, slots, rmax, self.device, tol=tol,
                                                                           inner_tol=inner_tol,
                                                                           amg_inner_tol=amg_inner_tol))
        self.buckets = {}
        self.bucket_log = []        # keys of the buckets created, in order
        self.reserved = {}
        self.pending = collections.deque()
        self.done = []
        self.lock = threading.Condition()
        self.threads = {}
        self.stop = False
        self.errors = []

    # ------------------------------------------------------------------------------------------- placement
    def used_bytes(self):
        return sum(self.reserved.values())

    def _rmax(self, key):
        if len(key) > 4 and key[4] == "amg":
            return len(G.LOADS)
        return self.rmax2d if key[0] == 2 else self.rmax

    def bucket_key(self, req):
        """The bucket of a request: its lattice size, plus "amg" for 3D requests on the standard boundary boxes."""
        if self.amg3d and req.dim == 3:
            if req.slot_map is None:
                req.slot_map = amg_slots(req)   # kept for the bucket's admission
            if req.slot_map is not None:
                return req.key + ("amg",)
        return req.key

    def _slots_for(self, key):
        """Largest slot count (<= max_slots) whose bucket fits in the remaining budget; 0 if none fits."""
        left = self.budget - self.used_bytes()
        for s in range(self.max_slots, 0, -1):
            if self.bytes_fn(key, s, self._rmax(key)) <= left:
                return s
        return 0

    def _release_idle(self, now):
        for key, b in list(self.buckets.items()):
            if b.occupied == 0 and not b.queue and now - b.idle_since >= self.idle_release_s:
                self._drop_bucket(key)

    def _drop_bucket(self, key):
        b = self.buckets.pop(key)
        self.reserved.pop(key, None)
        b.retired = True
        self.lock.notify_all()

    def _place(self, req):
        """Under the lock: hand req to its bucket, creating the bucket if the budget allows; False if it must wait."""
        key = self.bucket_key(req)
        b = self.buckets.get(key)
        if b is None:
            slots = self._slots_for(key)
            if slots == 0:
                self._release_idle(time.perf_counter() + self.idle_release_s)  # free every idle bucket now
                slots = self._slots_for(key)
            if slots == 0:
                return False
            b = self.factory(key, slots, self._rmax(key))
            b.retired = False
            self.buckets[key] = b
            self.bucket_log.append(key)
            self.reserved[key] = self.bytes_fn(key, slots, self._rmax(key))
            t = threading.Thread(target=self._worker, args=(key, b), daemon=True)
            self.threads[key] = t
            t.start()
        b.queue.append(req)
        self.lock.notify_all()
        return True

    def submit(self, req):
        if req.nloads < 1 or req.nloads > self._rmax(req.key):
            raise ValueError("a request brings 1..%d load cases (got %d)" % (self._rmax(req.key), req.nloads))
        if req.arrival is None:
            req.arrival = time.perf_counter()
        with self.lock:
            if not self.pending and self._place(req):
                return
            self.pending.append(req)

    def _retry_pending(self):
        while self.pending:
            if not self._place(self.pending[0]):
                break
            self.pending.popleft()

    # ---------------------------------------------------------------------------------------------- worker
    def _worker(self, key, b):
        try:
            while True:
                with self.lock:
                    while not self.stop and not b.retired and b.occupied == 0 and not b.queue:
                        self.lock.wait(0.05)
                        self._retry_pending()
                    if self.stop or b.retired:
                        return
                    admits = []
                    for s in b.free_slots:
                        if not b.queue:
                            break
                        req = b.queue.popleft()
                        b.slots[s] = req            # reserved under the lock: the bucket is not idle any more
                        admits.append((req, s))
                for req, s in admits:
                    b.admit(req, s)
                rel, st, its = b.round()
                finished = []
                for s, req in enumerate(b.slots):
                    if req is None:
                        continue
                    req.rounds += 1
                    sl = b.rows(s, req) if hasattr(b, "rows") else slice(s * b.R, s * b.R + req.nloads)
                    req.iters += int(its[sl].max())
                    conv = bool((rel[sl] <= self.tol).all())
                    broke = bool((st[sl] == L.STATUS_BREAKDOWN).any())
                    if conv or broke or req.rounds >= self.max_rounds:
                        status = L.STATUS_OK if conv else (L.STATUS_BREAKDOWN if broke else L.STATUS_NOT_CONVERGED)
                        finished.append((s, status))
                for s, status in finished:
                    req = b.retire(s, status)
                    with self.lock:
                        self.done.append(req)
                        self.lock.notify_all()
                with self.lock:
                    self._release_idle(time.perf_counter())
                    self._retry_pending()
        except Exception as exc:  # surface worker failures to the caller of wait_all
            with self.lock:
                self.errors.append(exc)
                self.lock.notify_all()

    def wait_all(self, n, timeout=None):
        """Block until n requests are done (or a worker failed); returns the finished requests."""
        t0 = time.perf_counter()
        with self.lock:
            while len(self.done) < n and not self.errors:
                self.lock.wait(0.05)
                self._retry_pending()
                if timeout is not None and time.perf_counter() - t0 > timeout:
                    break
            if self.errors:
                raise self.errors[0]
            return list(self.done)

    def close(self):
        with self.lock:
            self.stop = True
            self.lock.notify_all()
        for t in self.threads.values():
            t.join(timeout=30)


def bucket_stats(server):
    """Per-bucket activity of a server: rounds, GPU-side busy seconds of the rounds, admission seconds, inner PCG
    iterations (slowest system per round, summed), capacity."""
    out = {}
    for key, b in list(server.buckets.items()):
        name = "%dD %s" % (key[0], "x".join(str(v) for v in key[1:1 + key[0]]))
        out[name + (" amg" if len(key) > 4 else "")] = {
            "slots": b.S, "rounds": b.rounds, "busy_s": round(getattr(b, "busy_s", 0.0), 3),
            "admit_s": round(getattr(b, "admit_s", 0.0), 3), "inner_iters": getattr(b, "inner_iters", 0)}
    return out


def latency_stats(reqs):
    lat = np.array([r.latency for r in reqs if r.latency is not None])
    if lat.size == 0:
        return {}
    return {"p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "mean_ms": float(lat.mean() * 1e3), "max_ms": float(lat.max() * 1e3)}
