"""Benchmark of the LPM linear solve on B200: mixed-precision batched PCG solves per second.

Workloads (one "step" = one batched solve of every system from scratch, inputs resident in HBM):
  spheres48 (default): 48^3 simple-cubic fine LPM, seeded random non-overlapping spheres (r = 4 voxels, volume
    fraction 0.25, contrast 10, E = 1, nu = 0.2; per-bond Kn/Tv = two-end mean of the particle values), 6 KUBC
    macro-strain load cases (magnitude 1e-3) as 6 right-hand sides per specimen, a batch of B specimens per GPU.
  ellipsoids192: 192^3, seeded randomly oriented prolate ellipsoids 3:1:1 (volume of a sphere of radius 4, volume
    fraction 0.30, contrast 15, nu = 0.2), 9 load cases (6 KUBC strains + uniaxial tension along x, y, z) as 9
    right-hand sides of one specimen.
Each step forms b = -K u_p in FP64, packs FP32 coefficients, builds the preconditioner -- by default the aggregation
AMG of timing/t3d/amg3d.py (numeric setup of every specimen's hierarchies inside the step; the aggregation geometry is
built once per lattice and BC set, as the reference does), or the 3x3 block Jacobi (--precond bj) -- and runs FP32 PCG
inside FP64 iterative refinement until every system's FP64 true residual is <= 1e-8 |b|.  Synthetic data (no dataset
is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--workload spheres48|ellipsoids192]
                    [--precond amg|bj] [--inner-tol T] [--impl ours|reference]

Other workloads (one JSON line each): plain2d (cfg 1, FP64 plain CG on ten 128^2 specimens), coarse2d (cfg 3,
differentiable 2D coarse solve), serve (cfg 4, the serving stream), kernels (achieved bandwidth of the hot-path
kernels in single calls).

Under torchrun (N > 1) every rank solves its own B specimens (weak scaling, no data-path collective); the step time
is the max over ranks.  `--impl reference` times the CPU oracle (the reference's FP64 block-Jacobi PCG restated in C,
all host threads) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s at rel.res 1e-8 (mixed FP32/FP64-IR batched PCG)"
UNIT = "solves/s"
LOADS6 = ["k_xx", "k_yy", "k_zz", "k_yz", "k_xz", "k_xy"]
WORKLOADS = {
    "spheres48": dict(n=48, loads=LOADS6, micro="spheres", phi=0.25, contrast=10.0, nu=0.2,
                      label="SC 48^3 spheres r4 phi0.25 contrast10 nu0.2, 6 KUBC RHS per specimen"),
    "ellipsoids192": dict(n=192, loads=LOADS6 + ["lr_tx", "fb_ty", "tb_tz"], micro="prolate", phi=0.30,
                          contrast=15.0, nu=0.2,
                          label="SC 192^3 prolate ellipsoids 3:1:1 r4 phi0.30 contrast15 nu0.2, 6 KUBC + 3 "
                                "uniaxial tensions as 9 RHS"),
}
TOL = 1e-8


PRECONDS = {"amg": "aggregation AMG, W(1,1) cycle, one hierarchy per specimen and BC box (timing/t3d/amg3d.py, "
                   "settings of timing/t3d/problems.py:19); numeric setup inside every step",
            "bj": "3x3 block Jacobi"}


def workload_config(w, batch, n_gpus):
    """The workload (identical in the GPU arm and the reference arm); how each arm solves it goes under "method"."""
    W = WORKLOADS[w]
    n, L = W["n"], len(W["loads"])
    return {"workload": W["label"], "lattice": [n] * 3, "specimens_per_gpu": batch, "rhs_per_specimen": L,
            "systems_per_gpu": L * batch, "tol": TOL, "l2": "inputs larger than L2 (%.0f MB of FP64 coefficients per "
            "GPU)" % (batch * n ** 3 * 36 * 8 / 1e6), "parallelism": "dp%d (independent specimens per GPU)" % n_gpus}


def make_specimen(w, seed, geom, micro):
    W = WORKLOADS[w]
    n = W["n"]
    lat = geom.LatticeGeom(n, n, n, 1.0)
    rng = np.random.default_rng(seed)
    if W["micro"] == "spheres":
        ph, _ = micro.spheres(n, n, n, W["phi"], 4.0, rng, rjit=0.0)
    else:
        ph, _ = micro.prolate_ellipsoids(n, n, n, W["phi"], 4.0, rng, aspect=3.0, max_tries=60000)
    E = np.where(ph == 1, W["contrast"], 1.0)
    C = geom.iso_C(E, W["nu"])
    Kn, Tv = geom.bond_params_two_end_mean(lat, geom.sc_params_from_C(C, 0.5))
    return lat, Kn, Tv


def load_bcs(w, lat, geom):
    n = WORKLOADS[w]["n"]
    free, ups = [], []
    for ld in WORKLOADS[w]["loads"]:
        fixed, up, _ = geom.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        free.append(~fixed)
        ups.append(np.where(fixed[:, None], up, 0.0))
    return np.array(free), np.array(ups)


def load_workload(w, seeds):
    from lpm_b200 import geom, micro
    n = WORKLOADS[w]["n"]
    cache = os.path.join(tempfile.gettempdir(), "lpm_bench_cache")
    os.makedirs(cache, exist_ok=True)
    Kn, Tv = [], []
    lat = None
    for s in seeds:
        fn = os.path.join(cache, "%s_%d.npz" % (w, s))
        if os.path.exists(fn):
            d = np.load(fn)
            k, t = d["Kn"], d["Tv"]
            lat = lat or geom.LatticeGeom(n, n, n, 1.0)
        else:
            lat, k, t = make_specimen(w, s, geom, micro)
            np.savez(fn, Kn=k, Tv=t)
        Kn.append(k)
        Tv.append(t)
    free, ups = load_bcs(w, lat, geom)
    return lat, np.array(Kn), np.array(Tv), free, ups


# --------------------------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].strip().lower() == "active"})
        out.update(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=reasons, samples=len(rows))
        return out


# ------------------------------------------------------------------------------------------------ ranks
def shard_seeds(rank, batch):
    """Specimen seeds of a rank: every rank solves its own `batch` specimens (weak scaling, no shared data)."""
    return [rank * batch + j for j in range(batch)]


def max_over_ranks(ms, world, device):
    """Step time of the job: the slowest rank's (NCCL on GPUs, gloo in the CPU tests)."""
    if world <= 1:
        return float(ms)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(ms)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, systems_per_rank, steps, ms):
    """Whole-job solves/s: the systems all ranks solved over the max-over-ranks time."""
    return world * systems_per_rank * steps / (ms / 1e3)


# ------------------------------------------------------------------------------------------------ CPU side
def kmv_traffic(nsys, workload):
    """DRAM bytes per K.u launch for `nsys` systems, from the ncu capture recorded in profiles/k_sc_pair_traffic.json
    (dram__bytes_read.sum + dram__bytes_write.sum of one launch of the captured case, scaled by systems: the bytes of a
    launch grow with its systems and coefficient sets, which keep the same ratio here).  None if not recorded."""
    path = os.path.join(ROOT, "profiles", "k_sc_pair_traffic.json")
    if not os.path.exists(path):
        return None, None
    rec = json.load(open(path))
    cap = rec.get(workload)
    if not cap:
        return None, None
    return (cap["dram_bytes_read"] + cap["dram_bytes_write"]) / cap["systems"] * nsys, \
        "ncu dram bytes of one launch (%s, commit %s) scaled by systems" % (cap["case"], cap["commit"])


def cpu_solve_sample(lat, Kn, Tv, free, ups, picks, maxit=20000, threads=None):
    """FP64 block-Jacobi PCG of the CPU oracle (the reference's lin3d._pcg / solve_pcg restated in C, OpenMP) on the
    (specimen, load) pairs `picks`, at most `maxit` iterations each, with `threads` OpenMP threads (all host threads by
    default).  Returns (seconds, solves, threads, iterations of the last solve)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(threads or os.cpu_count() or 1)
    t0 = time.perf_counter()
    it = 0
    for j, l in picks:
        _, info = O.solve_pcg(lat, Kn[j], Tv[j], ~free[l], ups[l], tol=TOL, maxit=maxit)
        it = info["iters"]
    return time.perf_counter() - t0, len(picks), O.get_threads(), it


def cpu_amg_sample(lat, Kn, Tv, free, ups, j, l):
    """FP64 aggregation-AMG PCG of the reference's timing/t3d/amg3d.py (settings of timing/t3d/problems.py:19) as the
    NumPy oracle restates it, one load case: geometry, numeric setup and PCG to 1e-8.  Returns (seconds, iterations)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import amg as OA
    O.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    b = -O.sc_apply(lat, ups[l], Kn[j], Tv[j]) * free[l][:, None]
    h = OA.Hierarchy(OA.Geometry(lat, free[l]), Kn[j], Tv[j])
    _, it, _ = h.pcg(b, TOL)
    return time.perf_counter() - t0, it


def reference_picks(nspec, nload, k, per_step):
    """(specimen, load) pairs of step k of the bounded CPU sample: consecutive pairs of the whole batch, wrapping."""
    return [((k * per_step + q) // nload % nspec, (k * per_step + q) % nload) for q in range(per_step)]


def run_reference(a):
    """The reference arm: the reference's FP64 block-Jacobi PCG (coarse3d/lin3d.py:464-532, restated in C by the
    oracle) on the host cores, all threads, on a bounded sample of the same workload per step (one solve of the next
    (specimen, load) pair of the batch), same metric and config as the GPU arm."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    B = a.batch
    lat, Kn, Tv, free, ups = load_workload(a.workload, list(range(B)))
    L = len(WORKLOADS[a.workload]["loads"])
    per_step = 1
    for k in range(a.warmup):
        cpu_solve_sample(lat, Kn, Tv, free, ups, reference_picks(B, L, k, per_step))
    secs = []
    thr = 1
    for k in range(a.steps):
        s, n, thr, _ = cpu_solve_sample(lat, Kn, Tv, free, ups, reference_picks(B, L, a.warmup + k, per_step))
        secs.append(s)
    tot = sum(secs)
    value = a.steps * per_step / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * tot / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a.workload, a.batch, a.gpus),
            "method": "FP64 block-Jacobi PCG to rel. res. 1e-8 on the host cores (the C oracle restating "
                      "coarse3d/lin3d.py:464-532, OpenMP)",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port",
                             "sample": "%d solve(s) per step: the next (specimen, load) pairs of the %d x %d batch, "
                                       "FP64 block-Jacobi PCG to 1e-8" % (per_step, B, L)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def torch_sct_cg(lat, Kn, Tv, b, free, tol, check=10, maxit=50000):
    """The reference's FP64 GPU CG, restated in plain PyTorch tensor ops as coarse3d/torch_lpm3d.py:36-140 runs it
    (SCT.apply by gathers over the (N, 18) neighbour table with a zero ghost row, SCT.pcg with M = identity, a
    per-system activity mask and a host check every `check` iterations).  A comparator only: nothing of the library
    runs in it.  Kn, Tv (B, 1, N, 18), b (B, L, N, 3), free (L, N) float64 CUDA tensors.  Returns (x, iterations)."""
    import torch
    dev = b.device
    N = lat.N
    nbr = torch.as_tensor(np.where(lat.nbr >= 0, lat.nbr, N), device=dev)
    valid = torch.as_tensor(lat.valid, device=dev, dtype=torch.float64)
    ndir = torch.as_tensor(lat.ndir, device=dev, dtype=torch.float64)
    sh = torch.as_tensor(np.asarray(lat.shell), device=dev)
    slot = torch.arange(18, device=dev)
    ghost = lambda t: torch.cat([t, torch.zeros_like(t[..., :1, :])], -2)

    def apply(u):
        dL = ((u[..., :, None, :] - ghost(u)[..., nbr, :]) * ndir).sum(-1) * valid
        TdL = Tv * dL
        S = torch.stack([dL[..., :6].sum(-1), dL[..., 6:].sum(-1)], -1)[..., sh]
        TS = torch.stack([TdL[..., :6].sum(-1), TdL[..., 6:].sum(-1)], -1)[..., sh]
        Sq = ghost(S)[..., nbr, slot]
        TSq = ghost(TS)[..., nbr, slot]
        F = (2 * Kn * dL + 0.5 * (TS + TSq) + 0.5 * Tv * (S + Sq)) * valid
        return F @ ndir

    fr = free[..., None]
    x = torch.zeros_like(b)
    r = b.clone()
    bn = b.flatten(-2).norm(dim=-1)
    bn = torch.where(bn > 0, bn, torch.ones_like(bn))
    p = r.clone()
    rz = (r * r).flatten(-2).sum(-1)
    act = torch.ones_like(rz)
    it = 0
    for it in range(1, maxit + 1):
        Ap = apply(p) * fr
        pAp = (p * Ap).flatten(-2).sum(-1)
        alpha = torch.where(pAp != 0, rz / pAp, torch.zeros_like(rz)) * act
        x = x + alpha[..., None, None] * p
        r = r - alpha[..., None, None] * Ap
        if it % check == 0:
            act = ((r.flatten(-2).norm(dim=-1) / bn) > tol).to(b.dtype)
            if not bool(act.any()):
                break
        rz2 = (r * r).flatten(-2).sum(-1)
        beta = torch.where(rz != 0, rz2 / rz, torch.zeros_like(rz))
        rz = rz2
        p = r + beta[..., None, None] * p
    return x, it


# ---------------------------------------------------------------------------------------------- serving stream
SERVE_2D = [64, 128, 256, 512]
SERVE_3D = [24, 48, 72, 96]


def serve_requests(n_req, seed):
    """The serving mix: 60% 2D square boxes (n in {64..512}^2, Gaussian random field), 40% 3D SC boxes (n in
    {24..96}^3, random field or spheres), inclusion fraction U(0.15, 0.40), contrast U(5, 15), 1-6 (2D) or 1-9 (3D)
    load cases drawn from the load sets.  Returns a list of (dim, shape, Kn, Tv, free (L,N,d), up (L,N,d))."""
    from lpm_b200 import geom, micro
    rng = np.random.default_rng(seed)
    cache = os.path.join(tempfile.gettempdir(), "lpm_bench_cache")
    os.makedirs(cache, exist_ok=True)
    out = []
    for _ in range(n_req):
        is2d = rng.random() < 0.6
        phi, contrast = rng.uniform(0.15, 0.40), rng.uniform(5.0, 15.0)
        mseed = int(rng.integers(1 << 30))
        if is2d:
            n = int(rng.choice(SERVE_2D))
            lat = geom.SquareLattice(n, n, 1.0)
            ph = micro.grf_two_phase(n, n, 6.0, phi, mseed)
            C = geom.iso_C2d(np.where(ph == 1, contrast, 1.0), 0.25, plane="stress")
            Kn, Tv = geom.bond_params_two_end_mean(lat, geom.square_params_from_C(C))
            loads = list(rng.choice(geom.LOADS2D, size=int(rng.integers(1, 7)), replace=False))
            free, up = [], []
            for ld in loads:
                fixed, u, _ = geom.prescribed2d(ld, lat.x, lat.ij, n, n, 1, 1.0)
                free.append(np.repeat(~fixed[:, None], 2, 1))
                up.append(np.where(fixed[:, None], u, 0.0))
            out.append((2, (n, n), Kn, Tv, np.array(free), np.array(up)))
        else:
            n = int(rng.choice(SERVE_3D))
            lat = geom.LatticeGeom(n, n, n, 1.0)
            if rng.random() < 0.5:
                ph, _ = micro.grf3(n, n, n, 4.0, phi, np.random.default_rng(mseed))
            else:
                ph, _ = micro.spheres(n, n, n, phi, 4.0, np.random.default_rng(mseed), rjit=0.0)
            C = geom.iso_C(np.where(ph == 1, contrast, 1.0), 0.2)
            Kn, Tv = geom.bond_params_two_end_mean(lat, geom.sc_params_from_C(C, 0.5))
            loads = list(rng.choice(geom.LOADS, size=int(rng.integers(1, 10)), replace=False))
            free, up = [], []
            for ld in loads:
                fixed, u, _ = geom.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
                free.append(np.repeat(~fixed[:, None], 3, 1))
                up.append(np.where(fixed[:, None], u, 0.0))
            out.append((3, (n,) * 3, Kn, Tv, np.array(free), np.array(up)))
    return out


def run_serve(a):
    """Serving stream: continuous batching vs sequential plain FP64 CG, on one GPU (rank 0 only)."""
    import threading
    import torch
    from lpm_b200 import _lib, core, geom, serve
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    n_req = a.requests
    specs = serve_requests(n_req, 1234)
    nsolve = sum(sp[4].shape[0] for sp in specs)
    srv = serve.Server(device=dev, rmax=9, rmax2d=6, max_slots=8, tol=TOL, inner_tol=a.inner_tol,
                       idle_release_s=1e9, amg3d=a.precond == "amg")

    def stream(arrivals):
        reqs = [serve.Request(*sp) for sp in specs]
        t0 = time.perf_counter()
        done = [None]

        def feed():
            for r, t in zip(reqs, arrivals):
                dt = t0 + t - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                r.arrival = time.perf_counter()
                srv.submit(r)

        th = threading.Thread(target=feed)
        th.start()
        srv.done.clear()
        srv.wait_all(n_req, timeout=3600)
        th.join()
        t1 = max(r.done for r in reqs)
        return reqs, t1 - t0

    try:
        for _ in range(max(a.warmup, 1)):            # warm-up: creates and autotunes the buckets
            stream([0.0] * n_req)
        reqs_cap, t_cap = stream([0.0] * n_req)      # capacity: everything at t = 0 (saturated)
        cap = n_req / t_cap
        lat_cap = serve.latency_stats(reqs_cap)
        rate = a.load_factor * cap
        gaps = np.random.default_rng(7).exponential(1.0 / rate, n_req)
        arrivals = np.cumsum(gaps) - gaps[0]
        sampler = ClockSampler(dev.index or 0)
        sampler.start()
        for b in srv.buckets.values():
            b.rounds, b.busy_s, b.admit_s, b.inner_iters = 0, 0.0, 0.0, 0
        reqs, t_run = stream(list(arrivals))
        clocks = sampler.stop()
        bstats = serve.bucket_stats(srv)
        ok = all(r.status == 0 and (r.relres <= TOL).all() for r in reqs)
        lat_ms = serve.latency_stats(reqs)
    finally:
        srv.close()

    # sequential plain FP64 CG on the same GPU, same requests and arrival times (FIFO, one request at a time)
    seq_t, seq_by = [], {}
    for sp in specs:
        dim, shape, Kn, Tv, free, up = sp
        lat = geom.LatticeGeom(*shape, 1.0) if dim == 3 else geom.SquareLattice(*shape, 1.0)
        dl = core.DeviceLattice(lat, dev)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        Kt, Tt = torch.as_tensor(Kn, device=dev), torch.as_tensor(Tv, device=dev)
        fr = torch.as_tensor(free.astype(np.float64), device=dev)
        ut = torch.as_tensor(up, device=dev) * (1 - fr)
        b = -core.kmv(dl, ut, Kt, Tt) * fr
        if dim == 3:
            K64, T64 = core.pack(Kt[None], torch.float64), core.pack(Tt[None], torch.float64)
            x, info = core.cg(dl, K64, T64, b, free=fr, tol=TOL, maxit=100000, check=1, poll=20,
                              layout=_lib.LAYOUT_SOA, rhs_per_set=b.shape[0])
        else:
            x, info = core.cg(dl, Kt, Tt, b, free=fr, tol=TOL, maxit=100000, check=1, poll=20)
        (ut + x).cpu()
        seq_t.append(time.perf_counter() - t0)
        seq_by.setdefault("%dD %d" % (dim, shape[0]), []).append(round(seq_t[-1], 3))
    end, seq_lat = 0.0, []
    for t_arr, t_solve in zip(arrivals, seq_t):
        start = max(t_arr, end)
        end = start + t_solve
        seq_lat.append(end - t_arr)
    seq_lat = np.array(seq_lat)
    line = {"metric": "serving capacity solves/s at rel.res 1e-8 (continuous batching), p50/p99 latency at 0.7 load",
            "value": nsolve / t_cap, "unit": UNIT, "n_gpus": 1, "steps": 1, "warmup": max(a.warmup, 1),
            "ms_per_step": t_cap * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded random-field / sphere microstructures)",
            "config": {"workload": "serving mix: 60% 2D square n in {64,128,256,512}^2, 40% 3D SC n in {24,48,72,96}^3, "
                                   "phi U(0.15,0.40), contrast U(5,15), 1-6 / 1-9 load cases",
                       "requests": n_req, "systems": nsolve, "arrival": "Poisson, rate %.3f req/s = %.2f x measured "
                       "capacity %.3f req/s" % (rate, a.load_factor, cap), "tol": TOL,
                       "buckets": "per lattice size, up to 8 specimens x 9 systems, HBM budget 60% of free memory",
                       "inner_solvers": ("3D on the standard load boxes: AMG-PCG (inner tol 1e-4); other 3D and 2D: "
                                         "block-Jacobi PCG (inner tol %g)" % a.inner_tol) if a.precond == "amg" else
                                        "block-Jacobi PCG (inner tol %g)" % a.inner_tol},
            "latency_ms": lat_ms, "poisson_run": {"solves_per_s": nsolve / t_run, "seconds": t_run,
                                                    "requests_per_s": n_req / t_run},
            "capacity_run": {"requests_per_s": cap, "seconds": t_cap, "latency_ms": lat_cap},
            "all_converged": bool(ok), "buckets": bstats,
            "clocks": clocks,
            "sequential_fp64_cg": {"solves_per_s": nsolve / (sum(seq_t)), "p50_ms": float(np.percentile(seq_lat, 50)
                                   * 1e3), "p99_ms": float(np.percentile(seq_lat, 99) * 1e3),
                                   "path": "plain FP64 CG per request (fused FP64 operator in 3D), FIFO",
                                   "seconds_by_size": seq_by}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------ 2D configurations
def plain2d_specimens(seeds, n=128):
    """2D 128^2 square lattice, Gaussian random field (corr 6, phi 0.30), E 1 / 10, nu 0.25 plane stress, two-end
    mean bonds, uniaxial tension u_x = 1e-3 (n-1) on the right column (left column u_x = 0, corner pinned)."""
    from lpm_b200 import geom, micro
    lat = geom.SquareLattice(n, n, 1.0)
    Kn, Tv = [], []
    for sd in seeds:
        ph = micro.grf_two_phase(n, n, 6.0, 0.30, sd)
        C = geom.iso_C2d(np.where(ph == 1, 10.0, 1.0), 0.25, plane="stress")
        k, t = geom.bond_params_two_end_mean(lat, geom.square_params_from_C(C))
        Kn.append(k)
        Tv.append(t)
    fixed, up, _ = geom.uniaxial_tension_2d(lat, 1e-3)
    return lat, np.array(Kn), np.array(Tv), fixed, up


def run_plain2d(a):
    """cfg 1: FP64 unpreconditioned CG to rel. residual 1e-10 on ten 128^2 specimens (one batched solve per step)."""
    import torch
    from lpm_b200 import _lib as L, core
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    seeds = list(range(10))
    lat, Kn_h, Tv_h, fixed, up_h = plain2d_specimens(seeds)
    dl = core.DeviceLattice(lat, dev)
    Kn, Tv = torch.as_tensor(Kn_h, device=dev), torch.as_tensor(Tv_h, device=dev)
    free = torch.as_tensor((~fixed).astype(np.float64), device=dev)
    up = torch.as_tensor(np.where(fixed, up_h, 0.0), device=dev)
    B = len(seeds)

    def step(Kn, Tv, free, up, engine=L.ENGINE_AUTO):
        b = -core.kmv(dl, up[None].expand(B, -1, -1), Kn, Tv) * free
        x, info = core.cg(dl, Kn, Tv, b, free=free, tol=1e-10, maxit=200000, check=1, poll=50, precheck=True,
                          engine=engine)
        return up + x, info

    for _ in range(max(a.warmup, 3)):
        u, info = step(Kn, Tv, free, up)
    torch.cuda.synchronize(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    ev0.record()
    for _ in range(a.steps):
        u, info = step(Kn, Tv, free, up)
    ev1.record()
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    # end to end: host arrays in, host solution out
    Kp, Tp = torch.as_tensor(Kn_h).pin_memory(), torch.as_tensor(Tv_h).pin_memory()
    out = torch.empty((B, lat.N, 2), dtype=torch.float64).pin_memory()
    torch.cuda.synchronize(dev)
    ev0.record()
    for _ in range(a.steps):
        uu, _ = step(Kp.to(dev, non_blocking=True), Tp.to(dev, non_blocking=True), free, up)
        out.copy_(uu, non_blocking=True)
    ev1.record()
    torch.cuda.synchronize(dev)
    ms_e2e = ev0.elapsed_time(ev1)
    # comparator: the same solves on the graph-launched engine (one launch per step, host polls)
    engine = "persistent" if L.load().lpm_cg_persistent_fits(dl.ref, core._batch(B, 1, B), L.LPM_F64) else "launched"
    step(Kn, Tv, free, up, L.ENGINE_LAUNCHED)
    torch.cuda.synchronize(dev)
    ev0.record()
    for _ in range(a.steps):
        _, linfo = step(Kn, Tv, free, up, L.ENGINE_LAUNCHED)
    ev1.record()
    torch.cuda.synchronize(dev)
    ms_launched = ev0.elapsed_time(ev1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    _, cinfo = O.sq_solve_cg(lat, Kn_h[0], Tv_h[0], fixed, up_h, tol=1e-10)
    cpu_s = time.perf_counter() - t0
    its = info.iters
    bytes_per_it = B * lat.N * (128 + 32)            # FP64 2D K.u: Kn+Tv (2*8*8 B) + u, f (2*2*8 B) per particle
    line = {"metric": "solves/s at rel.res 1e-10 (plain FP64 CG, 2D 128^2)", "value": B * a.steps / (ms / 1e3),
            "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian random fields, shapes of the 128^2 config)",
            "config": {"workload": "2D square 128^2 GRF corr6 phi0.30 contrast10 nu0.25 plane stress, uniaxial "
                                   "tension, FP64 plain CG to 1e-10 (cg2plain semantics)", "specimens": B,
                       "l2": "L2-resident (%.1f MB of FP64 coefficients)" % (Kn_h.nbytes * 2 / 1e6),
                       "engine": engine},
            "iters_mean": float(its.mean()), "all_converged": bool((info.status == 0).all()),
            "kmv_effective_gbs": None,
            "e2e": {"value": B * a.steps / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(Kp.numel() * 16),
                    "d2h_bytes_per_step": int(out.numel() * 8)},
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": UNIT, "cores": O.get_threads(), "kind": "port",
                             "sample": "specimen 0 by the C oracle's plain CG (timing/t2d/cg2plain.py:11-68), "
                                       "%d iterations, %.2f s" % (cinfo["iters"], cpu_s)},
            "launched_engine": {"solves_per_s": B * a.steps / (ms_launched / 1e3),
                                "iters_mean": float(linfo.iters.mean())},
            "clocks": clocks}
    line["kmv_effective_gbs"] = bytes_per_it * float(its.max()) / (ms / a.steps / 1e3) / 1e9
    print(json.dumps(line), flush=True)


def run_coarse2d(a):
    """cfg 3: differentiable coarse 2D solve (128^2 coarse from 256^2 fine at s = 2), 3 loads, MSE loss against a
    seeded target; forward + backward time, gradient vs central finite differences on 64 random bonds (FP64)."""
    import torch
    from lpm_b200 import geom, micro
    from lpm_b200 import torch_lpm as T2
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    nf, s = 256, 2
    nc = nf // s
    ph = micro.grf_two_phase(nf, nf, 6.0, 0.30, 3)
    Cpix = geom.iso_C2d(np.where(ph == 1, 10.0, 1.0), 0.25, plane="stress")
    model = T2.CoarseT(nc, nc, s, 1.0, device=dev, loads=["lr_tx", "tb_ty", "tb_sx"])
    lat = model.lat
    cp = geom.cell_params_from_C6(geom.voigt_cells2d(Cpix, nf, nf, s))
    K0, T0 = geom.bond_params_from_cells2d(lat, cp)
    rng = np.random.default_rng(11)
    q = np.where(lat.valid, lat.nbr, 0)
    opp = np.repeat(lat.opp[None, :], lat.N, 0)

    def lognormal_sym(rg):
        z = rg.standard_normal((lat.N, 8))
        z = np.where(np.arange(8)[None, :] % 2 == 0, z, z[q, opp])      # one factor per undirected bond
        return np.exp(0.2 * z)
    f0 = lognormal_sym(rng).astype(np.float32).astype(np.float64)
    target = model.run(torch.as_tensor(K0 * lognormal_sym(rng), device=dev)[None],
                       torch.as_tensor(T0, device=dev)[None])
    tgt = {ld: v["u"].detach() for ld, v in target.items()}
    Kb = torch.as_tensor(K0 * f0, device=dev)[None]
    Tb = torch.as_tensor(T0, device=dev)[None]
    qt, ot = torch.as_tensor(q, device=dev), torch.as_tensor(opp, device=dev)
    valid = torch.as_tensor(lat.valid, device=dev, dtype=torch.float64)

    def loss_of(th):
        Kn = Kb * torch.exp(0.5 * (th + th[:, qt, ot])) * valid
        out = model.run(Kn, Tb)
        return sum(((out[ld]["u"] - tgt[ld]) ** 2).mean() for ld in tgt)

    th = torch.zeros((1, lat.N, 8), dtype=torch.float64, device=dev, requires_grad=True)
    for _ in range(max(a.warmup, 3)):
        th.grad = None
        loss_of(th).backward()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        th.grad = None
        L = loss_of(th)
        L.backward()
    torch.cuda.synchronize(dev)
    fb_ms = (time.perf_counter() - t0) / a.steps * 1e3
    # gradient check at a tighter solve tolerance, so that the differences of two solves resolve h = 1e-6
    model.tol = 1e-14
    th.grad = None
    loss_of(th).backward()
    g = th.grad.detach().clone()
    # The finite difference of a loss evaluated through an iterative solve carries the solve's own error: its noise
    # floor is |L(tol) - L(tol/10)| / h (the loss moved by tightening the solve), next to the rounding floor
    # eps |L| / h.  Bonds whose gradient is far above the floor are where the FD value can pin the adjoint.
    with torch.no_grad():
        L14 = float(loss_of(th))
        model.tol = 1e-15
        L15 = float(loss_of(th))
        model.tol = 1e-14
    h = 1e-6
    floor = max(abs(L14 - L15), 2.2e-16 * abs(L14)) / h
    # central differences on 64 random undirected bonds (perturbing theta of the (i, k) slot, k even)
    ii = rng.choice(np.flatnonzero(lat.valid[:, 0]), 64, replace=False)
    kk = rng.choice(np.arange(0, 8, 2), 64)
    errs, abs_err, mags = [], [], []
    with torch.no_grad():
        for i, k in zip(ii, kk):
            e = torch.zeros_like(th)
            e[0, i, k] = h
            fd = (float(loss_of(th + e)) - float(loss_of(th - e))) / (2 * h)
            ad = float(g[0, i, k])
            errs.append(abs(fd - ad) / max(abs(fd), abs(ad), 1e-300))
            abs_err.append(abs(fd - ad))
            mags.append(abs(ad))
    errs, abs_err, mags = np.array(errs), np.array(abs_err), np.array(mags)
    above = mags > 100 * floor
    line = {"metric": "forward+backward ms (differentiable 2D coarse solve, 128^2, 3 loads)", "value": fb_ms,
            "unit": "ms", "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": fb_ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded GRF 256^2 fine, Voigt cells s = 2, lognormal(0.2) per undirected bond, "
                    "parameters rounded to FP32)",
            "config": {"workload": "2D coarse 128^2 from 256^2 at s = 2, loads lr_tx tb_ty tb_sx, MSE loss vs "
                                   "seeded target displacements, adjoint gradient w.r.t. log bond stiffness",
                       "solve_tol": 1e-12, "gradient_check_solve_tol": 1e-14},
            "gradient_check": {"bonds": 64, "h": h, "rel_err_max": float(errs.max()),
                               "rel_err_median": float(np.median(errs)),
                               "fd_noise_floor": floor, "abs_err_max": float(abs_err.max()),
                               "abs_err_max_over_floor": float(abs_err.max() / floor),
                               "bonds_above_100x_floor": int(above.sum()),
                               "rel_err_max_above_100x_floor": float(errs[above].max()) if above.any() else None,
                               "gradient_max": float(mags.max())},
            "loss": float(L.detach())}
    print(json.dumps(line), flush=True)


def run_kernels(a):
    """Achieved bandwidth of the hot-path kernels outside the solver loop: CUDA events around single C-ABI calls (one
    kernel each, except where named), the L2 flushed by a 256 MB write before every timed call, mean of 10 calls after
    3 warm-up calls.  Bytes are algorithmic (every input read once, every output written once)."""
    import torch
    from lpm_b200 import _lib as L
    from lpm_b200 import core, geom, micro
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    T = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), device=dev, dtype=dt)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(pp))["hbm_gbs"] if os.path.exists(pp) else 6650.0
    rows = []

    def timed(fn, reps=10):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        tot = 0.0
        for _ in range(reps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize(dev)
            tot += e0.elapsed_time(e1)
        return tot / reps

    def row(row_id, what, kernels, fn, nbytes):
        ms = timed(fn)
        gbs = nbytes / (ms * 1e-3) / 1e9
        rows.append({"row": row_id, "what": what, "kernels": kernels, "ms": ms, "bytes": int(nbytes),
                     "achieved_gbs": gbs, "frac": gbs / peak})

    # 3D: 48^3 two-phase microstructure, 16 coefficient sets x 6 systems
    n, S, R = 48, 16, 6
    lat = geom.LatticeGeom(n, n, n, 1.0)
    rng = np.random.default_rng(0)
    C = geom.iso_C(np.where(rng.random(lat.N) < 0.3, 10.0, 1.0), 0.2)
    Kn, Tv = geom.bond_params_two_end_mean(lat, geom.sc_params_from_C(C, 0.5))
    dl = core.DeviceLattice(lat, dev)
    N = lat.N
    Kd = T(Kn)[None].expand(S, -1, -1).contiguous()
    Td = T(Tv)[None].expand(S, -1, -1).contiguous()
    K64, T64 = core.pack(Kd, torch.float64), core.pack(Td, torch.float64)
    u64 = torch.randn(S * R, N, 3, device=dev, dtype=torch.float64)
    u1 = u64[:R].contiguous()
    lam = torch.randn(R, N, 3, device=dev, dtype=torch.float64)
    row("a3", "SC K.u FP64 packed, 48^3 x 16 sets x 6", "k_sc_pair<double> (FP64 lean)",
        lambda: core.kmv(dl, u64, K64, T64, layout=L.LAYOUT_SOA, rhs_per_set=R), S * N * 288 + S * R * N * 48)
    row("a4", "SC K.u FP64 reference layout, 48^3 x 6", "k_shell_sums + k_apply",
        lambda: core.kmv(dl, u1, Kd[:1], Td[:1]), N * 288 + R * N * 48)
    row("a11", "SC block Jacobi, 48^3 x 16 sets (FP64 in, FP32 out)", "k_block_jacobi",
        lambda: core.block_jacobi(dl, Kd, Td, torch.float32), S * N * (288 + 36))
    row("a12", "SC bond gradient, 48^3 x 6 systems of 1 set", "bond-gradient kernels",
        lambda: core.bond_grad(dl, u1, lam, Kd[:1], Td[:1]), 2 * N * 288 + 2 * R * N * 24)
    row("a14", "SC particle stress, 48^3 x 6", "stress kernels",
        lambda: core.stress(dl, u1, Kd[:1], Td[:1]), N * 288 + R * N * (24 + 48))
    # 2D: 512^2 random-field specimen
    n2 = 512
    lat2 = geom.SquareLattice(n2, n2, 1.0)
    C2 = geom.iso_C2d(np.where(micro.grf_two_phase(n2, n2, 6.0, 0.30, 0) == 1, 10.0, 1.0), 0.25, plane="stress")
    k2, t2 = geom.bond_params_two_end_mean(lat2, geom.square_params_from_C(C2))
    dl2 = core.DeviceLattice(lat2, dev)
    N2 = lat2.N
    for dt, es, nm in ((torch.float64, 8, "FP64"), (torch.float32, 4, "FP32")):
        for S2, R2 in ((8, 1), (1, 6)):
            K2 = core.pack(T(k2)[None].expand(S2, -1, -1).contiguous(), dt)
            T2 = core.pack(T(t2)[None].expand(S2, -1, -1).contiguous(), dt)
            u2 = torch.randn(S2 * R2, N2, 2, device=dev, dtype=dt)
            kern = "k_sq_multi" if (es == 4 and R2 > 1) else "k_sq_fused"
            row("a5", "SQ K.u %s packed, 512^2 x %d sets x %d" % (nm, S2, R2), kern,
                lambda: core.kmv(dl2, u2, K2, T2, layout=L.LAYOUT_SOA, rhs_per_set=R2),
                S2 * N2 * 16 * es + S2 * R2 * N2 * 4 * es)
    print(json.dumps({"metric": "achieved GB/s of the hot-path kernels (single calls, L2 flushed)", "unit": "GB/s",
                      "peak": peak, "peak_source": "measured" if os.path.exists(pp) else "fallback",
                      "rows": rows}), flush=True)


# ------------------------------------------------------------------------------------------------- GPU side
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=None, help="specimens per GPU (default 16 for spheres48, 1 else)")
    ap.add_argument("--workload", default="spheres48", choices=sorted(WORKLOADS) + ["serve", "plain2d", "coarse2d", "kernels"])
    ap.add_argument("--requests", type=int, default=40, help="serving stream: number of requests")
    ap.add_argument("--load-factor", type=float, default=0.7, help="serving stream: arrival rate / capacity")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 CG comparator")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--precond", default="amg", choices=sorted(PRECONDS),
                    help="inner PCG preconditioner of the 3D workloads (default: AMG)")
    ap.add_argument("--tiles", default=None, help="pin the FP32 operator's z-chunk and variant, e.g. 48,staged "
                    "(default: autotune)")
    ap.add_argument("--inner-tol", type=float, default=None,
                    help="inner FP32 solve tolerance (default 1e-4 with AMG, 1e-3 with block Jacobi)")
    a = ap.parse_args()
    if a.inner_tol is None:  # serving: the block-Jacobi buckets' value (AMG buckets use 1e-4 themselves)
        a.inner_tol = 1e-4 if a.precond == "amg" and a.workload != "serve" else 1e-3
    if a.batch is None:
        a.batch = 16 if a.workload == "spheres48" else 1
    if a.workload == "serve":
        return run_serve(a)
    if a.workload == "plain2d":
        return run_plain2d(a)
    if a.workload == "coarse2d":
        return run_coarse2d(a)
    if a.workload == "kernels":
        return run_kernels(a)
    if a.impl == "reference":
        return run_reference(a)

    import torch
    import torch.distributed as dist
    from lpm_b200 import _lib, core

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    seeds = shard_seeds(rank, a.batch)
    lat, Kn_h, Tv_h, free_h, ups_h = load_workload(a.workload, seeds)
    B = a.batch
    Lc = len(WORKLOADS[a.workload]["loads"])
    dl = core.DeviceLattice(lat, dev)
    Kn = torch.as_tensor(Kn_h, device=dev)[:, None]          # (B, 1, N, 18)
    Tv = torch.as_tensor(Tv_h, device=dev)[:, None]
    free = torch.as_tensor(free_h, device=dev, dtype=torch.float64)      # (6, N)
    ups = torch.as_tensor(ups_h, device=dev)[None].expand(B, -1, -1, -1).contiguous()   # (B, 6, N, 3)
    nsys = B * Lc

    # tile tuning of the FP32 operator for this batch shape (the library records it for later launches); --tiles
    # pins them instead (a profiling aid: the same kernel configuration at a smaller batch)
    if a.tiles:
        zc, var = a.tiles.split(",")
        tiles = (int(zc), {"staged": 0, "lean": 1}[var])
        core.tune_set(dl, nsys, Lc, *tiles)
    else:
        tiles = core.autotune(dl, core.pack(Kn[:, 0], torch.float32), core.pack(Tv[:, 0], torch.float32), nsys, Lc,
                              with_variant=True)

    amgb = None
    if a.precond == "amg":
        # geometry of the hierarchies (aggregation, transfers): once per lattice and BC set, like the neighbour lists
        from lpm_b200 import amg as GA
        amgb = GA.AmgBatch(dl, nsys, Lc, free_h, **GA.AMG_CFG)

    def step(Kn, Tv, free, ups, prof=None):
        if amgb is None:
            b = -core.kmv(dl, ups, Kn, Tv) * free[None, :, :, None]
            x, info = core.ir(dl, Kn, Tv, b, free=free, tol=TOL, inner_tol=a.inner_tol, prof=prof)
            return ups + x, info
        # FP64 coefficients packed once per step: b = -K u_p and the refinement residuals run on the TMA operator
        K64, T64 = core.pack(Kn[:, 0], torch.float64), core.pack(Tv[:, 0], torch.float64)
        b = -core.kmv(dl, ups, K64, T64, layout=_lib.LAYOUT_SOA, rhs_per_set=Lc) * free[None, :, :, None]
        # per-specimen numeric setup (block inverses, rho, Galerkin products, coarse inverse) is part of every step
        K32, T32 = core.pack(Kn[:, 0], torch.float32), core.pack(Tv[:, 0], torch.float32)
        amgb.setup(K32, T32, core.block_jacobi(dl, Kn[:, 0], Tv[:, 0], torch.float32))
        x, info = amgb.ir(K64, T64, b.reshape(nsys, lat.N, 3), tol=TOL, inner_tol=a.inner_tol, prof=prof,
                          packed=True)
        return ups + x.reshape(ups.shape), info

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(max(a.warmup, 1)):
        u, info = step(Kn, Tv, free, ups)
    barrier()

    sampler = ClockSampler(local)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # one event per step boundary (recorded between steps, outside every captured graph): the per-step times
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    cap0 = _lib.graph_stats()
    barrier()
    ev0.record()
    infos = []
    for k in range(a.steps):
        evs[k].record()
        u, info = step(Kn, Tv, free, ups)
        infos.append(info)
    evs[a.steps].record()
    ev1.record()
    barrier()
    clocks = sampler.stop()
    cap1 = _lib.graph_stats()
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(a.steps)]
    graphs = {"captured_in_timed_region": cap1[0] - cap0[0], "evicted_in_timed_region": cap1[2] - cap0[2],
              "held_after": cap1[1]}
    # per-launch operator timings come from one more step outside the timed region (timing every launch with events
    # turns off the CUDA-graph replay of the iteration blocks)
    prof = core.new_prof()
    step(Kn, Tv, free, ups, prof)
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world, dev)
    value = job_throughput(world, nsys, a.steps, ms)
    ok = all((i.status == 0).all() and (i.relres <= TOL).all() for i in infos)
    iters = np.concatenate([i.iters for i in infos])

    # ---- roofline of the dominant kernel (FP32 K.u inside the inner PCG), from CUDA events in the timed region
    Nn = lat.N
    alg_bytes = B * Nn * 144 + nsys * Nn * 24            # FP32: Kn+Tv (2*18*4 B) per particle per set, u+f per RHS
    full_ms = prof[2] / max(prof[3], 1.0)
    all_ms = prof[0] / max(prof[1], 1.0)
    import json as _json
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = _json.load(open(pp))
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = alg_bytes / (full_ms / 1e3) / 1e9 if prof[3] > 0 else None
    traffic, traffic_src = kmv_traffic(nsys, a.workload)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                "kernel": "k_sc_pair: pair-packed FP32 SC K.u with the p.Ap epilogue (all %d systems, %d coefficient "
                          "sets) in the inner PCG" % (nsys, B),
                "traffic_source": traffic_src,
                "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": full_ms, "avg_launch_ms_all": all_ms,
                "launches_profiled": int(prof[1]), "peak_source": peak_src,
                "timing_source": "CUDA events around every operator launch of one extra step outside the timed region"}

    # ---- end to end through the public API with host buffers (pinned), copies inside the timed region
    Kn_pin = torch.as_tensor(Kn_h).pin_memory()
    Tv_pin = torch.as_tensor(Tv_h).pin_memory()
    fr_pin = torch.as_tensor(free_h, dtype=torch.float64).pin_memory()
    up_pin = torch.as_tensor(ups_h).pin_memory()
    u_host = torch.empty((B, Lc, Nn, 3), dtype=torch.float64).pin_memory()
    h2d = Kn_pin.numel() * 8 + Tv_pin.numel() * 8 + fr_pin.numel() * 8 + up_pin.numel() * 8
    d2h = u_host.numel() * 8

    # Copies run on their own stream, double-buffered: step k+1's inputs go up while step k computes, and step k's
    # solution comes down while step k+1 computes.  Every step still moves its own inputs and result.
    cstream = torch.cuda.Stream(dev)
    dbuf = [[torch.empty(t.shape, dtype=t.dtype, device=dev) for t in (Kn_pin, Tv_pin, fr_pin, up_pin)]
            for _ in range(2)]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_used = [torch.cuda.Event() for _ in range(2)]

    def upload(j):
        with torch.cuda.stream(cstream):
            cstream.wait_event(ev_used[j])              # the step that read this buffer set has finished
            for d, h in zip(dbuf[j], (Kn_pin, Tv_pin, fr_pin, up_pin)):
                d.copy_(h, non_blocking=True)
            ev_in[j].record(cstream)

    def e2e_run(nsteps):
        main = torch.cuda.current_stream(dev)
        for j in range(2):
            ev_used[j].record(main)
        upload(0)
        for k in range(nsteps):
            j = k & 1
            main.wait_event(ev_in[j])
            if k + 1 < nsteps:
                upload(1 - j)
            kd, td, fd, ud = dbuf[j]
            uu, _ = step(kd[:, None], td[:, None], fd, ud[None].expand(B, -1, -1, -1))
            ev_used[j].record(main)
            with torch.cuda.stream(cstream):
                cstream.wait_event(ev_used[j])
                u_host.copy_(uu, non_blocking=True)
                uu.record_stream(cstream)
        main.wait_stream(cstream)

    e2e_run(2)
    barrier()
    ev0.record()
    e2e_run(a.steps)
    ev1.record()
    barrier()
    ms_e2e = max_over_ranks(ev0.elapsed_time(ev1), world, dev)
    e2e = {"value": job_throughput(world, nsys, a.steps, ms_e2e), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h)}

    # ---- comparator: plain FP64 GPU CG on the same batch with this library's fastest FP64 path (packed
    # coefficients, TMA-fed fused operator, same engine), packing included; accuracy vs FP64 PCG to 1e-12
    b = -core.kmv(dl, ups, Kn, Tv) * free[None, :, :, None]
    fp64_cg = None
    if not a.no_fp64:
        torch.cuda.synchronize(dev)
        ev0.record()
        K64, T64 = core.pack(Kn[:, 0], torch.float64), core.pack(Tv[:, 0], torch.float64)
        x64, i64 = core.cg(dl, K64, T64, b, free=free, tol=TOL, maxit=50000, check=1, poll=20,
                           layout=_lib.LAYOUT_SOA, rhs_per_set=Lc)
        ev1.record()
        torch.cuda.synchronize(dev)
        del K64, T64, x64
        fp64_cg = {"solves_per_s": nsys / (ev0.elapsed_time(ev1) / 1e3), "iters_mean": float(i64.iters.mean()),
                   "all_converged": bool((i64.status == 0).all()),
                   "path": "FP64 plain CG, packed coefficients, FP64 instantiation of the pair operator (k_sc_pair<double>, lean)"}
    M64 = core.block_jacobi(dl, Kn[0:1, 0], Tv[0:1, 0], torch.float64)
    xr, ir_ = core.cg(dl, Kn[0:1], Tv[0:1], b[0:1], Minv=M64, free=free, tol=1e-12, maxit=20000, check=1, poll=20)
    uref = ups[0:1] + xr
    sref = core.stress(dl, uref, Kn[0:1], Tv[0:1])
    smix = core.stress(dl, u[0:1], Kn[0:1], Tv[0:1])
    fr4 = free[None, :, :, None]
    du = (((u[0:1] - uref) * fr4) ** 2).sum((-1, -2)).sqrt() / ((uref * fr4) ** 2).sum((-1, -2)).sqrt()
    ds = ((smix - sref) ** 2).sum((-1, -2)).sqrt() / (sref ** 2).sum((-1, -2)).sqrt()
    accuracy = {"vs": "FP64 block-Jacobi PCG to 1e-12 (GPU, parity-tested against the CPU oracle)",
                "u_rel_l2_per_load": [float(v) for v in du[0].cpu()], "stress_rel_l2_per_load":
                    [float(v) for v in ds[0].cpu()]}

    # ---- comparator: the reference's own FP64 GPU CG algorithm (SCT.pcg with M = identity, plain PyTorch tensor
    # ops) on a sample of the batch, timed with CUDA events on the same GPU
    torch_cg = None
    if not a.no_fp64 and a.workload == "spheres48":
        nb = min(B, 4)
        torch.cuda.synchronize(dev)
        ev0.record()
        _, it_t = torch_sct_cg(lat, Kn[:nb], Tv[:nb], b[:nb], free, TOL)
        ev1.record()
        torch.cuda.synchronize(dev)
        torch_cg = {"solves_per_s": nb * Lc / (ev0.elapsed_time(ev1) / 1e3), "iterations": it_t,
                    "sample": "%d specimens x %d loads" % (nb, Lc),
                    "path": "the algorithm of coarse3d/torch_lpm3d.py:36-140 (SCT.apply by tensor gathers, SCT.pcg "
                            "with M = identity, check every 10 iterations) restated in plain PyTorch"}

    cpu = None
    cpu_extra = None
    if rank == 0 and world == 1 and not a.no_cpu:
        if a.workload == "spheres48":
            picks = [(0, 0), (0, 1)]
            secs, n, thr, _ = cpu_solve_sample(lat, Kn_h, Tv_h, free_h, ups_h, picks)
            cpu = {"value": n / secs, "unit": UNIT, "cores": thr, "kind": "port",
                   "sample": "2 load cases (k_xx, k_yy) of specimen 0, FP64 block-Jacobi PCG to 1e-8 by the C oracle "
                             "(restating coarse3d/lin3d.py:464-532), %.1f s" % secs}
            # the reference's thread protocol (timing/t3d/bench3d.py:167-171): all cores, 6 threads, 1 thread; and its
            # strongest CPU solver, the aggregation-AMG PCG (timing/t3d/problems.py:112-132), on one load case
            cpu_extra = {"bj_pcg_threads": {}}
            for t in (6, 1):
                s_t, n_t, thr_t, _ = cpu_solve_sample(lat, Kn_h, Tv_h, free_h, ups_h, [(0, 0)], threads=t)
                cpu_extra["bj_pcg_threads"][str(thr_t)] = n_t / s_t
            cpu_extra["bj_pcg_threads"][str(thr)] = n / secs
            s_a, it_a = cpu_amg_sample(lat, Kn_h, Tv_h, free_h, ups_h, 0, 0)
            cpu_extra["amg_pcg"] = {"solves_per_s": 1.0 / s_a, "iterations": it_a, "cores": thr,
                                    "path": "NumPy restatement of timing/t3d/amg3d.py (setup + PCG, load k_xx of "
                                            "specimen 0)"}
        else:
            # a full CPU solve of this size takes tens of minutes: time 30 PCG iterations of load 0 and scale by the
            # iteration count the same FP64 PCG needs on the GPU
            M0 = core.block_jacobi(dl, Kn[0:1, 0], Tv[0:1, 0], torch.float64)
            _, i0 = core.cg(dl, Kn[0:1, 0], Tv[0:1, 0], b[0:1, 0], Minv=M0, free=free[0:1], tol=TOL, maxit=20000,
                            check=1, poll=50)
            need = int(i0.iters[0])
            secs, n, thr, done = cpu_solve_sample(lat, Kn_h, Tv_h, free_h, ups_h, [(0, 0)], maxit=30)
            cpu = {"value": 1.0 / (secs / max(done, 1) * need), "unit": UNIT, "cores": thr, "kind": "port",
                   "sample": "30 FP64 block-Jacobi PCG iterations of load k_xx by the C oracle (restating "
                             "coarse3d/lin3d.py:464-532), %.1f s, scaled to the %d iterations the same PCG needs "
                             "to 1e-8" % (secs, need)}

    # kernels of this library launched in the timed region: per inner PCG iteration 3 (pair-packed K.u with the p.Ap
    # epilogue, update, p-update); per step 2 (b = -K u_p) + 2 (FP32 packing) + 1 (block Jacobi); per refinement
    # step 2 (FP64 K.u) + 1 (residual) + 1 (scale) + 3 (preconditioner repack, PCG init, unpack) + 1 (correction);
    # plus the final residual check (3).  Iterations per inner solve are counted as the slowest system's.
    # With AMG: per step 2 (FP64 packing) + 1 (b = -K u_p on the packed TMA operator) + 2 (FP32 packing) + 1 (block
    # Jacobi) + the AMG setup, and
    # per inner iteration / inner solve / refinement step the counts of AmgBatch.launches (operator, update, cycle
    # with every coarse-level kernel, p-update).
    total_inner = int(sum(int(i.iters.max()) for i in infos))
    outer = sum(int(i.outer) for i in infos)
    if amgb is None:
        gpu_launches = total_inner * 3 + a.steps * (5 + 3) + outer * 8
    else:
        gpu_launches = a.steps * 6 + sum(amgb.launches(int(i.iters.max()), int(i.outer), int(i.outer)) for i in infos)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded %s microstructures, shapes of the %d^3 config)"
            % ("spheres" if a.workload == "spheres48" else "prolate-ellipsoid", WORKLOADS[a.workload]["n"]),
            "config": workload_config(a.workload, B, world),
            "method": {"precision": "fp32 inner PCG + fp64 refinement", "preconditioner": PRECONDS[a.precond],
                       "inner_tol": a.inner_tol,
                       "operator_tiles": {"zchunk": tiles[0], "variant": ["staged", "lean"][tiles[1]]},
                       "amg_levels": [[list(g) for g in amgb.grids(k)[0]] for k in range(len(amgb.boxes))]
                       if amgb is not None else None},
            "roofline": roofline, "cpu_baseline": cpu, "cpu_comparators": cpu_extra, "e2e": e2e,
            "clocks": clocks, "gpu_launches": gpu_launches, "all_converged": bool(ok),
            "inner_iters_mean": float(iters.mean()), "outer_steps": [i.outer for i in infos][:1],
            "step_ms": [round(v, 3) for v in step_ms], "graphs": graphs,
            "fp64_gpu_cg": fp64_cg,
            "speedup_vs_fp64_gpu_cg": value / world / fp64_cg["solves_per_s"] if fp64_cg else None,
            "reference_gpu_cg": torch_cg,
            "speedup_vs_reference_gpu_cg": value / world / torch_cg["solves_per_s"] if torch_cg else None,
            "accuracy": accuracy}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
