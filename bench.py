"""Benchmark of the LPM linear solve on B200: mixed-precision batched PCG solves per second.

Workloads (one "step" = one batched solve of every system from scratch, inputs resident in HBM):
  spheres48 (default): 48^3 simple-cubic fine LPM, seeded random non-overlapping spheres (r = 4 voxels, volume
    fraction 0.25, contrast 10, E = 1, nu = 0.2; per-bond Kn/Tv = two-end mean of the particle values), 6 KUBC
    macro-strain load cases (magnitude 1e-3) as 6 right-hand sides per specimen, a batch of B specimens per GPU.
  ellipsoids192: 192^3, seeded randomly oriented prolate ellipsoids 3:1:1 (volume of a sphere of radius 4, volume
    fraction 0.30, contrast 15, nu = 0.2), 9 load cases (6 KUBC strains + uniaxial tension along x, y, z) as 9
    right-hand sides of one specimen.
Each step forms b = -K u_p in FP64, packs FP32 coefficients, builds the 3x3 block-Jacobi preconditioner and runs FP32
PCG inside FP64 iterative refinement until every system's FP64 true residual is <= 1e-8 |b|.  Synthetic data (no
dataset is involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B] [--workload spheres48|ellipsoids192]
                    [--impl ours|reference]

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


def workload_config(w, batch, n_gpus):
    W = WORKLOADS[w]
    n, L = W["n"], len(W["loads"])
    return {"workload": W["label"], "lattice": [n] * 3, "specimens_per_gpu": batch, "rhs_per_specimen": L,
            "systems_per_gpu": L * batch, "tol": TOL, "precision": "fp32 inner PCG + fp64 refinement",
            "preconditioner": "3x3 block Jacobi", "l2": "inputs larger than L2 (%.0f MB of FP64 coefficients per GPU)"
            % (batch * n ** 3 * 36 * 8 / 1e6), "parallelism": "dp%d (independent specimens per GPU)" % n_gpus}


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


# ------------------------------------------------------------------------------------------------ CPU side
def kmv_traffic(nsys):
    """DRAM bytes per K.u launch for `nsys` systems of the 48^3 workload (6 per specimen), scaled from the ncu capture
    of a 4-specimen launch (24 systems) summarised in profiles/: read + write bytes grow with the systems and sets."""
    path = os.path.join(ROOT, "profiles", "k_sc_pair_48cube_batch4.md")
    if not os.path.exists(path):
        return None
    got = {}
    for line in open(path):
        for key in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            if line.startswith("| `%s`" % key):
                val, unit = line.split("|")[2].split()
                got[key] = float(val) * {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9}[unit]
    if len(got) != 2:
        return None
    return (got["dram__bytes_read.sum"] + got["dram__bytes_write.sum"]) / 24 * nsys


def cpu_solve_sample(lat, Kn, Tv, free, ups, nsolve, maxit=20000):
    """FP64 block-Jacobi PCG of the CPU oracle (the reference's lin3d._pcg restated in C, all host threads) on the
    first `nsolve` load cases of specimen 0, at most `maxit` iterations each.  Returns (seconds, solves, threads,
    iterations of the last solve)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    it = 0
    for l in range(nsolve):
        fixed = ~free[l]
        _, info = O.solve_pcg(lat, Kn[0], Tv[0], fixed, ups[l], tol=TOL, maxit=maxit)
        it = info["iters"]
    return time.perf_counter() - t0, nsolve, O.get_threads(), it


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    lat, Kn, Tv, free, ups = load_workload(a.workload, [0])
    nsolve = 1
    for _ in range(a.warmup):
        cpu_solve_sample(lat, Kn, Tv, free, ups, nsolve)
    secs = []
    for _ in range(a.steps):
        s, n, thr, _ = cpu_solve_sample(lat, Kn, Tv, free, ups, nsolve)
        secs.append(s)
    tot = sum(secs)
    value = a.steps * nsolve / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * tot / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a.workload, a.batch, a.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port",
                             "sample": "%d load case(s) per step of specimen 0, FP64 block-Jacobi PCG to 1e-8 "
                                       "(oracle restating coarse3d/lin3d.py:464-532)" % nsolve},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------------------- GPU side
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=None, help="specimens per GPU (default 16 for spheres48, 1 else)")
    ap.add_argument("--workload", default="spheres48", choices=sorted(WORKLOADS))
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 CG comparator")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--inner-tol", type=float, default=1e-5)
    a = ap.parse_args()
    if a.batch is None:
        a.batch = 16 if a.workload == "spheres48" else 1
    if a.impl == "reference":
        return run_reference(a)

    import torch
    import torch.distributed as dist
    from lpm_b200 import core

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    seeds = [rank * a.batch + j for j in range(a.batch)]
    lat, Kn_h, Tv_h, free_h, ups_h = load_workload(a.workload, seeds)
    B = a.batch
    Lc = len(WORKLOADS[a.workload]["loads"])
    dl = core.DeviceLattice(lat, dev)
    Kn = torch.as_tensor(Kn_h, device=dev)[:, None]          # (B, 1, N, 18)
    Tv = torch.as_tensor(Tv_h, device=dev)[:, None]
    free = torch.as_tensor(free_h, device=dev, dtype=torch.float64)      # (6, N)
    ups = torch.as_tensor(ups_h, device=dev)[None].expand(B, -1, -1, -1).contiguous()   # (B, 6, N, 3)
    nsys = B * Lc

    def step(Kn, Tv, free, ups, prof=None):
        b = -core.kmv(dl, ups, Kn, Tv) * free[None, :, :, None]
        x, info = core.ir(dl, Kn, Tv, b, free=free, tol=TOL, inner_tol=a.inner_tol, prof=prof)
        return ups + x, info

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(max(a.warmup, 1)):
        u, info = step(Kn, Tv, free, ups)
    barrier()

    prof = core.new_prof()
    sampler = ClockSampler(local)
    sampler.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record()
    infos = []
    for _ in range(a.steps):
        u, info = step(Kn, Tv, free, ups, prof)
        infos.append(info)
    ev1.record()
    barrier()
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * nsys * a.steps / (ms / 1e3)
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
    traffic = kmv_traffic(nsys) if a.workload == "spheres48" else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                "kernel": "k_sc_pair: pair-packed FP32 SC K.u with the p.Ap epilogue (all %d systems, %d coefficient "
                          "sets) in the inner PCG" % (nsys, B),
                "traffic_source": "ncu dram bytes of a 4-specimen launch (profiles/k_sc_pair_48cube_batch4.md) scaled "
                                  "by systems",
                "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": full_ms, "avg_launch_ms_all": all_ms,
                "launches_timed": int(prof[1]), "peak_source": peak_src}

    # ---- end to end through the public API with host buffers (pinned), copies inside the timed region
    Kn_pin = torch.as_tensor(Kn_h).pin_memory()
    Tv_pin = torch.as_tensor(Tv_h).pin_memory()
    fr_pin = torch.as_tensor(free_h, dtype=torch.float64).pin_memory()
    up_pin = torch.as_tensor(ups_h).pin_memory()
    u_host = torch.empty((B, Lc, Nn, 3), dtype=torch.float64).pin_memory()
    h2d = Kn_pin.numel() * 8 + Tv_pin.numel() * 8 + fr_pin.numel() * 8 + up_pin.numel() * 8
    d2h = u_host.numel() * 8

    def e2e_step():
        k = Kn_pin.to(dev, non_blocking=True)[:, None]
        t = Tv_pin.to(dev, non_blocking=True)[:, None]
        f = fr_pin.to(dev, non_blocking=True)
        up = up_pin.to(dev, non_blocking=True)[None].expand(B, -1, -1, -1)
        uu, _ = step(k, t, f, up)
        u_host.copy_(uu, non_blocking=True)

    e2e_step()
    barrier()
    ev0.record()
    for _ in range(a.steps):
        e2e_step()
    ev1.record()
    barrier()
    ms_e2e = ev0.elapsed_time(ev1)
    if world > 1:
        t = torch.tensor([ms_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    e2e = {"value": world * nsys * a.steps / (ms_e2e / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h)}

    # ---- comparator: plain FP64 GPU CG on the same batch with this library's fastest FP64 path (packed
    # coefficients, TMA-fed fused operator, same engine), packing included; accuracy vs FP64 PCG to 1e-12
    from lpm_b200 import _lib
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
                   "path": "FP64 plain CG, packed coefficients, TMA-fed fused operator (k_sc_tma<double>)"}
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

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        if a.workload == "spheres48":
            secs, n, thr, _ = cpu_solve_sample(lat, Kn_h, Tv_h, free_h, ups_h, 2)
            cpu = {"value": n / secs, "unit": UNIT, "cores": thr, "kind": "port",
                   "sample": "2 load cases (k_xx, k_yy) of specimen 0, FP64 block-Jacobi PCG to 1e-8 by the C oracle "
                             "(restating coarse3d/lin3d.py:464-532), %.1f s" % secs}
        else:
            # a full CPU solve of this size takes tens of minutes: time 30 PCG iterations of load 0 and scale by the
            # iteration count the same FP64 PCG needs on the GPU
            M0 = core.block_jacobi(dl, Kn[0:1, 0], Tv[0:1, 0], torch.float64)
            _, i0 = core.cg(dl, Kn[0:1, 0], Tv[0:1, 0], b[0:1, 0], Minv=M0, free=free[0:1], tol=TOL, maxit=20000,
                            check=1, poll=50)
            need = int(i0.iters[0])
            secs, n, thr, done = cpu_solve_sample(lat, Kn_h, Tv_h, free_h, ups_h, 1, maxit=30)
            cpu = {"value": 1.0 / (secs / max(done, 1) * need), "unit": UNIT, "cores": thr, "kind": "port",
                   "sample": "30 FP64 block-Jacobi PCG iterations of load k_xx by the C oracle (restating "
                             "coarse3d/lin3d.py:464-532), %.1f s, scaled to the %d iterations the same PCG needs "
                             "to 1e-8" % (secs, need)}

    # kernels of this library launched in the timed region: per inner PCG iteration 3 (pair-packed K.u with the p.Ap
    # epilogue, update, p-update); per step 2 (b = -K u_p) + 2 (FP32 packing) + 1 (block Jacobi); per refinement
    # step 2 (FP64 K.u) + 1 (residual) + 1 (scale) + 3 (preconditioner repack, PCG init, unpack) + 1 (correction);
    # plus the final residual check (3).  Iterations per inner solve are counted as the slowest system's.
    total_inner = int(sum(int(i.iters.max()) for i in infos))
    outer = sum(int(i.outer) for i in infos)
    gpu_launches = total_inner * 3 + a.steps * (5 + 3) + outer * 8
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic (seeded %s microstructures, shapes of the %d^3 config)"
            % ("spheres" if a.workload == "spheres48" else "prolate-ellipsoid", WORKLOADS[a.workload]["n"]),
            "config": workload_config(a.workload, B, world), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "clocks": clocks, "gpu_launches": gpu_launches, "all_converged": bool(ok),
            "inner_iters_mean": float(iters.mean()), "outer_steps": [i.outer for i in infos][:1],
            "fp64_gpu_cg": fp64_cg,
            "speedup_vs_fp64_gpu_cg": value / world / fp64_cg["solves_per_s"] if fp64_cg else None,
            "accuracy": accuracy}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
