"""Fine-LPM reference data in the format of coarse3d/gen_fine.py (``data/fine_SPLIT.npz``).

For every sample of a split (``data/micro_SPLIT.npz``: ``n``, ``phase`` (S, n^3), ``contrast`` (S,), ``nu_i`` (S,)) and
block sizes s = 2 and 3: block means of displacement ``u_s`` (S, 9, nc^3, 3) and stress ``sig_s`` (S, 9, nc^3, 6), block
energy density ``w_s`` (S, 9, nc^3) (FP32), grip reactions ``F_s`` (S, 9), interface cells ``iface_s`` (S, nc^3), the
solver iterations of every batch ``iters_s`` and the GPU seconds per sample ``tgpu_s``; plus ``n``.  The solve is the
library's: FP32 PCG in FP64 refinement to the reference's tolerance 1e-10 on the FP64 true residual, preconditioned by
the aggregation AMG (``precision="amg"``, default), block Jacobi (``"mixed"``), or the reference's FP64 block-Jacobi PCG
(``"fp64"``).

    python -m lpm_b200.fine_data SPLIT [--bs B] [--precision amg|mixed|fp64] [--root DIR]
"""
import argparse
import os
import time

import numpy as np
import torch

from . import geom as G
from .torch_lpm3d import FineRefT


def fine_params(lat, ph, contrast, nu_i):
    """Per-bond (Kn, Tv) of a two-phase voxel image and the voxel stiffness (coarse3d/gen_fine.py:15-19)."""
    E = np.where(ph == 1, contrast, 1.0)
    nu = np.where(ph == 1, nu_i, 0.2)
    Cv = G.iso_C(E, nu)
    return G.bond_params_two_end_mean(lat, G.sc_params_from_C(Cv, 0.5)), Cv


def generate(d, bs=None, device="cuda", precision="amg", tol=1e-10, blocks=(2, 3), log=print):
    """The arrays of data/fine_SPLIT.npz for the samples of `d` (keys n, phase, contrast, nu_i)."""
    n = int(d["n"])
    S = len(d["phase"])
    if bs is None:
        bs = 8 if n <= 24 else (2 if n <= 48 else 1)   # batch sizes of coarse3d/gen_fine.py:29
    lat = G.LatticeGeom(n, n, n, 1.0)
    out = {}
    for s in blocks:
        # the load chunks of coarse3d/gen_fine.py:35 (one batch of all nine loads up to n = 48)
        chunks = [G.LOADS] if n <= 48 else [G.RING, ["tb_tz", "tb_sx"], ["lr_tx"]]
        refs = [FineRefT(n, s, device=device, loads=ld, precision=precision) for ld in chunks]
        nc = n // s
        U = np.zeros((S, 9, nc ** 3, 3), np.float32)
        SG = np.zeros((S, 9, nc ** 3, 6), np.float32)
        W = np.zeros((S, 9, nc ** 3), np.float32)
        F = np.zeros((S, 9))
        its, tt = [], []
        for i0 in range(0, S, bs):
            idx = range(i0, min(S, i0 + bs))
            KT = [fine_params(lat, d["phase"][i], d["contrast"][i], d["nu_i"][i])[0] for i in idx]
            Kn = torch.as_tensor(np.array([k for k, _ in KT]), device=device)
            Tv = torch.as_tensor(np.array([t for _, t in KT]), device=device)
            torch.cuda.synchronize(device)
            t0 = time.time()
            l0 = 0
            for fr in refs:
                r = fr.run(Kn, Tv, tol=tol)
                L = len(fr.loads)
                U[i0:i0 + len(idx), l0:l0 + L] = r["u"].cpu().numpy()
                SG[i0:i0 + len(idx), l0:l0 + L] = r["sig"].cpu().numpy()
                W[i0:i0 + len(idx), l0:l0 + L] = r["w"].cpu().numpy()
                F[i0:i0 + len(idx), l0:l0 + L] = r["F"].cpu().numpy()
                its.append(r["iters"])
                l0 += L
            torch.cuda.synchronize(device)
            tt.append((time.time() - t0) / len(idx))
        out.update({"u_%d" % s: U, "sig_%d" % s: SG, "w_%d" % s: W, "F_%d" % s: F,
                    "iface_%d" % s: np.array([G.interface_cells(d["phase"][i], n, s) for i in range(S)]),
                    "iters_%d" % s: np.array(its), "tgpu_%d" % s: np.array(tt)})
        if log:
            log("s=%d: %d samples, PCG its %d-%d, GPU %.3f s/sample" % (s, S, min(its), max(its), np.mean(tt)))
    out["n"] = n
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("split")
    ap.add_argument("--bs", type=int, default=None)
    ap.add_argument("--precision", default="amg", choices=["amg", "mixed", "fp64"])
    ap.add_argument("--root", default=".", help="folder holding data/micro_SPLIT.npz")
    a = ap.parse_args(argv)
    d = dict(np.load(os.path.join(a.root, "data", "micro_%s.npz" % a.split), allow_pickle=True))
    t0 = time.time()
    out = generate(d, bs=a.bs, precision=a.precision, log=lambda m: print("%s %s" % (a.split, m), flush=True))
    os.makedirs(os.path.join(a.root, "data"), exist_ok=True)
    np.savez_compressed(os.path.join(a.root, "data", "fine_%s.npz" % a.split), **out)
    print("%s done in %.0f s" % (a.split, time.time() - t0), flush=True)


if __name__ == "__main__":
    main()
