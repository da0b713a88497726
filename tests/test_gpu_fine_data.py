"""GPU: the data/fine_*.npz generator (coarse3d/gen_fine.py format) on the AMG path agrees with the reference's FP64
block-Jacobi PCG path, and LatticeOperator.solve_amg solves batched load sets."""
import numpy as np
import pytest
import torch

from conftest import relmax
from lpm_b200 import fine_data as FD
from lpm_b200 import geom as G
from lpm_b200 import micro as M
from lpm_b200 import torch_lpm3d as T3

pytestmark = pytest.mark.gpu


def test_fine_data_amg_matches_fp64():
    n, S = 12, 2
    rng = np.random.default_rng(2)
    d = dict(n=n, phase=np.array([M.spheres(n, n, n, 0.25, 2.0, np.random.default_rng(10 + i), rjit=0.0)[0]
                                  for i in range(S)]),
             contrast=rng.uniform(5, 15, S), nu_i=rng.uniform(0.15, 0.3, S))
    a = FD.generate(d, precision="amg", log=None)
    b = FD.generate(d, precision="fp64", log=None)
    for s in (2, 3):
        nc = n // s
        assert a["u_%d" % s].shape == (S, 9, nc ** 3, 3) and a["u_%d" % s].dtype == np.float32
        assert a["sig_%d" % s].shape == (S, 9, nc ** 3, 6) and a["w_%d" % s].shape == (S, 9, nc ** 3)
        assert a["F_%d" % s].shape == (S, 9) and a["iface_%d" % s].shape == (S, nc ** 3)
        for k in ("u", "sig", "w", "F"):
            assert relmax(a["%s_%d" % (k, s)], b["%s_%d" % (k, s)]) < 1e-5, (k, s)
        assert np.array_equal(a["iface_%d" % s], b["iface_%d" % s])
        nb = -(-S // 8)   # one entry per batch of samples (8 per batch at n <= 24), as gen_fine.py
        assert len(a["tgpu_%d" % s]) == nb and len(a["iters_%d" % s]) == nb
    assert int(a["n"]) == n


def test_solve_amg_operator():
    """SCT.solve_amg on (B, L) = (2, 9) load sets (four BC boxes) vs the FP64 block-Jacobi solve."""
    n = 16
    lat = G.LatticeGeom(n, n, n, 1.0)
    ref = T3.FineRefT(n, 2, precision="fp64")
    ks, ts = [], []
    for sd in (1, 2):
        ph, _ = M.spheres(n, n, n, 0.25, 2.5, np.random.default_rng(sd), rjit=0.0)
        (K, Tt), _ = FD.fine_params(lat, ph, 10.0, 0.2)
        ks.append(K)
        ts.append(Tt)
    Kn = torch.as_tensor(np.array(ks), device="cuda")[:, None]
    Tv = torch.as_tensor(np.array(ts), device="cuda")[:, None]
    up = ref.bc.up[None].expand(2, -1, -1, -1)
    free = ref.bc.free[None].expand(2, -1, -1)
    u, info = ref.op.solve_amg(Kn, Tv, up, free, tol=1e-10)
    assert (info.status == 0).all() and (info.relres <= 1e-10).all()
    u64, _, rel = ref.op.solve(Kn, Tv, up, free, tol=1e-12)
    assert relmax(u.cpu().numpy(), u64.cpu().numpy()) < 1e-8
