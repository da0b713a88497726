"""Parity at the sizes of the benchmark configurations, against the CPU oracle (FP64) and the reference's own outputs.

* 48^3 spheres x 6 KUBC load cases (the headline batch, two specimens of it): the mixed-precision solve to relative
  residual 1e-8, with the AMG preconditioner and with 3x3 block Jacobi, against the oracle's FP64 block-Jacobi PCG
  (coarse3d/lin3d.py:464-532 restated) to 1e-12; bar 1e-6 relative displacement (L2) per load case, stress too.
* 96^3 prolate ellipsoids 3:1:1 x 9 load cases (the 192^3 configuration's microstructure and loads at an eighth of the
  sites, so the oracle finishes in seconds): AMG and block Jacobi, checked on two load cases (one KUBC ring, one
  plate tension).
* The differentiable 2D coarse solve of the third configuration at nc = 32 and 48: loss and gradient w.r.t. the log
  bond stiffness against the reference's dense torch_lpm gradient (tests/golden/golden_cfg3.npz); bar 1e-6.
"""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import relmax
from lpm_b200 import amg as GA
from lpm_b200 import core
from lpm_b200 import geom as G
from lpm_b200 import micro as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
LOADS6 = ["k_xx", "k_yy", "k_zz", "k_yz", "k_xz", "k_xy"]
LOADS9 = LOADS6 + ["lr_tx", "fb_ty", "tb_tz"]
TOL = 1e-8


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def sc_specimen(n, seed, kind):
    lat = G.LatticeGeom(n, n, n, 1.0)
    rng = np.random.default_rng(seed)
    if kind == "spheres":
        ph, _ = M.spheres(n, n, n, 0.25, 4.0, rng, rjit=0.0)
        contrast = 10.0
    else:
        ph, _ = M.prolate_ellipsoids(n, n, n, 0.30, 4.0, rng, aspect=3.0, max_tries=60000)
        contrast = 15.0
    C = G.iso_C(np.where(ph == 1, contrast, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    return lat, Kn, Tv


def load_bcs(lat, n, loads):
    free, ups = [], []
    for ld in loads:
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        free.append(~fixed)
        ups.append(np.where(fixed[:, None], up, 0.0))
    return np.array(free), np.array(ups)


def mixed_solve(lat, Kn, Tv, free, ups, precond, inner_tol):
    """The benchmark's step: b = -K u_p masked, then FP32 PCG (AMG or block Jacobi) inside FP64 refinement to 1e-8.
    Kn, Tv: (B, N, 18); free, ups: (L, N), (L, N, 3).  Returns u (B, L, N, 3) and the solve info."""
    B, L = Kn.shape[0], free.shape[0]
    dl = core.DeviceLattice(lat, DEV)
    Kd = torch.as_tensor(Kn, device=DEV)[:, None]
    Td = torch.as_tensor(Tv, device=DEV)[:, None]
    fr = torch.as_tensor(free, device=DEV, dtype=torch.float64)
    up = torch.as_tensor(ups, device=DEV)[None].expand(B, -1, -1, -1).contiguous()
    b = -core.kmv(dl, up, Kd, Td) * fr[None, :, :, None]
    if precond == "bj":
        x, info = core.ir(dl, Kd, Td, b, free=fr, tol=TOL, inner_tol=inner_tol)
        return (up + x).cpu().numpy(), info, dl
    ab = GA.AmgBatch(dl, B * L, L, free, **GA.AMG_CFG)
    ab.setup(core.pack(Kd[:, 0], torch.float32), core.pack(Td[:, 0], torch.float32),
             core.block_jacobi(dl, Kd[:, 0], Td[:, 0], torch.float32))
    x, info = ab.ir(Kd[:, 0], Td[:, 0], b.reshape(B * L, lat.N, 3), tol=TOL, inner_tol=inner_tol)
    return (up + x.reshape(up.shape)).cpu().numpy(), info, dl


def stress_of(dl, u, Kn, Tv):
    ud = torch.as_tensor(u, device=DEV)[None, None]
    return core.stress(dl, ud, torch.as_tensor(Kn, device=DEV)[None, None],
                       torch.as_tensor(Tv, device=DEV)[None, None])[0, 0].cpu().numpy()


@pytest.fixture(scope="module")
def spheres48():
    n = 48
    specs = [sc_specimen(n, s, "spheres") for s in (0, 1)]
    lat = specs[0][0]
    free, ups = load_bcs(lat, n, LOADS6)
    Kn = np.stack([s[1] for s in specs])
    Tv = np.stack([s[2] for s in specs])
    # the oracle's FP64 block-Jacobi PCG to 1e-12: every load of specimen 0, two of specimen 1
    ref = {}
    for j, l in [(0, l) for l in range(6)] + [(1, 0), (1, 5)]:
        ref[j, l] = O.solve_pcg(lat, Kn[j], Tv[j], ~free[l], ups[l], tol=1e-12)[0]
    return dict(n=n, lat=lat, Kn=Kn, Tv=Tv, free=free, ups=ups, ref=ref)


@pytest.mark.parametrize("precond,inner_tol", [("amg", 1e-4), ("bj", 1e-3)])
def test_spheres48_batch_vs_oracle(spheres48, precond, inner_tol):
    c = spheres48
    u, info, dl = mixed_solve(c["lat"], c["Kn"], c["Tv"], c["free"], c["ups"], precond, inner_tol)
    assert (info.status == 0).all() and (info.relres <= TOL).all()
    for (j, l), uref in c["ref"].items():
        assert rel_l2(u[j, l], uref) < 1e-6, (precond, j, LOADS6[l], rel_l2(u[j, l], uref))
    for l in (0, 3):   # stress of specimen 0 on a normal and a shear load
        sm = stress_of(dl, u[0, l], c["Kn"][0], c["Tv"][0])
        sr = stress_of(dl, c["ref"][0, l], c["Kn"][0], c["Tv"][0])
        assert rel_l2(sm, sr) < 1e-6, (precond, LOADS6[l])


@pytest.fixture(scope="module")
def prolate96():
    n = 96
    lat, Kn, Tv = sc_specimen(n, 0, "prolate")
    free, ups = load_bcs(lat, n, LOADS9)
    ref = {l: O.solve_pcg(lat, Kn, Tv, ~free[l], ups[l], tol=1e-12)[0] for l in (5, 6)}   # k_xy, lr_tx
    return dict(n=n, lat=lat, Kn=Kn[None], Tv=Tv[None], free=free, ups=ups, ref=ref)


@pytest.mark.parametrize("precond,inner_tol", [("amg", 1e-4), ("bj", 1e-3)])
def test_prolate96_nine_loads_vs_oracle(prolate96, precond, inner_tol):
    c = prolate96
    u, info, _ = mixed_solve(c["lat"], c["Kn"], c["Tv"], c["free"], c["ups"], precond, inner_tol)
    assert (info.status == 0).all() and (info.relres <= TOL).all()
    for l, uref in c["ref"].items():
        assert rel_l2(u[0, l], uref) < 1e-6, (precond, LOADS9[l], rel_l2(u[0, l], uref))


@pytest.mark.parametrize("nc", [32, 48])
def test_coarse2d_gradient_vs_reference_dense(nc):
    """The adjoint gradient of the matrix-free 2D coarse solve equals the reference's dense-Cholesky autograd gradient
    (torch_lpm.CoarseT.run) on the third configuration's inputs at nc = 32 and 48."""
    from lpm_b200 import torch_lpm as T2
    with np.load(__import__("os").path.join(__import__("conftest").GOLDEN, "golden_cfg3.npz")) as d:
        g = {k: d[k] for k in d.files if k.startswith("n%d_" % nc)}
    pre = "n%d_" % nc
    loads = ["lr_tx", "tb_ty", "tb_sx"]
    m = T2.CoarseT(nc, nc, 2, 1.0, device=DEV, loads=loads)
    m.tol = 1e-13
    lat = m.lat
    q = torch.as_tensor(np.where(lat.valid, lat.nbr, 0), device=DEV)
    opp = torch.as_tensor(np.repeat(lat.opp[None, :], lat.N, 0), device=DEV)
    valid = torch.as_tensor(lat.valid, device=DEV, dtype=torch.float64)
    Kb = torch.as_tensor(g[pre + "Kb"], device=DEV)[None]
    Tb = torch.as_tensor(g[pre + "T0"], device=DEV)[None]
    tgt = {ld: torch.as_tensor(g[pre + "tgt_" + ld], device=DEV)[None] for ld in loads}
    th = torch.zeros((1, lat.N, 8), dtype=torch.float64, device=DEV, requires_grad=True)
    out = m.run(Kb * torch.exp(0.5 * (th + th[:, q, opp])) * valid, Tb)
    L = sum(((out[ld]["u"] - tgt[ld]) ** 2).mean() for ld in loads)
    L.backward()
    for ld in loads:
        assert relmax(out[ld]["u"].detach().cpu().numpy()[0], g[pre + "u_" + ld]) < 1e-8, ld
    assert abs(float(L) - float(g[pre + "loss"])) < 1e-6 * abs(float(g[pre + "loss"]))
    gref = g[pre + "gth"]
    assert relmax(th.grad.cpu().numpy()[0], gref) < 1e-6
    assert rel_l2(th.grad.cpu().numpy()[0], gref) < 1e-7
