"""GPU parity of the AMG preconditioner (csrc/amg.cu, through the C ABI) against the AMG oracle (oracle/amg.py, itself
pinned to the reference's timing/t3d/amg3d.py in test_oracle_amg.py): levels, rho, one cycle, PCG iterations, the
mixed-precision solve, batching, and the reference-named mirror (AMGGeom / AMG3D).

Tolerances: the CUDA hierarchy is FP32 (level 1 from the bonds in FP32 with FP64 moments, or from FP32 K.u probes for
aggregates wider than 5 sites; FP32 smoothing), so levels and cycles agree with
the FP64 oracle to FP32 round-off amplified by the operator's conditioning (<= 2e-4 relative); solved displacements
agree to the solve tolerance.
"""
import numpy as np
import pytest
import torch

import amg as OA
import oracle as O
from conftest import relmax
from lpm_b200 import amg as GA
from lpm_b200 import core
from lpm_b200 import geom as G
from lpm_b200 import micro as M

pytestmark = pytest.mark.gpu

LOADS = ("k_xx", "tb_tz", "lr_tx")   # one load of each BC box: ring, z plates, x plates


def specimen(n, seed, r):
    lat = G.LatticeGeom(n, n, n, 1.0)
    ph, _ = M.spheres(n, n, n, 0.25, r, np.random.default_rng(seed), rjit=0.0)
    C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    return lat, Kn, Tv


def bcs(lat, n, loads=LOADS):
    fr, ups = [], []
    for ld in loads:
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        fr.append(~fixed)
        ups.append(np.where(fixed[:, None], up, 0.0))
    return np.array(fr), np.array(ups)


@pytest.fixture(scope="module")
def case24():
    """24^3 spheres, the three BC boxes as three systems of one set; GPU hierarchy and oracle hierarchies (same
    power-iteration start vectors, rho0 of the first box reused as timing/t3d/problems.py does)."""
    n = 24
    lat, Kn, Tv = specimen(n, 3, 3.0)
    free, ups = bcs(lat, n)
    dev = torch.device("cuda")
    dl = core.DeviceLattice(lat, dev)
    Kd = torch.as_tensor(Kn, device=dev)[None]
    Td = torch.as_tensor(Tv, device=dev)[None]
    ab = GA.AmgBatch(dl, 3, 3, free, **GA.AMG_CFG)
    ab.setup(core.pack(Kd, torch.float32), core.pack(Td, torch.float32), core.block_jacobi(dl, Kd, Td, torch.float32))
    orc, rho0 = [], None
    for k in range(3):
        geo = OA.Geometry(lat, free[k])
        h = OA.Hierarchy(geo, Kn, Tv, rho0=rho0, start="hash")
        rho0 = h.rho0
        orc.append(h)
    return dict(n=n, lat=lat, Kn=Kn, Tv=Tv, free=free, ups=ups, dl=dl, Kd=Kd, Td=Td, ab=ab, orc=orc)


def test_amg_levels_match_oracle(case24):
    ab, orc = case24["ab"], case24["orc"]
    assert np.allclose(ab.rho0(), orc[0].rho0, rtol=1e-4)
    for k in range(3):
        grids, _ = ab.grids(k)
        assert grids == [tuple(g) for g in orc[k].geo.grids]
        for lvl in range(1, len(grids) + 1):
            A, rho = ab.level(k, 0, lvl)
            assert relmax(A, orc[k].A[lvl - 1]) < 2e-5, (k, lvl)
            if lvl < len(grids):
                assert abs(rho - orc[k].rho[lvl - 1]) < 1e-4 * orc[k].rho[lvl - 1]


@pytest.mark.parametrize("agg", [4, 5])
def test_amg_level1_probing_path_matches_oracle(agg):
    """Aggregates of 4 or 5 sites (chunks up to 7 or 9 wide) take the probing construction of the level-1 operator
    instead of the direct bond product (which covers widths up to 5, all of agg = 3): both must give P^T K_ff P."""
    n = 20
    lat, Kn, Tv = specimen(n, 9, 2.5)
    free, _ = bcs(lat, n, ("k_xx", "lr_tx"))
    dl = core.DeviceLattice(lat, "cuda")
    Kd = torch.as_tensor(Kn, device="cuda")[None]
    Td = torch.as_tensor(Tv, device="cuda")[None]
    ab = GA.AmgBatch(dl, 2, 2, free, agg=agg, coarse_max=100, nu=1, gamma=2, power_its=5)
    ab.setup(core.pack(Kd, torch.float32), core.pack(Td, torch.float32), core.block_jacobi(dl, Kd, Td, torch.float32))
    for k in range(2):
        geo = OA.Geometry(lat, free[k], agg=agg, coarse_max=100)
        A, _ = ab.level(k, 0, 1)
        assert relmax(A, OA.galerkin0(geo, Kn, Tv)) < 2e-5, (agg, k)
    ab.close()


def test_amg_cycle_matches_oracle(case24):
    ab, orc, free = case24["ab"], case24["orc"], case24["free"]
    rng = np.random.default_rng(8)
    r = rng.standard_normal((3, case24["lat"].N, 3)) * free[:, :, None]
    z = ab.apply(torch.as_tensor(r, device="cuda", dtype=torch.float32)).double().cpu().numpy()
    for k in range(3):
        assert relmax(z[k], orc[k].vcycle(r[k].copy())) < 2e-4, k


def test_amg_pcg_iterations_match_oracle(case24):
    """FP32 AMG-PCG to 1e-5 needs the oracle's FP64 iteration count, within 1."""
    ab, orc, lat = case24["ab"], case24["orc"], case24["lat"]
    b = np.stack([-O.sc_apply(lat, case24["ups"][k], case24["Kn"], case24["Tv"]) * case24["free"][k][:, None]
                  for k in range(3)])
    x, info = ab.pcg(torch.as_tensor(b, device="cuda", dtype=torch.float32), 1e-5, maxit=500)
    assert (info.status == 0).all()
    for k in range(3):
        _, it, _ = orc[k].pcg(b[k], 1e-5)
        assert abs(int(info.iters[k]) - it) <= 1, (k, info.iters[k], it)


def test_ir_amg_solution(case24):
    """Mixed precision with the AMG inner solver: FP64 residual <= 1e-8 and the displacements of the oracle's FP64
    block-Jacobi PCG to 1e-12."""
    ab, lat, Kn, Tv = case24["ab"], case24["lat"], case24["Kn"], case24["Tv"]
    ups, free = case24["ups"], case24["free"]
    b = np.stack([-O.sc_apply(lat, ups[k], Kn, Tv) * free[k][:, None] for k in range(3)])
    x, info = ab.ir(case24["Kd"], case24["Td"], torch.as_tensor(b, device="cuda"), tol=1e-8)
    assert (info.status == 0).all() and (info.relres <= 1e-8).all()
    x = x.cpu().numpy()
    for k in range(3):
        uref, _ = O.solve_pcg(lat, Kn, Tv, ~free[k], ups[k], tol=1e-12)
        assert relmax(ups[k] + x[k], uref) < 1e-6, k


def test_amg_batch_equals_alone():
    """Two specimens x three loads in one batch give each specimen's results solved alone."""
    n = 16
    specs = [specimen(n, s, 2.5) for s in (5, 6)]
    lat = specs[0][0]
    free, ups = bcs(lat, n)
    dl = core.DeviceLattice(lat, "cuda")
    Kd = torch.as_tensor(np.stack([s[1] for s in specs]), device="cuda")
    Td = torch.as_tensor(np.stack([s[2] for s in specs]), device="cuda")
    upd = torch.as_tensor(np.stack([ups, ups]), device="cuda")
    b = -core.kmv(dl, upd, Kd[:, None], Td[:, None]) * torch.as_tensor(free, device="cuda")[None, :, :, None]

    def solve(K, T, bb):
        ab = GA.AmgBatch(dl, bb.shape[0] * 3, 3, free, **GA.AMG_CFG)
        ab.setup(core.pack(K, torch.float32), core.pack(T, torch.float32), core.block_jacobi(dl, K, T, torch.float32))
        x, info = ab.ir(K, T, bb.reshape(-1, lat.N, 3), tol=1e-8)
        ab.close()
        return x.reshape(bb.shape), info

    xb, ib = solve(Kd, Td, b)
    assert (ib.status == 0).all()
    for s in range(2):
        xa, ia = solve(Kd[s:s + 1], Td[s:s + 1], b[s:s + 1])
        assert (ia.status == 0).all()
        assert relmax(xb[s].cpu().numpy(), xa[0].cpu().numpy()) < 1e-7


def test_amg3d_mirror(case24):
    """The reference-named mirror: AMGGeom / AMG3D(...).vcycle / .pcg on one BC box."""
    lat, Kn, Tv, free, ups = case24["lat"], case24["Kn"], case24["Tv"], case24["free"], case24["ups"]
    geo = GA.AMGGeom(lat, free[0], agg=3, coarse_max=1000)
    assert geo.grids == [tuple(g) for g in case24["orc"][0].geo.grids]
    h = GA.AMG3D(geo, Kn, Tv, nu=1, gamma=2, power_its=5)
    assert h.rho0 > 0 and all(r > 0 for r in h.rho)
    b = -O.sc_apply(lat, ups[0], Kn, Tv) * free[0][:, None]
    x, it, rel = h.pcg(b, 1e-8)
    assert rel <= 1e-8 and it > 0
    uref, _ = O.solve_pcg(lat, Kn, Tv, ~free[0], ups[0], tol=1e-12)
    assert relmax(ups[0] + x, uref) < 1e-6
    z = h.vcycle(b)
    assert z.shape == b.shape and np.isfinite(z).all()


def test_repeated_solves_with_reused_workspace(case24):
    """Back-to-back solves reuse the caching allocator's blocks: a solve must not depend on what an earlier solve left
    in its workspace (the zero start skips the first FP64 K x)."""
    ab, lat, Kn, Tv = case24["ab"], case24["lat"], case24["Kn"], case24["Tv"]
    ups, free = case24["ups"], case24["free"]
    b = torch.as_tensor(np.stack([-O.sc_apply(lat, ups[k], Kn, Tv) * free[k][:, None] for k in range(3)]),
                        device="cuda")
    x1, i1 = ab.ir(case24["Kd"], case24["Td"], b, tol=1e-8)
    x2, i2 = ab.ir(case24["Kd"], case24["Td"], 3.0 * b, tol=1e-8)
    x3, i3 = ab.ir(case24["Kd"], case24["Td"], b, tol=1e-8)
    for i in (i1, i2, i3):
        assert (i.status == 0).all() and (i.relres <= 1e-8).all() and (i.iters > 0).all()
    assert relmax(x2.cpu().numpy(), 3.0 * x1.cpu().numpy()) < 1e-7
    assert relmax(x3.cpu().numpy(), x1.cpu().numpy()) < 1e-12


def test_core_ir_repeated_solves():
    """The block-Jacobi mixed solve (core.ir) twice on one batch: the second from zero again, same answer."""
    n = 16
    lat, Kn, Tv = specimen(n, 7, 2.5)
    free, ups = bcs(lat, n)
    dl = core.DeviceLattice(lat, "cuda")
    Kd = torch.as_tensor(Kn, device="cuda")[None, None]
    Td = torch.as_tensor(Tv, device="cuda")[None, None]
    upd = torch.as_tensor(ups, device="cuda")[None]
    fr = torch.as_tensor(free, device="cuda", dtype=torch.float64)
    b = -core.kmv(dl, upd, Kd, Td) * fr[None, :, :, None]
    x1, i1 = core.ir(dl, Kd, Td, b, free=fr, tol=1e-8)
    x2, i2 = core.ir(dl, Kd, Td, 2.0 * b, free=fr, tol=1e-8)
    assert (i1.status == 0).all() and (i2.status == 0).all() and (i2.iters > 0).all()
    assert relmax(x2.cpu().numpy(), 2.0 * x1.cpu().numpy()) < 1e-7
