"""GPU parity of the persistent CG engine (csrc/cg_persist.cu: one cooperative kernel per solve, team barriers between
the phases of an iteration) against the graph-launched engine of csrc/cg.cu, which the other GPU tests pin to the
oracle and the reference's golden vectors.

Both engines run the same algorithm with the same stopping and freezing rules; only the grouping of the FP64 inner
product partials differs, so iteration counts agree within 1 on short solves and within 0.5% on runs of thousands of
iterations of ill-conditioned problems (where rounding differences shift the last test), and solutions agree to the
solve tolerance.  Covered: 2D and 3D, plain CG and block-Jacobi PCG, FP64 and FP32 (inside the mixed-precision
refinement), per-DOF masks, empty and early-converging systems, a nonzero start, team shapes with one system per team
over several blocks and with several systems per single-block team, and a masked lattice (table neighbours).
"""
import numpy as np
import pytest

import oracle as O
from conftest import relmax
from lpm_b200 import _lib as L
from lpm_b200 import core, geom as G, micro

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda"
LA, PE = L.ENGINE_LAUNCHED, L.ENGINE_PERSISTENT


def T(a, dt=torch.float64):
    return torch.as_tensor(np.asarray(a), device=DEV, dtype=dt)


def grf2d(n, seeds):
    """Two-phase 2D specimens (the cfg-1 generator) with uniaxial tension."""
    lat = G.SquareLattice(n, n, 1.0)
    Kn, Tv = [], []
    for sd in seeds:
        ph = micro.grf_two_phase(n, n, 6.0, 0.30, sd)
        C = G.iso_C2d(np.where(ph == 1, 10.0, 1.0), 0.25, plane="stress")
        k, t = G.bond_params_two_end_mean(lat, G.square_params_from_C(C))
        Kn.append(k)
        Tv.append(t)
    fixed, up, _ = G.uniaxial_tension_2d(lat, 1e-3)
    return lat, np.array(Kn), np.array(Tv), fixed, np.where(fixed, up, 0.0)


def close_iters(ia, ib):
    a, b = ia.iters.astype(int), ib.iters.astype(int)
    return bool((np.abs(a - b) <= np.maximum(1, np.maximum(a, b) // 200)).all())


def both(dl, Kn, Tv, b, **kw):
    xa, ia = core.cg(dl, Kn, Tv, b, engine=LA, **kw)
    xp, ip = core.cg(dl, Kn, Tv, b, engine=PE, **kw)
    return xa.cpu().numpy(), ia, xp.cpu().numpy(), ip


def test_persistent_2d_plain_fp64_cfg1_shape():
    """cg2plain semantics on three 128^2 specimens (the cfg-1 solve): same iterations within 1, same solution."""
    lat, Kn, Tv, fixed, up = grf2d(128, [0, 1, 2])
    dl = core.DeviceLattice(lat)
    free = T(~fixed)
    b = -core.kmv(dl, T(up)[None].expand(3, -1, -1), T(Kn), T(Tv)) * free
    assert L.load().lpm_cg_persistent_fits(dl.ref, core._batch(3, 1, 1), L.LPM_F64) == 1
    xa, ia, xp, ip = both(dl, T(Kn), T(Tv), b, free=free, tol=1e-10, maxit=100000, check=1, precheck=True)
    assert (ia.status == 0).all() and (ip.status == 0).all() and (ip.relres <= 1e-10).all()
    assert close_iters(ia, ip)
    assert relmax(xp, xa) < 1e-8
    # the oracle's own plain CG on specimen 0 (timing/t2d/cg2plain.py:11-68)
    _, cinfo = O.sq_solve_cg(lat, Kn[0], Tv[0], fixed, up, tol=1e-10)
    assert abs(int(ip.iters[0]) - int(cinfo["iters"])) <= max(2, int(cinfo["iters"]) // 200)


def test_persistent_3d_pcg_masks_and_freezing():
    """Block-Jacobi PCG on a 10^3 box, 4 loads of two BC boxes, one empty right-hand side and one scaled copy."""
    lat = G.LatticeGeom(10, 10, 10, 1.0)
    rng = np.random.default_rng(2)
    ph = (rng.random(lat.N) < 0.3).astype(float)
    C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    dl = core.DeviceLattice(lat)
    free, bs = [], []
    for ld in ("k_xx", "tb_tz", "k_xx", "k_xx"):
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk // 2, (5, 5, 5), 2)
        upm = np.where(fixed[:, None], up, 0.0)
        free.append(~fixed)
        bs.append(-O.sc_apply(lat, upm, Kn, Tv) * (~fixed)[:, None])
    bs[2] = 0.0 * bs[2]
    bs[3] = 2.5 * bs[3]
    fr = T(np.array(free))
    Kd, Td = T(Kn)[None], T(Tv)[None]
    M = core.block_jacobi(dl, Kd, Td, torch.float64)
    xa, ia, xp, ip = both(dl, Kd, Td, T(np.array(bs))[None], Minv=M, free=fr[None], tol=1e-10, maxit=3000, check=1)
    assert ip.iters[2] == 0 and ip.relres[2] == 0.0 and np.abs(xp[0, 2]).max() == 0.0
    assert (ip.status == 0).all() and close_iters(ia, ip)
    assert relmax(xp, xa) < 1e-8
    assert relmax(xp[0, 3], 2.5 * xp[0, 0]) < 1e-9


def test_persistent_many_systems_per_team():
    """More systems than resident blocks: several systems per single-block team (8^2 lattice, 1000 systems)."""
    lat = G.SquareLattice(8, 8, 1.0)
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(5)
    Kn = rng.uniform(0.8, 1.2, (lat.N, lat.NN)) * lat.valid
    Tv = rng.uniform(-0.03, 0.03, (lat.N, lat.NN)) * lat.valid
    Kn = 0.5 * (Kn + Kn[np.maximum(lat.nbr, 0), np.arange(lat.NN) ^ 1] * lat.valid)  # symmetric per bond
    Tv = 0.5 * (Tv + Tv[np.maximum(lat.nbr, 0), np.arange(lat.NN) ^ 1] * lat.valid)
    fixed, _, _ = G.uniaxial_tension_2d(lat, 1e-3)
    S = 1000
    b = rng.standard_normal((S, lat.N, 2)) * (~fixed)
    xa, ia, xp, ip = both(dl, T(Kn), T(Tv), T(b), free=T(~fixed), tol=1e-9, maxit=2000, check=1)
    assert (ip.status == 0).all() and (ip.relres <= 1e-9).all()
    assert close_iters(ia, ip)
    assert relmax(xp, xa) < 1e-7


def test_persistent_nonzero_start_and_fp32_ir():
    """A nonzero start (x_is_zero = 0: the kernel reads K x) and the FP32 inner solves of the refinement."""
    lat, Kn, Tv, fixed, up = grf2d(64, [4, 5])
    dl = core.DeviceLattice(lat)
    free = T(~fixed)
    b = -core.kmv(dl, T(up)[None].expand(2, -1, -1), T(Kn), T(Tv)) * free
    x0, _ = core.cg(dl, T(Kn), T(Tv), b, free=free, tol=1e-3, maxit=10000, engine=LA)
    xa, ia = core.cg(dl, T(Kn), T(Tv), b, x=x0, free=free, tol=1e-10, maxit=10000, engine=LA)
    xp, ip = core.cg(dl, T(Kn), T(Tv), b, x=x0, free=free, tol=1e-10, maxit=10000, engine=PE)
    assert (ip.status == 0).all() and close_iters(ia, ip)
    assert relmax(xp.cpu().numpy(), xa.cpu().numpy()) < 1e-8
    ya, ja = core.ir(dl, T(Kn), T(Tv), b, free=free, tol=1e-9, inner_tol=1e-4, engine=LA)
    yp, jp = core.ir(dl, T(Kn), T(Tv), b, free=free, tol=1e-9, inner_tol=1e-4, engine=PE)
    assert (jp.status == 0).all() and (jp.relres <= 1e-9).all()
    assert relmax(yp.cpu().numpy(), ya.cpu().numpy()) < 1e-7


def test_persistent_masked_lattice():
    """Table neighbours (a 10 x 8 x 6 box with a spherical void, the x = 0 face clamped): plain FP64 CG on both
    engines."""
    nx, ny, nz = 10, 8, 6
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    active = ((i - 5.0) ** 2 + (j - 4.0) ** 2 + (k - 3.0) ** 2 > 4.0).ravel()
    lat = G.LatticeGeom(nx, ny, nz, 1.0, active=active)
    assert not lat.full
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(9)
    Kn = np.where(lat.valid, 1.0 + 0.1 * rng.random((lat.N, lat.NN)), 0.0)
    Tv = np.where(lat.valid, 0.02 * rng.random((lat.N, lat.NN)), 0.0)
    Kn = 0.5 * (Kn + Kn[np.maximum(lat.nbr, 0), np.arange(lat.NN) ^ 1] * lat.valid)
    Tv = 0.5 * (Tv + Tv[np.maximum(lat.nbr, 0), np.arange(lat.NN) ^ 1] * lat.valid)
    free = lat.ijk[:, 0] > 0
    b = rng.standard_normal((2, lat.N, 3)) * free[:, None]
    xa, ia, xp, ip = both(dl, T(Kn), T(Tv), T(b), free=T(free), tol=1e-10, maxit=5000, check=1)
    assert (ia.status == 0).all() and (ip.status == 0).all()
    assert close_iters(ia, ip)
    assert relmax(xp, xa) < 1e-8


def test_team_barrier_expiry_reports_timeout_and_leaves_the_gpu_usable():
    """With the wait bound at 0 every team-barrier wait that does not find its barrier passed at once expires: the
    solve returns LPM_ERR_TIMEOUT (the kernel's blocks record the code and return; nothing hangs or faults), and the
    next solve with the default bound on the same GPU gives the launched engine's answer."""
    lat, Kn, Tv, fixed, up = grf2d(128, [0])
    dl = core.DeviceLattice(lat)
    free = T(~fixed)
    b = -core.kmv(dl, T(up)[None], T(Kn), T(Tv)) * free
    lib = L.load()
    prev = lib.lpm_set_wait_limit_ns(0)
    try:
        with pytest.raises(L.LPMError, match=r"code -5"):
            core.cg(dl, T(Kn), T(Tv), b, free=free, tol=1e-10, maxit=20000, check=1, engine=PE)
    finally:
        assert lib.lpm_set_wait_limit_ns(prev) == 0
    assert prev == 2000000000
    torch.cuda.synchronize()
    xa, ia, xp, ip = both(dl, T(Kn), T(Tv), b, free=free, tol=1e-10, maxit=20000, check=1)
    assert (ip.status == 0).all() and close_iters(ia, ip)
    assert relmax(xp, xa) < 1e-8
