"""Batches whose last coefficient set is only partly filled (5 systems over sets of 3): the packed operators run a pair
(FP32) or lane group (FP64) with no system behind it, and the engines must neither read nor write past the batch.
Each solve is checked against the oracle's FP64 block-Jacobi PCG to 1e-12 on the same coefficient set and load.

Bars: FP64 CG to 1e-10 within 1e-7 relative displacement; FP32 CG to 1e-5 within 1e-4; the AMG mixed-precision
solve to 1e-8 within 1e-6 (relative L2 per system)."""
import numpy as np
import pytest
import torch

import oracle as O
from lpm_b200 import _lib as L
from lpm_b200 import amg as GA
from lpm_b200 import core
from lpm_b200 import geom as G
from lpm_b200 import micro as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
LOADS = ["k_xx", "k_yz", "k_xy"]   # one load per system slot of a set (the KUBC box for all three)
NSYS, RPS = 5, 3


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.fixture(scope="module")
def case():
    n = 16
    lat = G.LatticeGeom(n, n, n, 1.0)
    Kn, Tv = [], []
    for seed in (0, 1):
        ph, _ = M.spheres(n, n, n, 0.25, 2.5, np.random.default_rng(seed), rjit=0.0)
        C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
        k, t = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
        Kn.append(k)
        Tv.append(t)
    free, ups = [], []
    for ld in LOADS:
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        free.append(~fixed)
        ups.append(np.where(fixed[:, None], up, 0.0))
    sys_set = [s // RPS for s in range(NSYS)]
    sys_load = [s % RPS for s in range(NSYS)]
    b = np.stack([-O.sc_apply(lat, ups[sys_load[s]], Kn[sys_set[s]], Tv[sys_set[s]]) * free[sys_load[s]][:, None]
                  for s in range(NSYS)])
    ref = [O.solve_pcg(lat, Kn[sys_set[s]], Tv[sys_set[s]], ~free[sys_load[s]], ups[sys_load[s]], tol=1e-12)[0] -
           ups[sys_load[s]] for s in range(NSYS)]
    return dict(lat=lat, dl=core.DeviceLattice(lat, DEV), Kn=np.array(Kn), Tv=np.array(Tv), free=np.array(free),
                b=b, ref=ref, sys_load=sys_load)


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_packed_cg_partial_last_set(case, dt):
    """Plain CG on the packed operators (FP32: pair engine, FP64: the FP64 pair operator) with 5 systems, sets of 3."""
    tdt = torch.float64 if dt == "f64" else torch.float32
    Kd, Td = torch.as_tensor(case["Kn"], device=DEV), torch.as_tensor(case["Tv"], device=DEV)
    Kp, Tp = core.pack(Kd, tdt), core.pack(Td, tdt)
    fr = torch.as_tensor(case["free"][case["sys_load"]], device=DEV, dtype=tdt)
    b = torch.as_tensor(case["b"], device=DEV, dtype=tdt)
    tol = 1e-10 if dt == "f64" else 1e-5
    x, info = core.cg(case["dl"], Kp, Tp, b, free=fr, tol=tol, maxit=20000, check=1, layout=L.LAYOUT_SOA,
                      rhs_per_set=RPS, engine=L.ENGINE_LAUNCHED)
    assert (info.status == 0).all()
    bar = 1e-7 if dt == "f64" else 1e-4
    for s in range(NSYS):
        assert rel_l2(x[s].double().cpu().numpy(), case["ref"][s]) < bar, (dt, s)


def test_amg_ir_partial_last_set(case):
    """AMG-preconditioned mixed-precision solve with 5 systems over sets of 3 (one box: the KUBC ring)."""
    dl = case["dl"]
    Kd, Td = torch.as_tensor(case["Kn"], device=DEV), torch.as_tensor(case["Tv"], device=DEV)
    ab = GA.AmgBatch(dl, NSYS, RPS, case["free"], **GA.AMG_CFG)
    ab.setup(core.pack(Kd, torch.float32), core.pack(Td, torch.float32), core.block_jacobi(dl, Kd, Td, torch.float32))
    x, info = ab.ir(Kd, Td, torch.as_tensor(case["b"], device=DEV), tol=1e-8, inner_tol=1e-4)
    assert (info.status == 0).all() and (info.relres <= 1e-8).all()
    for s in range(NSYS):
        assert rel_l2(x[s].cpu().numpy(), case["ref"][s]) < 1e-6, s
    ab.close()


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_packed_cg_2d_partial_last_set(dt):
    """Square-lattice CG on the packed operator (FP32: two systems per pass of the multi-system tile kernel) with 5
    systems over sets of 3 and three grip loads, so systems leave the batch at different iterations; each against
    the oracle's plain CG to 1e-12 (FP32 CG runs to 1e-6 here), and against the same systems given one coefficient
    set each."""
    nx, ny = 40, 28
    lat = G.Lattice2D("square", nx, ny, 1.0)
    dl = core.DeviceLattice(lat)
    Kn, Tv = [], []
    for seed in (0, 1):
        ph = np.random.default_rng(seed).random(lat.N) < 0.3
        C = G.iso_C2d(np.where(ph, 10.0, 1.0), 0.25, plane="stress")
        k, t = G.bond_params_two_end_mean(lat, G.square_params_from_C(C))
        Kn.append(k)
        Tv.append(t)
    loads = ["tb_ty", "tb_sx", "lr_tx"]
    sys_set = [s // RPS for s in range(NSYS)]
    fr, ups, b, ref = [], [], [], []
    for s in range(NSYS):
        fixed, up, _ = G.prescribed2d(loads[s % RPS], lat.x, lat.ij, nx, ny, 1, 1.0)
        fd = np.repeat(fixed[:, None], 2, axis=1)
        upm = np.where(fd, up, 0.0)
        fr.append(~fd)
        ups.append(upm)
        b.append(-O.sq_kmv(lat, upm.ravel(), Kn[sys_set[s]], Tv[sys_set[s]]).reshape(-1, 2) * ~fd)
        ref.append(O.sq_solve_cg(lat, Kn[sys_set[s]], Tv[sys_set[s]], fd, upm, tol=1e-12)[0] - upm)
    tdt = torch.float64 if dt == "f64" else torch.float32
    tol = 1e-10 if dt == "f64" else 1e-6
    bd = torch.as_tensor(np.array(b), device=DEV, dtype=tdt)
    fd = torch.as_tensor(np.array(fr), device=DEV, dtype=tdt)
    xs = []
    for sets in ([0, 1], sys_set):   # sets of 3 (the last partly filled), then one set per system
        Kp = core.pack(torch.as_tensor(np.array(Kn)[sets], device=DEV), tdt)
        Tp = core.pack(torch.as_tensor(np.array(Tv)[sets], device=DEV), tdt)
        x, info = core.cg(dl, Kp, Tp, bd, free=fd, tol=tol, maxit=20000, check=1, layout=L.LAYOUT_SOA,
                          rhs_per_set=RPS if len(sets) == 2 else 1, engine=L.ENGINE_LAUNCHED)
        assert (info.status == 0).all()
        xs.append(x.double().cpu().numpy())
    bar = 1e-7 if dt == "f64" else 1e-4
    for s in range(NSYS):
        assert rel_l2(xs[0][s], ref[s]) < bar, (dt, s, rel_l2(xs[0][s], ref[s]))
        # same arithmetic per system either way; FP32 CG may amplify last-bit differences of contracted products
        assert rel_l2(xs[0][s], xs[1][s]) < (1e-12 if dt == "f64" else 1e-5), (dt, s, rel_l2(xs[0][s], xs[1][s]))


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_cg_2d_reference_layout_staged(dt):
    """Square-lattice CG on reference-layout coefficients without packing (the operator stages both coefficient
    arrays of each tile in shared memory) against the same solve on packed coefficients and against the oracle."""
    nx, ny = 45, 30
    lat = G.Lattice2D("square", nx, ny, 1.0)
    dl = core.DeviceLattice(lat)
    ph = np.random.default_rng(4).random(lat.N) < 0.3
    C = G.iso_C2d(np.where(ph, 10.0, 1.0), 0.25, plane="stress")
    k, t = G.bond_params_two_end_mean(lat, G.square_params_from_C(C))
    fr, b, ref = [], [], []
    for ld in ("tb_ty", "lr_tx"):
        fixed, up, _ = G.prescribed2d(ld, lat.x, lat.ij, nx, ny, 1, 1.0)
        fd = np.repeat(fixed[:, None], 2, axis=1)
        upm = np.where(fd, up, 0.0)
        fr.append(~fd)
        b.append(-O.sq_kmv(lat, upm.ravel(), k, t).reshape(-1, 2) * ~fd)
        ref.append(O.sq_solve_cg(lat, k, t, fd, upm, tol=1e-12)[0] - upm)
    tdt = torch.float64 if dt == "f64" else torch.float32
    Kd = torch.as_tensor(k, device=DEV, dtype=tdt)[None]
    Td = torch.as_tensor(t, device=DEV, dtype=tdt)[None]
    bd = torch.as_tensor(np.array(b), device=DEV, dtype=tdt)
    fd_ = torch.as_tensor(np.array(fr), device=DEV, dtype=tdt)
    tol = 1e-10 if dt == "f64" else 1e-6
    xs = []
    for pk in (False, True):
        x, info = core.cg(dl, Kd, Td, bd, free=fd_, tol=tol, maxit=20000, check=1, engine=L.ENGINE_LAUNCHED,
                          pack2d=pk)
        assert (info.status == 0).all()
        xs.append(x.double().cpu().numpy())
    bar = 1e-7 if dt == "f64" else 1e-4
    for s in range(2):
        assert rel_l2(xs[0][s], ref[s]) < bar, (dt, s, rel_l2(xs[0][s], ref[s]))
        assert rel_l2(xs[0][s], xs[1][s]) < (1e-12 if dt == "f64" else 1e-5), (dt, s)


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_packed_pcg_2d_sets(dt):
    """Block-Jacobi PCG on the packed square-lattice operator with 2 sets x 3 systems (the FP32 operator applies a
    set's systems two per pass and forms the p-update while staging), against the oracle's solution."""
    nx, ny = 40, 28
    lat = G.Lattice2D("square", nx, ny, 1.0)
    dl = core.DeviceLattice(lat)
    Kn, Tv = [], []
    for seed in (2, 3):
        ph = np.random.default_rng(seed).random(lat.N) < 0.3
        C = G.iso_C2d(np.where(ph, 10.0, 1.0), 0.25, plane="stress")
        k, t = G.bond_params_two_end_mean(lat, G.square_params_from_C(C))
        Kn.append(k)
        Tv.append(t)
    loads = ["tb_ty", "tb_sx", "lr_tx"]
    fr, b, ref = [], [], []
    for s in range(6):
        fixed, up, _ = G.prescribed2d(loads[s % 3], lat.x, lat.ij, nx, ny, 1, 1.0)
        fd = np.repeat(fixed[:, None], 2, axis=1)
        upm = np.where(fd, up, 0.0)
        fr.append(~fd)
        b.append(-O.sq_kmv(lat, upm.ravel(), Kn[s // 3], Tv[s // 3]).reshape(-1, 2) * ~fd)
        ref.append(O.sq_solve_cg(lat, Kn[s // 3], Tv[s // 3], fd, upm, tol=1e-12)[0] - upm)
    tdt = torch.float64 if dt == "f64" else torch.float32
    K64 = torch.as_tensor(np.array(Kn), device=DEV)
    T64 = torch.as_tensor(np.array(Tv), device=DEV)
    M = core.block_jacobi(dl, K64, T64, tdt)
    tol = 1e-10 if dt == "f64" else 1e-6
    x, info = core.cg(dl, core.pack(K64, tdt), core.pack(T64, tdt), torch.as_tensor(np.array(b), device=DEV, dtype=tdt),
                      Minv=M, free=torch.as_tensor(np.array(fr), device=DEV, dtype=tdt), tol=tol, maxit=20000,
                      check=1, layout=L.LAYOUT_SOA, rhs_per_set=3, engine=L.ENGINE_LAUNCHED)
    assert (info.status == 0).all()
    bar = 1e-7 if dt == "f64" else 1e-4
    for s in range(6):
        assert rel_l2(x[s].double().cpu().numpy(), ref[s]) < bar, (dt, s, rel_l2(x[s].double().cpu().numpy(), ref[s]))
