"""GPU parity of the CUDA library (through the C ABI) against the CPU oracle and the reference's golden vectors.

Tolerances: FP64 kernels 1e-13 (max-abs relative to the max of the reference array); FP32 kernels 2e-6; solves to
rel. residual 1e-12 agree with SuperLU to 1e-9; mixed-precision solves to 1e-8 agree with the FP64 oracle to 1e-6
(displacement, relative L2), the bar of the mixed-precision path.  Connectivity is bit-exact.
"""
import numpy as np
import pytest

import oracle as O
from conftest import relmax
from lpm_b200 import _lib as L
from lpm_b200 import core, geom as G

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda"
ENGINES = pytest.mark.parametrize("engine", [L.ENGINE_LAUNCHED, L.ENGINE_PERSISTENT], ids=["launched", "persistent"])


def T(a, dt=torch.float64):
    return torch.as_tensor(np.asarray(a), device=DEV, dtype=dt)


def rel_l2(a, b):
    a = np.asarray(a, float).ravel()
    b = np.asarray(b, float).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def sym_params(lat, rng, kn=(0.8, 1.2), tv=(-0.03, 0.03)):
    """Random symmetric per-bond parameters (same value on (i,k) and (q,k^1)), zero on missing bonds."""
    Kn = np.zeros((lat.N, lat.NN))
    Tv = np.zeros((lat.N, lat.NN))
    i, k = np.nonzero(lat.valid & (np.arange(lat.NN)[None, :] % 2 == 0))
    q = lat.nbr[i, k]
    a = rng.uniform(*kn, size=i.size)
    b = rng.uniform(*tv, size=i.size)
    Kn[i, k] = a
    Kn[q, k ^ 1] = a
    Tv[i, k] = b
    Tv[q, k ^ 1] = b
    return Kn, Tv


@pytest.fixture(scope="module")
def sc12(gsc):
    lat = G.LatticeGeom(12, 12, 12, 1.0)
    return lat, core.DeviceLattice(lat), gsc["Kn"], gsc["Tv"]


# ------------------------------------------------------------------------------------------------------- K . u
def test_kmv_sc_golden(gsc, sc12):
    lat, dl, Kn, Tv = sc12
    f = core.kmv(dl, T(gsc["u"]), T(Kn), T(Tv)).cpu().numpy()
    assert relmax(f, gsc["Ku"]) < 1e-13
    f32 = core.kmv(dl, T(gsc["u"], torch.float32), T(Kn, torch.float32), T(Tv, torch.float32)).cpu().numpy()
    assert relmax(f32, gsc["Ku"]) < 2e-6


@pytest.mark.parametrize("shape", [(5, 7, 9), (33, 9, 3), (3, 3, 3), (40, 17, 6)])
def test_kmv_sc_odd_sizes_batched(shape):
    rng = np.random.default_rng(sum(shape))
    lat = G.LatticeGeom(*shape)
    dl = core.DeviceLattice(lat)
    B, Lc = 2, 3
    Kn = [sym_params(lat, rng)[0] for _ in range(B)]
    Tv = [rng.uniform(-0.05, 0.05, (lat.N, 18)) * lat.valid for _ in range(B)]   # non-symmetric Tv
    u = rng.standard_normal((B, Lc, lat.N, 3))
    f = core.kmv(dl, T(u), T(np.array(Kn))[:, None], T(np.array(Tv))[:, None]).cpu().numpy()
    for b in range(B):
        for l in range(Lc):
            assert relmax(f[b, l], O.sc_apply(lat, u[b, l], Kn[b], Tv[b])) < 1e-13
    # packed SoA layout gives the same result
    Kp = core.pack(T(np.array(Kn)), torch.float64)
    Tp = core.pack(T(np.array(Tv)), torch.float64)
    from lpm_b200 import _lib
    fp = core.kmv(dl, T(u).reshape(B * Lc, lat.N, 3), Kp, Tp, layout=_lib.LAYOUT_SOA, rhs_per_set=Lc).cpu().numpy()
    assert relmax(fp.reshape(f.shape), f) < 1e-13


def test_kmv_sc_masked_lattice(gsc):
    lat = G.LatticeGeom(7, 5, 4, 1.5, active=gsc["m_active"])
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(3)
    Kn, Tv = sym_params(lat, rng)
    u = rng.standard_normal((2, lat.N, 3))
    f = core.kmv(dl, T(u), T(Kn), T(Tv)).cpu().numpy()
    for s in range(2):
        assert relmax(f[s], O.sc_apply(lat, u[s], Kn, Tv)) < 1e-13


def test_kmv_sq(gsq):
    lat = G.Lattice2D("square", 16, 12, 1.0)
    dl = core.DeviceLattice(lat)
    u = gsq["u"].reshape(-1, 2)
    f = core.kmv(dl, T(u), T(gsq["Kn_ns"]), T(gsq["Tv_ns"])).cpu().numpy().ravel()
    assert relmax(f, gsq["f_ns"]) < 1e-13
    f32 = core.kmv(dl, T(u, torch.float32), T(gsq["Kn_ns"], torch.float32), T(gsq["Tv_ns"], torch.float32))
    assert relmax(f32.cpu().numpy().ravel(), gsq["f_ns"]) < 2e-6
    # masked square lattice through the neighbour table
    lm = G.Lattice2D("square", 9, 7, 0.5, active=gsq["m_active"])
    dm = core.DeviceLattice(lm)
    rng = np.random.default_rng(8)
    Kn, Tv = rng.uniform(0.5, 1.5, (lm.N, 8)) * lm.valid, rng.uniform(-0.1, 0.1, (lm.N, 8)) * lm.valid
    um = rng.standard_normal((lm.N, 2))
    assert relmax(core.kmv(dm, T(um), T(Kn), T(Tv)).cpu().numpy().ravel(), O.sq_kmv(lm, um, Kn, Tv)) < 1e-13


# ----------------------------------------------------------------------------------------- geometry on device
def test_build_nbr_bit_exact(gsc, gsq):
    lat = G.LatticeGeom(7, 5, 4, 1.5, active=gsc["m_active"])
    nb = core.build_nbr(lat).cpu().numpy()
    assert nb.dtype == np.int64 and np.array_equal(nb, gsc["m_nbr"].astype(np.int64))
    full = G.LatticeGeom(12, 12, 12)
    assert np.array_equal(core.build_nbr(full).cpu().numpy(), gsc["nbr"].astype(np.int64))
    lm = G.Lattice2D("square", 9, 7, 0.5, active=gsq["m_active"])
    assert np.array_equal(core.build_nbr(lm).cpu().numpy(), gsq["m_nbr"].astype(np.int64))


# ---------------------------------------------------------------------------------------------- preconditioner
def test_block_jacobi(gsc, gsq, sc12):
    lat, dl, Kn, Tv = sc12
    M, D = core.block_jacobi(dl, T(Kn), T(Tv), torch.float64, want_D=True)
    assert relmax(D[0].cpu().numpy(), gsc["D"]) < 1e-13
    I = torch.einsum("nab,nbc->nac", M[0], D[0]).cpu().numpy()
    assert np.abs(I - np.eye(3)[None]).max() < 1e-10
    lat2 = G.Lattice2D("square", 16, 12, 1.0)
    d2 = core.DeviceLattice(lat2)
    M2 = core.block_jacobi(d2, T(gsq["Kn"]), T(gsq["Tv"]), torch.float64)[0].cpu().numpy()
    free = ~gsq["diag_fixed"]
    assert relmax(M2[free], gsq["Binv"][free]) < 1e-13


# ------------------------------------------------------------------------------------------------------- solves
def _bc(lat, ld, s):
    nc = lat.nx // s
    fixed, up, mov = G.prescribed(ld, lat.x, lat.ijk // s, (nc,) * 3, s)
    return fixed, up, mov


@ENGINES
def test_cg_fp64_matches_oracle(gsc, sc12, engine):
    """Plain FP64 CG (cgplain.cg3) and block-Jacobi PCG (lin3d.solve_pcg): same iterations, same answer, on both
    engines (graph-launched kernels; one persistent cooperative kernel)."""
    lat, dl, Kn, Tv = sc12
    for ld in ("k_xx", "tb_sx"):
        fixed, up, _ = _bc(lat, ld, 2)
        free = ~fixed
        upm = np.where(fixed[:, None], up, 0.0)
        b = -O.sc_apply(lat, upm, Kn, Tv) * free[:, None]
        x, info = core.cg(dl, T(Kn), T(Tv), T(b), free=T(free), tol=1e-8, maxit=5000, check=1, engine=engine)
        assert abs(int(info.iters[0]) - int(gsc["cg_it_%s" % ld])) <= 1
        assert relmax(x.cpu().numpy() + upm, gsc["cg_u_%s" % ld]) < 1e-6
        M = core.block_jacobi(dl, T(Kn), T(Tv), torch.float64)
        x, info = core.cg(dl, T(Kn), T(Tv), T(b), Minv=M, free=T(free), tol=1e-8, maxit=5000, check=1,
                          engine=engine)
        assert abs(int(info.iters[0]) - int(gsc["pcg_it_%s" % ld])) <= 1
        assert relmax(x.cpu().numpy() + upm, gsc["pcg_u_%s" % ld]) < 1e-6


def test_pcg_batched_vs_superlu(gsc, sc12):
    """All 9 loads of s = 2 as one batch (3 BC sets, per-system masks) to 1e-12 vs the reference's SuperLU."""
    lat, dl, Kn, Tv = sc12
    free, ups = [], []
    for ld in G.LOADS:
        fixed, up, _ = _bc(lat, ld, 2)
        free.append(~fixed)
        ups.append(np.where(fixed[:, None], up, 0.0))
    free, ups = np.array(free), np.array(ups)
    Kt, Tt = T(Kn), T(Tv)
    b = -core.kmv(dl, T(ups), Kt, Tt) * T(free)[..., None]
    M = core.block_jacobi(dl, Kt, Tt, torch.float64)
    x, info = core.cg(dl, Kt, Tt, b, Minv=M, free=T(free), tol=1e-12, maxit=5000, check=1)
    assert (info.status == 0).all() and (info.relres <= 1e-12).all()
    u = x.cpu().numpy() + ups
    cid = G.block_index(lat.ijk, 2, (6, 6, 6))
    for l, ld in enumerate(G.LOADS):
        ub = np.stack([np.bincount(cid, u[l][:, k]) for k in range(3)], 1) / 8
        assert relmax(ub, gsc["u_2_%s" % ld]) < 1e-9


@ENGINES
def test_mixed_precision_ir(gsc, sc12, engine):
    """FP32 inner PCG + FP64 refinement to 1e-8: FP64 true residual <= 1e-8 and <= 1e-6 rel. error vs SuperLU."""
    lat, dl, Kn, Tv = sc12
    for ld in ("k_xx", "lr_tx", "tb_tz"):
        s = 3 if ld == "tb_tz" else 2
        fixed, up, _ = _bc(lat, ld, s)
        free = ~fixed
        upm = np.where(fixed[:, None], up, 0.0)
        b = -O.sc_apply(lat, upm, Kn, Tv) * free[:, None]
        x, info = core.ir(dl, T(Kn), T(Tv), T(b), free=T(free), tol=1e-8, inner_tol=1e-5, engine=engine)
        xn = x.cpu().numpy()
        r = (b - O.sc_apply(lat, xn, Kn, Tv)) * free[:, None]
        assert np.linalg.norm(r) <= 1.0000001e-8 * np.linalg.norm(b)
        assert info.relres[0] <= 1e-8 and info.status[0] == 0
        assert rel_l2(xn + upm, gsc["ufull_%d_%s" % (s, ld)]) < 1e-6


def test_kmv_sq_sets_of_several_systems():
    """FP32 2D K.u with three systems per coefficient set (one block per tile and set, coefficients staged once) vs
    the oracle, and launched-engine FP32 PCG over such sets equals each set's systems solved alone."""
    lat = G.Lattice2D("square", 40, 19, 1.0)
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(11)
    KT = [sym_params(lat, rng) for _ in range(2)]
    Kn, Tv = np.array([k for k, _ in KT]), np.array([t for _, t in KT])
    u = rng.standard_normal((2, 3, lat.N, 2))
    f = core.kmv(dl, T(u, torch.float32), T(Kn, torch.float32)[:, None], T(Tv, torch.float32)[:, None])
    f = f.cpu().numpy()
    for c in range(2):
        for j in range(3):
            ref = O.sq_kmv(lat, u[c, j].ravel(), Kn[c], Tv[c]).reshape(-1, 2)
            assert relmax(f[c, j], ref) < 2e-6, (c, j)
    fixed, _, _ = G.uniaxial_tension_2d(lat, 1e-3)
    b = rng.standard_normal((2, 3, lat.N, 2)) * (~fixed)
    K32, T32 = T(Kn, torch.float32)[:, None], T(Tv, torch.float32)[:, None]
    M = core.block_jacobi(dl, T(Kn), T(Tv), torch.float32)
    kw = dict(free=T(~fixed), tol=1e-5, maxit=5000, check=1, engine=L.ENGINE_LAUNCHED)
    xb, ib = core.cg(dl, K32, T32, T(b, torch.float32), Minv=M, **kw)
    for c in range(2):
        for j in range(3):
            xa, ia = core.cg(dl, K32[c:c + 1], T32[c:c + 1], T(b[c:c + 1, j:j + 1], torch.float32), Minv=M[c:c + 1],
                             **kw)
            assert ib.status[3 * c + j] == 0 and abs(int(ib.iters[3 * c + j]) - int(ia.iters[0])) <= 1
            assert relmax(xb[c, j].cpu().numpy(), xa[0, 0].cpu().numpy()) < 1e-4


@ENGINES
def test_cg_2d_per_dof_mask(gsq, engine):
    """cg2plain.cg_mf semantics (per-DOF mask, initial-residual test) in FP64, and the mixed-precision path."""
    lat = G.Lattice2D("square", 16, 12, 1.0)
    dl = core.DeviceLattice(lat)
    fd, up = gsq["cg_fixed"], gsq["cg_up"]
    ub = np.where(fd, up, 0.0)
    Kn, Tv = gsq["Kn"], gsq["Tv"]
    b = (-O.sq_kmv(lat, ub, Kn, Tv) * (~fd).ravel()).reshape(-1, 2)
    x, info = core.cg(dl, T(Kn), T(Tv), T(b), free=T(~fd), tol=1e-10, maxit=100000, check=1, precheck=True,
                      engine=engine)
    assert abs(int(info.iters[0]) - int(gsq["cg_it"])) <= 1
    assert relmax(x.cpu().numpy().ravel() + ub.ravel(), gsq["cg_u"]) < 1e-8
    x, info = core.ir(dl, T(Kn), T(Tv), T(b), free=T(~fd), tol=1e-10, inner_tol=1e-5, precond=False,
                      engine=engine)
    assert rel_l2(x.cpu().numpy().ravel() + ub.ravel(), gsq["lu_u"]) < 1e-6


@ENGINES
def test_cg_freezing_and_status(engine):
    """Systems converge independently; a zero right-hand side returns 0 iterations; maxit reports NOT_CONVERGED."""
    lat = G.LatticeGeom(6, 6, 6)
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(0)
    Kn, Tv = sym_params(lat, rng)
    fixed, up, _ = _bc(lat, "k_xx", 2)
    free = ~fixed
    b0 = -O.sc_apply(lat, np.where(fixed[:, None], up, 0.0), Kn, Tv) * free[:, None]
    b = np.stack([b0, 0 * b0, 3 * b0])
    x, info = core.cg(dl, T(Kn), T(Tv), T(b), free=T(free), tol=1e-10, maxit=2000, engine=engine)
    assert info.iters[1] == 0 and info.relres[1] == 0.0
    assert info.iters[0] == info.iters[2] and (info.status == 0).all()
    xa = x.cpu().numpy()
    assert relmax(xa[2], 3 * xa[0]) < 1e-9 and np.abs(xa[1]).max() == 0.0
    _, info = core.cg(dl, T(Kn), T(Tv), T(b0), free=T(free), tol=1e-14, maxit=3, engine=engine)
    assert info.status[0] == 1 and info.iters[0] == 3


# ---------------------------------------------------------------------------------------------------- gradients
def test_grad_sc(ggrad):
    lat = G.LatticeGeom(4, 4, 4, 2.0)
    dl = core.DeviceLattice(lat)
    for pre in ("g3", "g3n"):
        gK, gT = core.bond_grad(dl, T(ggrad["g3_u"]), T(ggrad["g3_lam"]), T(ggrad[pre + "_Kn"]),
                                T(ggrad[pre + "_Tv"]))
        assert relmax(gK[0].cpu().numpy(), ggrad[pre + "_gK"]) < 1e-13
        assert relmax(gT[0].cpu().numpy(), ggrad[pre + "_gT"]) < 1e-13


def test_grad_sq(ggrad):
    lat = G.Lattice2D("square", 6, 5, 2.0)
    dl = core.DeviceLattice(lat)
    gK, gT = core.bond_grad(dl, T(ggrad["g2_u"].reshape(-1, 2)), T(ggrad["g2_lam"].reshape(-1, 2)),
                            T(ggrad["g2_Kn"]), T(ggrad["g2_Tv"]))
    assert relmax(gK[0].cpu().numpy(), ggrad["g2_gK"]) < 1e-13
    assert relmax(gT[0].cpu().numpy(), ggrad["g2_gT"]) < 1e-13


def test_grad_sums_over_loads(gsc, sc12):
    lat, dl, Kn, Tv = sc12
    rng = np.random.default_rng(4)
    u = rng.standard_normal((3, lat.N, 3))
    lam = rng.standard_normal((3, lat.N, 3))
    gK, gT = core.bond_grad(dl, T(u), T(lam), T(Kn)[None], T(Tv)[None])
    eK = sum(O.sc_grad(lat, Kn, Tv, u[l], lam[l])[0] for l in range(3))
    assert relmax(gK[0].cpu().numpy(), eK) < 1e-13


# ------------------------------------------------------------------------------------------------- post-process
def test_stress_energy(gsc, gsq, sc12):
    lat, dl, Kn, Tv = sc12
    u = T(gsc["u"])
    assert relmax(core.stress(dl, u, T(Kn), T(Tv)).cpu().numpy(), gsc["st"]) < 1e-13
    assert relmax(core.energy(dl, u, T(Kn), T(Tv)).cpu().numpy(), gsc["U"]) < 1e-13
    lat2 = G.Lattice2D("square", 16, 12, 1.0)
    d2 = core.DeviceLattice(lat2)
    u2 = T(gsq["u"].reshape(-1, 2))
    assert relmax(core.stress(d2, u2, T(gsq["Kn"]), T(gsq["Tv"])).cpu().numpy(), gsq["stress"]) < 1e-13
    assert relmax(core.energy(d2, u2, T(gsq["Kn"]), T(gsq["Tv"])).cpu().numpy(), gsq["energy"]) < 1e-13


# ------------------------------------------------------------------------------------- fused single-pass operator
@pytest.mark.parametrize("shape,rps,nset", [((5, 7, 9), 1, 2), ((33, 9, 3), 2, 1), ((40, 17, 6), 3, 2),
                                             ((64, 16, 20), 6, 1), ((31, 8, 17), 5, 2), ((48, 48, 48), 4, 1),
                                             ((36, 9, 5), 5, 2), ((8, 3, 2), 3, 1), ((4, 20, 33), 1, 3),
                                             ((96, 12, 40), 9, 1)])
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_fused_kmv(shape, rps, nset, dt):
    """Packed (SoA) full-box SC input runs the fused z-marching kernel: all tile/halo/partial-group cases."""
    from lpm_b200 import _lib
    rng = np.random.default_rng(sum(shape) + rps)
    lat = G.LatticeGeom(*shape)
    dl = core.DeviceLattice(lat)
    Kn = np.array([sym_params(lat, rng)[0] for _ in range(nset)])
    Tv = np.array([rng.uniform(-0.05, 0.05, (lat.N, 18)) * lat.valid for _ in range(nset)])
    u = rng.standard_normal((nset * rps, lat.N, 3))
    tdt = torch.float64 if dt == "f64" else torch.float32
    Kp, Tp = core.pack(T(Kn), tdt), core.pack(T(Tv), tdt)
    f = core.kmv(dl, T(u, tdt), Kp, Tp, layout=_lib.LAYOUT_SOA, rhs_per_set=rps).cpu().numpy()
    tol = 1e-13 if dt == "f64" else 3e-6
    for s in range(nset * rps):
        ref = O.sc_apply(lat, u[s], Kn[s // rps], Tv[s // rps])
        assert relmax(f[s], ref) < tol, s


@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_fused_kmv_partial_last_set(dt):
    """5 systems over coefficient sets of 3: the second set holds two systems, so the last pair group / lane of the
    packed operators has no system behind it and must neither read past u nor write past out."""
    from lpm_b200 import _lib
    rng = np.random.default_rng(11)
    lat = G.LatticeGeom(16, 12, 10)
    dl = core.DeviceLattice(lat)
    Kn = np.array([sym_params(lat, rng)[0] for _ in range(2)])
    Tv = np.array([rng.uniform(-0.05, 0.05, (lat.N, 18)) * lat.valid for _ in range(2)])
    u = rng.standard_normal((5, lat.N, 3))
    tdt = torch.float64 if dt == "f64" else torch.float32
    Kp, Tp = core.pack(T(Kn), tdt), core.pack(T(Tv), tdt)
    import ctypes
    uu = T(u, tdt).contiguous()
    out = torch.full((6, lat.N, 3), 7.0, dtype=tdt, device=DEV)   # one spare system after the batch, to catch writes
    lib = _lib.load()
    prec = _lib.LPM_F64 if dt == "f64" else _lib.LPM_F32
    scr = torch.empty(max(1, lib.lpm_kmv_scratch_bytes(dl.ref, prec, 5)), dtype=torch.uint8, device=DEV)
    name = "lpm_kmv_sc_f64" if dt == "f64" else "lpm_kmv_sc_f32"
    _lib.check(getattr(lib, name)(dl.ref, _lib.ptr(uu), _lib.ptr(Kp), _lib.ptr(Tp), _lib.LAYOUT_SOA,
                                  ctypes.byref(core._batch(5, 3)), _lib.ptr(out), _lib.ptr(scr), scr.numel(),
                                  _lib.stream_ptr(uu.device)), name)
    tol = 1e-13 if dt == "f64" else 3e-6
    for s in range(5):
        assert relmax(out[s].cpu().numpy(), O.sc_apply(lat, u[s], Kn[s // 3], Tv[s // 3])) < tol, s
    assert torch.all(out[5] == 7.0)


@pytest.mark.parametrize("shape,rps,nsys", [((40, 17), 3, 6), ((33, 9), 2, 4), ((64, 24), 5, 10), ((36, 20), 3, 5),
                                             ((70, 9), 4, 7), ((31, 8), 2, 3)])
@pytest.mark.parametrize("dt", ["f64", "f32"])
def test_fused_kmv_sq_sets(shape, rps, nsys, dt):
    """Packed square-lattice K.u with several systems per coefficient set (FP32 applies them two per pass over one
    staging of a tile's coefficients): even, odd and partly filled last sets, tiles cut by the box edge, and no
    write past the batch (one spare system after it keeps its fill)."""
    import ctypes
    rng = np.random.default_rng(sum(shape) + rps)
    lat = G.Lattice2D("square", *shape, 1.0)
    dl = core.DeviceLattice(lat)
    nset = -(-nsys // rps)
    Kn = np.array([rng.uniform(0.5, 1.5, (lat.N, lat.NN)) * lat.valid for _ in range(nset)])
    Tv = np.array([rng.uniform(-0.1, 0.1, (lat.N, lat.NN)) * lat.valid for _ in range(nset)])
    u = rng.standard_normal((nsys, lat.N, 2))
    tdt = torch.float64 if dt == "f64" else torch.float32
    Kp, Tp = core.pack(T(Kn), tdt), core.pack(T(Tv), tdt)
    uu = T(u, tdt).contiguous()
    out = torch.full((nsys + 1, lat.N, 2), 7.0, dtype=tdt, device=DEV)
    lib = L.load()
    prec = L.LPM_F64 if dt == "f64" else L.LPM_F32
    scr = torch.empty(max(1, lib.lpm_kmv_scratch_bytes(dl.ref, prec, nsys)), dtype=torch.uint8, device=DEV)
    name = "lpm_kmv_sq_f64" if dt == "f64" else "lpm_kmv_sq_f32"
    L.check(getattr(lib, name)(dl.ref, L.ptr(uu), L.ptr(Kp), L.ptr(Tp), L.LAYOUT_SOA,
                               ctypes.byref(core._batch(nsys, rps)), L.ptr(out), L.ptr(scr), scr.numel(),
                               L.stream_ptr(uu.device)), name)
    tol = 1e-13 if dt == "f64" else 3e-6
    for s in range(nsys):
        ref = O.sq_kmv(lat, u[s].ravel(), Kn[s // rps], Tv[s // rps])
        assert relmax(out[s].cpu().numpy().ravel(), ref) < tol, s
    assert torch.all(out[nsys] == 7.0)


@pytest.mark.parametrize("precond", [False, True])
def test_fused_cg_fp64_matches_oracle(gsc, sc12, precond):
    """FP64 CG on the fused path (packed coefficients): same iteration counts as the reference at 1e-8."""
    from lpm_b200 import _lib
    lat, dl, Kn, Tv = sc12
    Kp, Tp = core.pack(T(Kn)[None], torch.float64), core.pack(T(Tv)[None], torch.float64)
    M = core.block_jacobi(dl, T(Kn), T(Tv), torch.float64) if precond else None
    bs, frees, ups = [], [], []
    for ld in ("k_xx", "tb_sx"):
        fixed, up, _ = _bc(lat, ld, 2)
        free = ~fixed
        upm = np.where(fixed[:, None], up, 0.0)
        bs.append(-O.sc_apply(lat, upm, Kn, Tv) * free[:, None])
        frees.append(free)
        ups.append(upm)
    x, info = core.cg(dl, Kp, Tp, T(np.array(bs)), Minv=M, free=T(np.array(frees)), tol=1e-8, maxit=5000, check=1,
                      layout=_lib.LAYOUT_SOA, rhs_per_set=2)
    key = "pcg" if precond else "cg"
    for l, ld in enumerate(("k_xx", "tb_sx")):
        assert abs(int(info.iters[l]) - int(gsc["%s_it_%s" % (key, ld)])) <= 1
        assert relmax(x[l].cpu().numpy() + ups[l], gsc["%s_u_%s" % (key, ld)]) < 1e-6


def test_fused_pcg_fp32_batched_mixed_bcs():
    """FP32 PCG on the fused path, 2 specimens x 3 loads with different BC sets, vs the FP64 oracle solution."""
    from lpm_b200 import _lib
    lat = G.LatticeGeom(20, 18, 16)
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(9)
    ph = (rng.random((2, lat.N)) < 0.3)
    Kn, Tv = [], []
    for b in range(2):
        C = G.iso_C(np.where(ph[b], 10.0, 1.0), 0.2)
        k, t = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
        Kn.append(k)
        Tv.append(t)
    Kn, Tv = np.array(Kn), np.array(Tv)
    loads = ["k_xx", "tb_tz", "lr_tx"]
    frees, ups = [], []
    for ld in loads:
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk // 2, (10, 9, 8), 2)
        frees.append(~fixed)
        ups.append(np.where(fixed[:, None], up, 0.0))
    frees, ups = np.array(frees), np.array(ups)
    b = np.array([[-O.sc_apply(lat, ups[l], Kn[s], Tv[s]) * frees[l][:, None] for l in range(3)] for s in range(2)])
    Kp, Tp = core.pack(T(Kn), torch.float32), core.pack(T(Tv), torch.float32)
    M = core.block_jacobi(dl, T(Kn), T(Tv), torch.float32)
    x, info = core.cg(dl, Kp, Tp, T(b, torch.float32).reshape(6, lat.N, 3), Minv=M, free=T(np.tile(frees, (2, 1))), tol=1e-5,
                      maxit=5000, layout=_lib.LAYOUT_SOA, rhs_per_set=3)
    assert (info.status == 0).all()
    for s in range(2):
        for l, ld in enumerate(loads):
            ref, _ = O.solve_pcg(lat, Kn[s], Tv[s], ~frees[l], ups[l], tol=1e-12)
            assert rel_l2(x[3 * s + l].cpu().numpy() + ups[l], ref) < 1e-4
