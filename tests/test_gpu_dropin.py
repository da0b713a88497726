"""GPU parity of the drop-in modules (torch_lpm3d, torch_lpm, lin3d, lin2d) against the reference's own outputs.

The golden vectors come from the reference's torch modules run on the CPU (tests/golden/make_golden.py, part
"grad"): autograd vector-Jacobian products of apply / stress / energy, the differentiable coarse solve with a
weighted loss, the fine-reference block means, and the 2D coarse model's loss gradient.

Tolerances: VJPs and single-kernel outputs 1e-12 (max-abs relative to the reference array's max); solves to
rel. residual 1e-12 / 1e-13 agree with the reference's direct or PCG solves to 1e-8; loss gradients through the
adjoint solve 1e-7.
"""
import numpy as np
import pytest

from conftest import relmax
from lpm_b200 import geom as G

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda"


def T(a, grad=False):
    t = torch.as_tensor(np.asarray(a), device=DEV, dtype=torch.float64)
    return t.requires_grad_(True) if grad else t


def _vjp(fn, u, Kn, Tv, Gw):
    ut, Kt, Tt = T(u, True), T(Kn, True), T(Tv, True)
    e = (fn(ut, Kt, Tt) * T(Gw)).sum()
    return [g.cpu().numpy() for g in torch.autograd.grad(e, (ut, Kt, Tt))]


# ------------------------------------------------------------------------------------------ vector-Jacobian products
@pytest.mark.parametrize("name", ["st", "en", "ap"])
def test_vjp_sc(ggrad, name):
    """d/d(u, Kn, Tv) of sum(G * f(u; Kn, Tv)) for f = stress, energy, K u on a 5x4x3 box, two displacement fields
    sharing one parameter set (the parameter gradient sums over them)."""
    from lpm_b200.torch_lpm3d import SCT
    op = SCT(G.LatticeGeom(5, 4, 3, 1.0), DEV)
    fn = {"st": op.stress, "en": op.energy, "ap": op.apply}[name]
    du, dK, dT = _vjp(fn, ggrad["v3_u"], ggrad["v3_Kn"], ggrad["v3_Tv"], ggrad["v3%s_G" % name])
    assert relmax(du, ggrad["v3%s_du" % name]) < 1e-12
    assert relmax(dK, ggrad["v3%s_dK" % name]) < 1e-12
    assert relmax(dT, ggrad["v3%s_dT" % name]) < 1e-12


@pytest.mark.parametrize("name", ["st", "en"])
def test_vjp_sq(ggrad, name):
    """The same for the 2D coarse model's stress (xx yy xy) and energy density on a 7x5 square lattice."""
    from lpm_b200 import torch_lpm as T2
    m = T2.CoarseT(7, 5, 1, device=DEV)
    fn = {"st": m.op.stress, "en": lambda u, K, Tv: m.op.energy(u, K, Tv) / (m.s * m.h) ** 2}[name]
    u = ggrad["v2_u"].reshape(1, -1, 2)
    du, dK, dT = _vjp(fn, u, ggrad["v2_Kn"], ggrad["v2_Tv"], ggrad["v2%s_G" % name])
    assert relmax(du.reshape(1, -1), ggrad["v2%s_du" % name]) < 1e-12
    assert relmax(dK, ggrad["v2%s_dK" % name]) < 1e-12
    assert relmax(dT, ggrad["v2%s_dT" % name]) < 1e-12


def test_apply_grad_matches_autograd(ggrad):
    """K u parameter gradient (symmetric and non-symmetric parameters) through the autograd wrapper."""
    from lpm_b200.torch_lpm3d import SCT
    op = SCT(G.LatticeGeom(4, 4, 4, 2.0), DEV)
    for p in ("g3", "g3n"):
        _, dK, dT = _vjp(op.apply, ggrad["g3_u"], ggrad[p + "_Kn"], ggrad[p + "_Tv"], ggrad["g3_lam"])
        assert relmax(dK, ggrad[p + "_gK"]) < 1e-12
        assert relmax(dT, ggrad[p + "_gT"]) < 1e-12


# ----------------------------------------------------------------------------------- differentiable coarse solves
def test_coarse3d_linsolve_loss_gradient(ggrad):
    """CoarseT(4, 2).run over the 9 load cases with LinSolve, a weighted loss of u, stress, energy density and grip
    reaction, and its gradient w.r.t. Kn, Tv (forward PCG + adjoint PCG + per-bond gradient kernel)."""
    from lpm_b200 import torch_lpm3d as T3
    cm = T3.CoarseT(4, 2, device=DEV)
    kn, tv = T(ggrad["g3_Kn"][None], True), T(ggrad["g3_Tv"][None], True)
    o = cm.run(kn, tv, tol=1e-13)
    L = (o["sig"] * T(ggrad["c3_Wsig"])).sum() + 1e3 * (o["u"] * T(ggrad["c3_Wu"])).sum() + o["F"].sum() \
        + o["w"].sum()
    L.backward()
    assert relmax(o["u"].detach().cpu().numpy()[0], ggrad["c3_u"]) < 1e-9
    assert relmax(o["sig"].detach().cpu().numpy()[0], ggrad["c3_sig"]) < 1e-9
    assert relmax(o["w"].detach().cpu().numpy()[0], ggrad["c3_w"]) < 1e-9
    assert relmax(o["F"].detach().cpu().numpy()[0], ggrad["c3_F"]) < 1e-9
    assert abs(float(L.detach()) - float(ggrad["c3_loss"])) < 1e-9 * abs(float(ggrad["c3_loss"]))
    assert relmax(kn.grad.cpu().numpy()[0], ggrad["c3_gK"]) < 1e-7
    assert relmax(tv.grad.cpu().numpy()[0], ggrad["c3_gT"]) < 1e-7


def test_fine_reference_block_means(ggrad):
    """FineRefT(6, 2).run: block means of u, stress, energy density and the grip reactions, FP64 PCG to 1e-12, and
    the mixed-precision variant (FP32 PCG inside FP64 refinement) to the same FP64 tolerance."""
    from lpm_b200 import torch_lpm3d as T3
    K, Tv = T(ggrad["f3_Kn"][None]), T(ggrad["f3_Tv"][None])
    for prec, tol in (("fp64", 1e-8), ("mixed", 1e-7)):
        fr = T3.FineRefT(6, 2, device=DEV, precision=prec)
        r = fr.run(K, Tv, tol=1e-12)
        for k in ("u", "sig", "w", "F"):
            assert relmax(r[k].cpu().numpy()[0], ggrad["f3_" + k]) < tol, (prec, k)


def test_coarse2d_losses_gradient(ggrad):
    """2D CoarseT(8, 8, 2).run over the 6 load cases, the reference's losses against a stiffer reference model, and
    the gradient w.r.t. a log-parameterisation theta of the symmetric bond stiffnesses."""
    from lpm_b200 import torch_lpm as T2
    m = T2.CoarseT(8, 8, 2, device=DEV)
    lat = m.lat
    K0, T0 = ggrad["c2_K0"], ggrad["c2_T0"]
    with torch.no_grad():
        ref = m.run(T(K0) * 1.1, T(T0))
    for ld in T2.LOADS:
        assert relmax(ref[ld]["u"].cpu().numpy(), ggrad["c2_refu_%s" % ld]) < 1e-8
    q = torch.as_tensor(np.where(lat.valid, lat.nbr, 0), device=DEV)
    opp = torch.as_tensor(np.repeat(lat.opp[None, :], lat.N, 0), device=DEV)
    th = T(ggrad["c2_th"], True)
    Kn = T(K0) * torch.exp(0.5 * (th + th[:, q, opp]))
    out = m.run(Kn, T(T0))
    a, b, c = T2.losses(m, out, ref)
    loss = (a + b + c).sum()
    loss.backward()
    for ld in T2.LOADS:
        assert relmax(out[ld]["u"].detach().cpu().numpy(), ggrad["c2_u_%s" % ld]) < 1e-8
        assert relmax(out[ld]["sig"].detach().cpu().numpy(), ggrad["c2_sig_%s" % ld]) < 1e-8
        assert relmax(out[ld]["w"].detach().cpu().numpy(), ggrad["c2_w_%s" % ld]) < 1e-8
        if "c2_F_%s" % ld in ggrad:
            assert relmax(out[ld]["F"].detach().cpu().numpy(), ggrad["c2_F_%s" % ld]) < 1e-8
    assert abs(float(loss.detach()) - float(ggrad["c2_loss"])) < 1e-6 * abs(float(ggrad["c2_loss"]))
    assert relmax(th.grad.cpu().numpy(), ggrad["c2_gth"]) < 1e-6


def test_coarse2d_gradient_fd():
    """Central finite differences of the 2D loss along a random direction of theta agree with the adjoint gradient."""
    from lpm_b200 import torch_lpm as T2
    m = T2.CoarseT(6, 6, 2, device=DEV)
    lat = m.lat
    rng = np.random.default_rng(5)
    K0 = np.where(lat.shell[None, None, :] == 0, 0.38, 0.19) * (1 + 0.2 * rng.random((1, lat.N, 8)))
    q = np.where(lat.valid, lat.nbr, 0)
    opp = np.repeat(lat.opp[None, :], lat.N, 0)
    K0 = 0.5 * (K0 + K0[:, q, opp]) * lat.valid
    T0 = np.full((1, lat.N, 8), 0.03) * lat.valid
    with torch.no_grad():
        ref = m.run(T(K0) * 1.2, T(T0))
    qt, ot = torch.as_tensor(q, device=DEV), torch.as_tensor(opp, device=DEV)

    def loss(th):
        out = m.run(T(K0) * torch.exp(0.5 * (th + th[:, qt, ot])), T(T0))
        return sum(t.sum() for t in T2.losses(m, out, ref))

    th = T(0.1 * rng.standard_normal((1, lat.N, 8)), True)
    loss(th).backward()
    d = T(rng.standard_normal((1, lat.N, 8)))
    eps = 1e-5
    with torch.no_grad():
        fd = (float(loss(th + eps * d)) - float(loss(th - eps * d))) / (2 * eps)
    ad = float((th.grad * d).sum())
    assert abs(fd - ad) < 1e-5 * abs(ad)


def test_stability_penalty():
    """group_hessians / stability_penalty: an isotropic parameter set is stable (zero penalty); a strongly negative
    Tv makes every group's smallest eigenvalue negative and the penalty positive."""
    from lpm_b200 import torch_lpm as T2
    m = T2.CoarseT(5, 4, 1, device=DEV)
    Kn = T(np.where(m.lat.shell[None, None, :] == 0, 0.4, 0.2) * m.lat.valid)
    pen, lam = m.stability_penalty(Kn, T(np.full((1, m.N, 8), 0.01) * m.lat.valid))
    assert float(pen) == 0.0 and float(lam.min()) > 0
    pen, lam = m.stability_penalty(Kn, T(np.full((1, m.N, 8), -0.3) * m.lat.valid))
    assert float(pen) > 0 and float(lam.max()) < 0


# ------------------------------------------------------------------------------------------- NumPy-facing mirrors
def _bc(lat, ld, s):
    nc = lat.nx // s
    return G.prescribed(ld, lat.x, lat.ijk // s, (nc,) * 3, s)


def test_lin3d_solvers(gsc):
    """lin3d.solve_pcg / solve_cg on the 12^3 golden lattice: the reference's iteration counts and solutions; the
    mixed-precision solver reaches the same solution."""
    from lpm_b200 import lin3d
    lat = lin3d.Lattice3D(12, 12, 12)
    Kn, Tv = gsc["Kn"], gsc["Tv"]
    assert relmax(lat.apply(gsc["u"], Kn, Tv), gsc["Ku"]) < 1e-13
    assert relmax(lat.stress(gsc["u"], Kn, Tv), gsc["st"]) < 1e-13
    assert relmax(lat.energy_per_particle(gsc["u"], Kn, Tv), gsc["U"]) < 1e-13
    assert relmax(lat.block_diag(Kn, Tv), gsc["D"]) < 1e-13
    for ld in ("k_xx", "tb_sx"):
        fixed, up, _ = _bc(lat, ld, 2)
        u, info = lin3d.solve_pcg(lat, Kn, Tv, fixed, up, tol=1e-8)
        assert abs(info["iters"] - int(gsc["pcg_it_%s" % ld])) <= 1
        assert relmax(u, gsc["pcg_u_%s" % ld]) < 1e-6
        u, info = lin3d.solve_cg(lat, Kn, Tv, fixed, up, tol=1e-8, maxit=5000)
        assert abs(info["iters"] - int(gsc["cg_it_%s" % ld])) <= 1
        assert relmax(u, gsc["cg_u_%s" % ld]) < 1e-6
        um, info = lin3d.solve_mixed(lat, Kn, Tv, fixed, up, tol=1e-10)
        assert info["status"] == 0 and relmax(um, gsc["pcg_u_%s" % ld]) < 1e-6


def test_lin2d_solvers(gsq):
    """lin2d.solve_mf: cg2plain semantics (per-DOF mask, initial test) and the block-Jacobi PCG of solver2d."""
    from lpm_b200 import lin2d
    lat = lin2d.Lattice2D("square", 16, 12, 1.0)
    Kn, Tv = gsq["Kn"], gsq["Tv"]
    assert relmax(lat.stress(gsq["u"], Kn, Tv), gsq["stress"]) < 1e-13
    assert relmax(lat.energy_per_particle(gsq["u"], Kn, Tv), gsq["energy"]) < 1e-13
    fd, up = gsq["cg_fixed"], gsq["cg_up"]
    dofs = np.flatnonzero(fd.ravel())
    u, info = lin2d.solve_mf(lat, Kn, Tv, dofs, up.ravel()[dofs], tol=1e-10)
    assert abs(info["iters"] - int(gsq["cg_it"])) <= 1 and relmax(u, gsq["cg_u"]) < 1e-8
    pf, pu = gsq["pcg_fixed"], gsq["pcg_up"]
    dofs = np.flatnonzero(np.repeat(pf, 2))
    u, info = lin2d.solve_mf(lat, Kn, Tv, dofs, pu.ravel()[dofs], tol=1e-10, precond=True)
    assert abs(info["iters"] - int(gsq["pcg_it"])) <= 1 and relmax(u, gsq["pcg_u"]) < 1e-8
    um, info = lin2d.solve_mixed(lat, Kn, Tv, dofs, pu.ravel()[dofs], tol=1e-10, precond=True)
    assert info["status"] == 0 and relmax(um, gsq["pcg_u"]) < 1e-6
