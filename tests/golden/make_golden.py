"""Generates the golden fixtures of tests/golden/ by running the reference itself (FP64, CPU).

Run where the reference checkout is available, with LPM_REFERENCE set to its root directory:

    LPM_REFERENCE=<reference checkout> python tests/golden/make_golden.py          # all parts, fresh interpreters
    LPM_REFERENCE=<reference checkout> python tests/golden/make_golden.py cfg3     # one part

The reference is imported read-only: Numba's cache goes to a temporary directory, and the two modules that create
folders inside the reference tree at import time (timing/t2d/a2common.py, timing/t3d/common.py) are replaced by stubs.
Parts:
  sc     3D simple-cubic: the arrays of coarse3d/dev/export_check.py (n = 12, seed 5), SuperLU block means for
         s = 2, 3 and the 9 loads, PCG / plain-CG iteration counts, masked-lattice connectivity, BCs, generators
  sq     2D square: timing/t2d/solver2d.py kernels, cg2plain / pcg_mf solves, SuperLU, masked connectivity, BCs
  grad   gradients: torch_lpm3d autograd of lam . K u, LinSolve through CoarseT.run (as coarse3d/check_torch3d.py),
         torch_lpm dense-assembly gradient of lam^T K u and of the CoarseT.run losses (as coarse2d/check_gradient.py)
  amg    aggregation AMG of timing/t3d/amg3d.py with the settings of timing/t3d/problems.py (geometry, levels, rho,
         one cycle, PCG iterations; 14^3 and the 48^3 bench specimen) and geom3d.interface_cells
  sctv   the per-specimen void operator of cement3d/torch_v1.py (SCTV, CoarseTV): apply, stress, energy and block
         diagonals under two specimens' solid masks, and a differentiable CoarseTV.run (9 loads) with its loss gradient
  asm    parameter assembly upstream of the 3D solve (coarse3d/train3d.py): the symmetric Scatter of per-group bond
         values to (B, N, 18) and the group_penalty stability term, with their autograd gradients
  cfg3   the differentiable 2D coarse solve of the benchmark's third configuration at nc = 32 and 48 (the sizes the
         reference's dense torch_lpm path handles): GRF fine field -> Voigt cells -> two-end-mean bonds (coarse2d/
         micro.py, coarse2d/cg.py:201-234), lognormal(0.2) factors per undirected bond rounded to FP32, loads lr_tx,
         tb_ty, tb_sx, loss = sum over loads of the MSE of u against a seeded target, and its gradient w.r.t. the log
         bond stiffness theta from torch_lpm.CoarseT.run (dense assembly + Cholesky, torch autograd)
"""
import os
import subprocess
import sys
import tempfile
import types

REF = os.environ.get("LPM_REFERENCE", "")
HERE = os.path.dirname(os.path.abspath(__file__))


def _env():
    os.environ["NUMBA_CACHE_DIR"] = os.path.join(tempfile.gettempdir(), "lpm_golden_numba")
    os.environ.setdefault("NUMBA_NUM_THREADS", "8")
    sys.dont_write_bytecode = True


def _stub(name):
    sys.modules[name] = types.ModuleType(name)


def part_sc():
    _env()
    sys.path.insert(0, os.path.join(REF, "coarse3d"))
    import numpy as np
    import geom3d as G
    import lin3d as L3
    import micro3d
    sys.path.insert(0, os.path.join(REF, "timing", "t3d"))
    _stub("common")
    from cgplain import cg3

    out = {}
    # ---- export_check.py arrays (n = 12, rng(5)) ----
    n = 12
    rng = np.random.default_rng(5)
    ph, E, nu, info = micro3d.sample(n, rng)
    lat = L3.Lattice3D(n, n, n, 1.0)
    C = G.iso_C(E, nu)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    u = rng.standard_normal((lat.N, 3))
    out.update(phase=ph.astype(np.int8), E=E, nu=nu, Kn=Kn, Tv=Tv, u=u, Ku=lat.apply(u, Kn, Tv),
               st=lat.stress(u, Kn, Tv), U=lat.energy_per_particle(u, Kn, Tv), D=lat.block_diag(Kn, Tv),
               nbr=lat.nbr.astype(np.int32))
    dL, F = lat.bond_forces(u, Kn, Tv)
    out.update(F_row=F[::97], dL_row=dL[::97])
    K = lat.stiffness(Kn, Tv)
    for s in (2, 3):
        nc = n // s
        IJK = lat.ijk // s
        cid = G.block_index(lat.ijk, s, (nc,) * 3)
        for ld in G.LOADS:
            fixed, up, mov = G.prescribed(ld, lat.x, IJK, (nc,) * 3, s)
            uu, _ = L3.solve_direct(K, fixed, up)
            st = lat.stress(uu, Kn, Tv)
            out["u_%d_%s" % (s, ld)] = np.stack([np.bincount(cid, uu[:, k]) for k in range(3)], 1) / s ** 3
            out["s_%d_%s" % (s, ld)] = np.stack([np.bincount(cid, st[:, k]) for k in range(6)], 1) / s ** 3
            out["w_%d_%s" % (s, ld)] = np.bincount(cid, lat.energy_per_particle(uu, Kn, Tv)) / s ** 3
            P = lat.apply(uu, Kn, Tv)
            out["F_%d_%s" % (s, ld)] = P[mov, G.GDIR[ld]].sum() if mov is not None else 0.0
            if (s, ld) in ((2, "k_xx"), (3, "tb_tz"), (2, "lr_tx")):
                out["ufull_%d_%s" % (s, ld)] = uu
    # ---- iterative solvers on (s = 2, k_xx) and (s = 2, tb_sx) ----
    for ld in ("k_xx", "tb_sx"):
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk // 2, (6,) * 3, 2)
        u_p, info_p = L3.solve_pcg(lat, Kn, Tv, fixed, up, tol=1e-8)
        out["pcg_u_%s" % ld] = u_p
        out["pcg_it_%s" % ld] = info_p["iters"]
        out["pcg_rel_%s" % ld] = info_p["relres"]
        free = ~fixed
        upm = np.zeros((lat.N, 3))
        upm[fixed] = up[fixed]
        b = -L3.k_apply(upm, lat.nbr, lat.ndir, Kn, Tv)
        b[fixed] = 0.0
        x = np.zeros((lat.N, 3))
        it, rr = cg3(lat.nbr, lat.ndir, Kn, Tv, free, b, x, 1e-8, 200000)
        out["cg_u_%s" % ld] = upm + x
        out["cg_it_%s" % ld] = int(it)
        out["cg_rel_%s" % ld] = float(rr)
    # ---- masked lattice connectivity ----
    mrng = np.random.default_rng(11)
    act = mrng.random(7 * 5 * 4) < 0.7
    lm = G.LatticeGeom(7, 5, 4, 1.5, origin=(0.1, -0.2, 0.3), active=act)
    out.update(m_active=act, m_nbr=lm.nbr.astype(np.int32), m_ijk=lm.ijk.astype(np.int32), m_x=lm.x,
               m_site_of=lm.site_of.astype(np.int32), m_nb_initial=lm.nb_initial.astype(np.int32))
    # ---- BCs on a 6^3 lattice, s = 2 ----
    lb = G.LatticeGeom(6, 6, 6, 1.0)
    for ld in G.LOADS:
        fixed, up, mov = G.prescribed(ld, lb.x, lb.ijk // 2, (3, 3, 3), 2)
        out["bc_fixed_%s" % ld] = fixed
        out["bc_up_%s" % ld] = up
        out["bc_mov_%s" % ld] = np.zeros(lb.N, bool) if mov is None else mov
    # ---- material maps ----
    cpr = np.random.default_rng(3)
    C66 = cpr.standard_normal((5, 6, 6))
    out["cp_C66"] = C66
    out["cp_params"] = G.cell_params_from_C66(C66, 0.7)
    # ---- generators ----
    out["gen_spheres"] = micro3d.spheres(16, 16, 16, 0.25, 4.0, np.random.default_rng(7), rjit=0.0)[0].astype(np.int8)
    out["gen_ellip"] = micro3d.ellipsoids(16, 16, 16, 0.3, 3.0, np.random.default_rng(8), aspect=(3.0, 3.0),
                                          rjit=0.0)[0].astype(np.int8)
    out["gen_grf3"] = micro3d.grf(12, 12, 12, 2.0, 0.3, np.random.default_rng(9))[0].astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "golden_sc.npz"), **out)
    print("golden_sc.npz:", len(out), "arrays")


def part_sq():
    _env()
    sys.path.insert(0, os.path.join(REF, "timing", "t2d"))
    _stub("a2common")
    import numpy as np
    import lin2d
    import micro
    import solver2d as S2
    from cg2plain import cg_mf

    out = {}
    nx, ny = 16, 12
    lat = lin2d.Lattice2D("square", nx, ny, 1.0)
    ph = micro.grf_two_phase(nx, ny, 3.0, 0.3, 4)
    E = np.where(ph == 1, 10.0, 1.0)
    Cpix = lin2d.iso_C(E, 0.25, plane="stress")
    Kn, Tv = lin2d.bond_params_two_end_mean(lat, lin2d.square_params_from_C(Cpix))
    rng = np.random.default_rng(21)
    # non-symmetric per-slot parameters: the g-form kernel is the exact Hessian for any values
    Kn_ns = Kn * (1 + 0.2 * rng.random(Kn.shape)) * lat.valid
    Tv_ns = Tv * (1 + 0.2 * rng.random(Tv.shape)) * lat.valid
    u = rng.standard_normal(2 * lat.N)
    arr = (np.where(lat.valid, lat.nbr, 0).astype(np.int64), lat.valid, np.ascontiguousarray(lat.ndir),
           lat.shell.astype(np.int64), lat.opp.astype(np.int64))
    g = np.empty((lat.N, 8))
    f = np.empty(2 * lat.N)
    S2._kmv(u, *arr, Kn_ns, Tv_ns, g, f)
    K, _, _ = lat.stiffness(Kn_ns, Tv_ns)
    out.update(phase=ph.astype(np.int8), Kn=Kn, Tv=Tv, Kn_ns=Kn_ns, Tv_ns=Tv_ns, u=u, f_ns=f, Ku_csr_ns=K @ u,
               nbr=lat.nbr.astype(np.int32))
    fixed_p = np.zeros(lat.N, bool)
    fixed_p[lat.ij[:, 0] == 0] = True
    Binv = np.empty((lat.N, 2, 2))
    S2._diag_inv(*arr, Kn, Tv, fixed_p, Binv)
    out.update(diag_fixed=fixed_p, Binv=Binv)
    out["stress"] = S2.stress(lat, u, Kn, Tv)
    out["energy"] = lat.energy_per_particle(u, Kn, Tv)
    # ---- per-DOF uniaxial tension, plain CG (cg2plain) and pcg_mf, SuperLU ----
    fd = np.zeros((lat.N, 2), bool)
    up = np.zeros((lat.N, 2))
    left, right = lat.ij[:, 0] == 0, lat.ij[:, 0] == nx - 1
    fd[left, 0] = fd[right, 0] = True
    fd[left & (lat.ij[:, 1] == 0), 1] = True
    up[right, 0] = 1e-3 * (nx - 1)
    mask = (~fd).astype(np.float64).ravel()
    ub = up.ravel()
    fk = np.empty(2 * lat.N)
    S2._kmv(ub, *arr, Kn, Tv, g, fk)
    b = -fk * mask
    x = np.zeros(2 * lat.N)
    it = cg_mf(*arr, Kn, Tv, mask, b, x, 1e-10, 200000, g)
    out.update(cg_fixed=fd, cg_up=up, cg_u=x + ub, cg_it=int(it))
    Ks, _, _ = lat.stiffness(Kn, Tv)
    fdofs = np.nonzero(fd.ravel())[0]
    usol, _ = lin2d.solve_disp(Ks, fdofs, ub[fdofs])
    out["lu_u"] = usol
    # pcg_mf on a particle-fixed problem (left column clamped, right column pulled)
    fixed = left | right
    mask_p = np.repeat((~fixed).astype(np.float64), 2)
    ub2 = np.zeros((lat.N, 2))
    ub2[right, 0] = 1e-3 * (nx - 1)
    ub2 = ub2.ravel()
    S2._kmv(ub2, *arr, Kn, Tv, g, fk)
    b2 = -fk * mask_p
    B2 = np.empty((lat.N, 2, 2))
    S2._diag_inv(*arr, Kn, Tv, fixed, B2)
    x2 = np.zeros(2 * lat.N)
    snaps = np.empty((1, 2 * lat.N))
    iters = np.zeros(1, np.int64)
    S2.pcg_mf(*arr, Kn, Tv, B2, mask_p, b2, x2, np.array([1e-10]), 20000, snaps, iters, g)
    out.update(pcg_fixed=fixed, pcg_up=ub2.reshape(-1, 2), pcg_u=snaps[0] + ub2, pcg_it=int(iters[0]))
    # ---- masked connectivity ----
    mrng = np.random.default_rng(12)
    act = mrng.random(9 * 7) < 0.65
    lm = lin2d.Lattice2D("square", 9, 7, 0.5, origin=(0.3, 0.1), active=act)
    out.update(m_active=act, m_nbr=lm.nbr.astype(np.int32), m_ij=lm.ij.astype(np.int32), m_x=lm.x)
    # ---- BCs (el_prob / torch_lpm convention, L = 1 and 2) ----
    import el_prob as EP
    lb = lin2d.Lattice2D("square", 8, 8, 1.0)
    for L in (1, 2):
        for ld in EP.LOADS:
            fixed, upb, mov = EP.prescribed(ld, lb.x, lb.ij // 2, 4, 4, 2, 1.0, L)
            out["bc_fixed_%d_%s" % (L, ld)] = fixed
            out["bc_up_%d_%s" % (L, ld)] = upb
    # ---- generators ----
    out["gen_grf"] = micro.grf_two_phase(40, 32, 6.0, 0.30, 3).astype(np.int8)
    np.savez_compressed(os.path.join(HERE, "golden_sq.npz"), **out)
    print("golden_sq.npz:", len(out), "arrays")


def part_grad():
    _env()
    sys.path.insert(0, os.path.join(REF, "coarse3d"))
    import numpy as np
    import torch
    import geom3d as G
    import torch_lpm3d as T3
    torch.set_default_dtype(torch.float64)
    out = {}
    # ---- 3D: autograd of lam . apply(u; Kn, Tv) on a coarse 4^3 lattice with symmetric random bonds ----
    nc, s = 4, 2
    lat = G.LatticeGeom(nc, nc, nc, s)
    rng = np.random.default_rng(1)
    Kn0 = np.zeros((lat.N, 18))
    Tv0 = np.zeros((lat.N, 18))
    for i in range(lat.N):
        for k in range(0, 18, 2):
            q = lat.nbr[i, k]
            if q >= 0:
                Kn0[i, k] = Kn0[q, k ^ 1] = rng.uniform(0.8, 1.2)
                Tv0[i, k] = Tv0[q, k ^ 1] = rng.uniform(-0.03, 0.03)
    op = T3.SCT(lat, "cpu")
    u = rng.standard_normal((lat.N, 3))
    lam = rng.standard_normal((lat.N, 3))
    Kt = torch.tensor(Kn0, requires_grad=True)
    Tt = torch.tensor(Tv0, requires_grad=True)
    e = (torch.tensor(lam) * op.apply(torch.tensor(u), Kt, Tt)).sum()
    gK, gT = torch.autograd.grad(e, (Kt, Tt))
    out.update(g3_Kn=Kn0, g3_Tv=Tv0, g3_u=u, g3_lam=lam, g3_gK=gK.numpy(), g3_gT=gT.numpy())
    # non-symmetric parameters too (the closed form does not assume symmetry)
    Kns = Kn0 * (1 + 0.3 * rng.random(Kn0.shape))
    Tvs = Tv0 + 0.01 * rng.standard_normal(Tv0.shape) * lat.valid
    Kt = torch.tensor(Kns, requires_grad=True)
    Tt = torch.tensor(Tvs, requires_grad=True)
    e = (torch.tensor(lam) * op.apply(torch.tensor(u), Kt, Tt)).sum()
    gK, gT = torch.autograd.grad(e, (Kt, Tt))
    out.update(g3n_Kn=Kns, g3n_Tv=Tvs, g3n_gK=gK.numpy(), g3n_gT=gT.numpy())
    # ---- 3D: autograd of stress / energy / apply (vector-Jacobian products) on a masked-free 5x4x3 box ----
    latv = G.LatticeGeom(5, 4, 3, 1.0)
    opv = T3.SCT(latv, "cpu")
    rv = np.random.default_rng(13)
    Knv = rv.uniform(0.5, 1.5, (latv.N, 18)) * latv.valid
    Tvv = rv.uniform(-0.1, 0.1, (latv.N, 18)) * latv.valid
    uv = rv.standard_normal((2, latv.N, 3))
    Gs = rv.standard_normal((2, latv.N, 6))
    Ge = rv.standard_normal((2, latv.N))
    Gf = rv.standard_normal((2, latv.N, 3))
    for name, fn, Gw in (("st", opv.stress, Gs), ("en", opv.energy, Ge), ("ap", opv.apply, Gf)):
        ut = torch.tensor(uv, requires_grad=True)
        Kt = torch.tensor(Knv, requires_grad=True)
        Tt = torch.tensor(Tvv, requires_grad=True)
        e = (fn(ut, Kt, Tt) * torch.tensor(Gw)).sum()
        du, dK, dT = torch.autograd.grad(e, (ut, Kt, Tt))
        out.update({"v3%s_du" % name: du.numpy(), "v3%s_dK" % name: dK.numpy(), "v3%s_dT" % name: dT.numpy(),
                    "v3%s_G" % name: Gw})
    out.update(v3_Kn=Knv, v3_Tv=Tvv, v3_u=uv)
    # ---- 3D: full differentiable coarse solve (LinSolve through CoarseT.run), 9 loads, tol 1e-13 ----
    cm = T3.CoarseT(nc, s, device="cpu")
    torch.manual_seed(0)
    Wsig = torch.randn(1, len(G.LOADS), lat.N, 6)
    Wu = torch.randn(1, len(G.LOADS), lat.N, 3)
    kn = torch.tensor(Kn0)[None].requires_grad_(True)
    tv = torch.tensor(Tv0)[None].requires_grad_(True)
    o = cm.run(kn, tv, tol=1e-13)
    L = (o["sig"] * Wsig).sum() + 1e3 * (o["u"] * Wu).sum() + o["F"].sum() + o["w"].sum()
    L.backward()
    out.update(c3_Wsig=Wsig.numpy(), c3_Wu=Wu.numpy(), c3_loss=float(L), c3_gK=kn.grad.numpy()[0],
               c3_gT=tv.grad.numpy()[0], c3_u=o["u"].detach().numpy()[0], c3_sig=o["sig"].detach().numpy()[0],
               c3_w=o["w"].detach().numpy()[0], c3_F=o["F"].detach().numpy()[0])
    # fine reference on the n = 6 box (s = 2), PCG tol 1e-12
    fr = T3.FineRefT(6, 2, device="cpu")
    rf = np.random.default_rng(2)
    Knf = np.zeros((fr.lat.N, 18))
    Tvf = np.zeros((fr.lat.N, 18))
    for i in range(fr.lat.N):
        for k in range(0, 18, 2):
            q = fr.lat.nbr[i, k]
            if q >= 0:
                Knf[i, k] = Knf[q, k ^ 1] = rf.uniform(0.5, 1.5)
                Tvf[i, k] = Tvf[q, k ^ 1] = rf.uniform(-0.05, 0.05)
    r = fr.run(torch.tensor(Knf)[None], torch.tensor(Tvf)[None], tol=1e-12)
    out.update(f3_Kn=Knf, f3_Tv=Tvf, f3_u=r["u"].numpy()[0], f3_sig=r["sig"].numpy()[0], f3_w=r["w"].numpy()[0],
               f3_F=r["F"].numpy()[0])

    # ---- 2D: torch_lpm dense assembly ----
    sys.path.insert(0, os.path.join(REF, "coarse2d"))
    import torch_lpm as T2
    m = T2.CoarseT(6, 5, 2, device="cpu")
    lat2 = m.lat
    N = lat2.N
    r2 = np.random.default_rng(0)
    Kn2 = np.where(lat2.shell[None, :] == 0, 0.38, 0.19) * (1 + 0.3 * r2.random((N, 8)))
    Kn2 = Kn2 * lat2.valid
    Tv2 = (0.03 + 0.01 * r2.standard_normal((N, 8))) * lat2.valid
    u2 = r2.standard_normal(2 * N)
    l2 = r2.standard_normal(2 * N)
    Kt = torch.tensor(Kn2, requires_grad=True)
    Tt = torch.tensor(Tv2, requires_grad=True)
    Kd = m.assemble(Kt[None], Tt[None])[0]
    e = torch.tensor(l2) @ (Kd @ torch.tensor(u2))
    gK, gT = torch.autograd.grad(e, (Kt, Tt))
    out.update(g2_Kn=Kn2, g2_Tv=Tv2, g2_u=u2, g2_lam=l2, g2_gK=gK.numpy(), g2_gT=gT.numpy(),
               g2_Ku=(Kd @ torch.tensor(u2)).detach().numpy())
    # stress / energy-density VJPs of the 2D model (bond_forces-based, torch_lpm.py:231-258)
    m7 = T2.CoarseT(7, 5, 1, device="cpu")
    l7 = m7.lat
    r7 = np.random.default_rng(17)
    K7 = r7.uniform(0.3, 0.6, (1, l7.N, 8)) * l7.valid
    T7 = r7.uniform(-0.05, 0.05, (1, l7.N, 8)) * l7.valid
    u7 = r7.standard_normal((1, 2 * l7.N))
    Gs7 = r7.standard_normal((1, l7.N, 3))
    Ge7 = r7.standard_normal((1, l7.N))
    for name, fn, Gw in (("st", m7.stress, Gs7), ("en", m7.energy_density, Ge7)):
        ut = torch.tensor(u7, requires_grad=True)
        Kt = torch.tensor(K7, requires_grad=True)
        Tt = torch.tensor(T7, requires_grad=True)
        e = (fn(ut, Kt, Tt) * torch.tensor(Gw)).sum()
        du, dK, dT = torch.autograd.grad(e, (ut, Kt, Tt))
        out.update({"v2%s_du" % name: du.numpy(), "v2%s_dK" % name: dK.numpy(), "v2%s_dT" % name: dT.numpy(),
                    "v2%s_G" % name: Gw})
    out.update(v2_Kn=K7, v2_Tv=T7, v2_u=u7)
    # full CoarseT.run + losses gradient (check_gradient.py style; nc = 8, s = 2, B = 2)
    m8 = T2.CoarseT(8, 8, 2, device="cpu")
    lat8 = m8.lat
    N8 = lat8.N
    r8 = np.random.default_rng(0)
    B = 2
    K0 = np.where(lat8.shell[None, None, :] == 0, 0.38, 0.19) * (1 + 0.3 * r8.random((B, N8, 8)))
    q = np.where(lat8.valid, lat8.nbr, 0)
    opp = lat8.opp[None, :].repeat(N8, 0)
    K0 = 0.5 * (K0 + K0[:, q, opp]) * lat8.valid
    T0 = np.full((B, N8, 8), 0.03) * lat8.valid
    ref = m8.run(torch.tensor(K0) * 1.1, torch.tensor(T0))
    ref = {k: {kk: (vv.detach() if vv is not None else None) for kk, vv in v.items()} for k, v in ref.items()}
    th = torch.tensor(0.1 * r8.standard_normal((B, N8, 8)), requires_grad=True)
    qt = torch.as_tensor(q)
    ot = torch.as_tensor(opp)
    Kn8 = torch.tensor(K0) * torch.exp(0.5 * (th + th[:, qt, ot]))
    Tv8 = torch.tensor(T0)
    o8 = m8.run(Kn8, Tv8)
    a, b_, c = T2.losses(m8, o8, ref)
    Lg = (a + b_ + c).sum()
    Lg.backward()
    out.update(c2_K0=K0, c2_T0=T0, c2_th=th.detach().numpy(), c2_loss=float(Lg), c2_gth=th.grad.numpy())
    for ld in T2.LOADS:
        out["c2_u_%s" % ld] = o8[ld]["u"].detach().numpy()
        out["c2_sig_%s" % ld] = o8[ld]["sig"].detach().numpy()
        out["c2_w_%s" % ld] = o8[ld]["w"].detach().numpy()
        if o8[ld]["F"] is not None:
            out["c2_F_%s" % ld] = o8[ld]["F"].detach().numpy()
        out["c2_refu_%s" % ld] = ref[ld]["u"].numpy()
    np.savez_compressed(os.path.join(HERE, "golden_grad.npz"), **out)
    print("golden_grad.npz:", len(out), "arrays")


def part_amg():
    """Aggregation AMG of timing/t3d/amg3d.py with the settings of timing/t3d/problems.py:19 (AMG_CFG) on a 14^3
    spheres specimen, one hierarchy per BC set (ring, tb, lr) as problems.solve_amg; coarse_max = 100 so that the
    hierarchy has a W-cycled level 1 above a dense level 2.  Plus the iteration count of the 48^3 spheres workload."""
    _env()
    sys.path.insert(0, os.path.join(REF, "coarse3d"))
    sys.path.insert(0, os.path.join(REF, "timing", "t3d"))
    _stub("common")
    import numpy as np
    import geom3d as G
    import lin3d as L3
    import micro3d
    import amg3d as A3

    out = {}

    def specimen(n, seed, r):
        ph, _ = micro3d.spheres(n, n, n, 0.25, r, np.random.default_rng(seed), rjit=0.0)
        lat = L3.Lattice3D(n, n, n, 1.0)
        C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
        Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
        return lat, Kn, Tv

    n = 14
    lat, Kn, Tv = specimen(n, 3, 2.5)
    out.update(a_n=n, a_Kn=Kn, a_Tv=Tv)
    D = lat.block_diag(Kn, Tv)
    rho0 = None
    brng = np.random.default_rng(21)
    for name, ld in (("ring", "k_xx"), ("tb", "tb_tz"), ("lr", "lr_tx")):
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        geo = A3.AMGGeom(lat, ~fixed, agg=3, coarse_max=100)
        M = L3.k_block_jacobi(D, ~fixed)
        h = A3.AMG3D(geo, Kn, Tv, nu=1, gamma=2, power_its=5, Minv0=M, rho0=rho0)
        rho0 = h.rho0
        pre = "a_%s_" % name
        out[pre + "g"] = np.array([geo.l0["g"]] + [L["gc"] for L in geo.levels], np.int64)
        out[pre + "P"] = geo.l0["P"]
        out[pre + "agg_of"] = geo.l0["agg_of"]
        out[pre + "Q1"] = geo.levels[0]["Q"]
        out[pre + "rho"] = np.array([h.rho0] + list(h.rho))
        out[pre + "A1"] = h.A[0].astype(np.float32)
        out[pre + "A2"] = h.A[1]
        r = brng.standard_normal((lat.N, 3))
        A3._mask(r, ~fixed)
        out[pre + "vin"] = r
        out[pre + "vout"] = h.vcycle(r.copy())
        b = -L3.k_apply(up, lat.nbr, lat.ndir, Kn, Tv)
        A3._mask(b, ~fixed)
        x, it, rel = h.pcg(b, 1e-8)
        out[pre + "pcg_x"] = up + x
        out[pre + "pcg_it"] = it
        out[pre + "pcg_rel"] = rel
    # 48^3 spheres (r = 4, seed 0, the bench specimen), ring BCs, load k_xx
    n = 48
    lat, Kn, Tv = specimen(n, 0, 4.0)
    fixed, up, _ = G.prescribed("k_xx", lat.x, lat.ijk, (n,) * 3, 1)
    geo = A3.AMGGeom(lat, ~fixed, agg=3, coarse_max=1000)
    h = A3.AMG3D(geo, Kn, Tv, nu=1, gamma=2, power_its=5,
                 Minv0=L3.k_block_jacobi(lat.block_diag(Kn, Tv), ~fixed))
    b = -L3.k_apply(up, lat.nbr, lat.ndir, Kn, Tv)
    A3._mask(b, ~fixed)
    x, it, rel = h.pcg(b, 1e-8)
    out.update(a48_it=it, a48_rel=rel, a48_rho=np.array([h.rho0] + list(h.rho)),
               a48_g=np.array([geo.l0["g"]] + [L["gc"] for L in geo.levels], np.int64))
    # interface cells (coarse3d/geom3d.py:134-147) of the 14^3 specimen and a 12^3 spheres image
    ph12, _ = micro3d.spheres(12, 12, 12, 0.25, 2.0, np.random.default_rng(4), rjit=0.0)
    out.update(iface_ph12=ph12.astype(np.int8), iface_12_2=G.interface_cells(ph12, 12, 2),
               iface_12_3=G.interface_cells(ph12, 12, 3))
    np.savez_compressed(os.path.join(HERE, "golden_amg.npz"), **out)
    print("golden_amg.npz:", len(out), "arrays")


def part_cfg3():
    """Dense-Cholesky gradient of the reference's 2D coarse model on the third benchmark configuration's inputs, at
    the coarse sizes its dense path reaches (nc = 32 from a 64^2 fine field, nc = 48 from 96^2; s = 2)."""
    _env()
    sys.path.insert(0, os.path.join(REF, "coarse2d"))
    import numpy as np
    import torch
    import cg as CG
    import lin2d as L2
    import micro as MI
    import torch_lpm as T2
    torch.set_default_dtype(torch.float64)
    out = {}
    loads = ["lr_tx", "tb_ty", "tb_sx"]
    for nc in (32, 48):
        s = 2
        nf = nc * s
        ph = MI.grf_two_phase(nf, nf, 6.0, 0.30, 3)
        E = np.where(ph == 1, 10.0, 1.0)
        Cpix = L2.iso_C(E, 0.25, plane="stress")
        m = T2.CoarseT(nc, nc, s, 1.0, device="cpu", loads=loads)
        lat = m.lat
        cp = CG.cell_params_from_C6(CG.voigt_cells(Cpix, nf, nf, s))
        K0, T0 = CG.bond_params_from_cells(lat, cp)
        rng = np.random.default_rng(11)
        q = np.where(lat.valid, lat.nbr, 0)
        opp = np.repeat(lat.opp[None, :], lat.N, 0)

        def lognormal_sym(rg):
            z = rg.standard_normal((lat.N, 8))
            z = np.where(np.arange(8)[None, :] % 2 == 0, z, z[q, opp])      # one factor per undirected bond
            return np.exp(0.2 * z)
        f0 = lognormal_sym(rng).astype(np.float32).astype(np.float64)
        ft = lognormal_sym(rng)
        with torch.no_grad():
            tgt = m.run(torch.tensor(K0 * ft)[None], torch.tensor(T0)[None])
        tgt = {ld: v["u"] for ld, v in tgt.items()}
        Kb = torch.tensor(K0 * f0)[None]
        Tb = torch.tensor(T0)[None]
        qt, ot = torch.as_tensor(q), torch.as_tensor(opp)
        valid = torch.as_tensor(lat.valid, dtype=torch.float64)
        th = torch.zeros((1, lat.N, 8), requires_grad=True)
        Kn = Kb * torch.exp(0.5 * (th + th[:, qt, ot])) * valid
        o = m.run(Kn, Tb)
        L = sum(((o[ld]["u"] - tgt[ld]) ** 2).mean() for ld in loads)
        L.backward()
        pre = "n%d_" % nc
        out.update({pre + "ph": ph, pre + "K0": K0, pre + "T0": T0, pre + "Kb": Kb.numpy()[0], pre + "loss": float(L),
                    pre + "gth": th.grad.numpy()[0]})
        for ld in loads:
            out[pre + "tgt_" + ld] = tgt[ld].numpy()[0]
            out[pre + "u_" + ld] = o[ld]["u"].detach().numpy()[0]
        print("nc", nc, "loss", float(L))
    np.savez_compressed(os.path.join(HERE, "golden_cfg3.npz"), **out)
    print("golden_cfg3.npz:", len(out), "arrays")


def part_sctv():
    """cement3d/torch_v1.py on a 6^3 coarse grid (s = 2) with two specimens whose solid masks remove ~20% of the
    cells: the operator's outputs under the masks and the gradient of a loss through CoarseTV.run (LinSolve)."""
    _env()
    sys.path.insert(0, os.path.join(REF, "coarse3d"))
    sys.path.insert(0, os.path.join(REF, "cement3d"))
    import numpy as np
    import torch
    import torch_v1 as TV
    torch.set_default_dtype(torch.float64)
    out = {}
    nc, s, B = 6, 2, 2
    cm = TV.CoarseTV(nc, s, device="cpu")
    lat = cm.lat
    N = lat.N
    rng = np.random.default_rng(31)
    solid = rng.random((B, N)) > 0.2
    Kn = np.zeros((B, N, 18))
    Tv = np.zeros((B, N, 18))
    for b in range(B):
        for i in range(N):
            for k in range(0, 18, 2):
                q = lat.nbr[i, k]
                if q >= 0:
                    Kn[b, i, k] = Kn[b, q, k ^ 1] = rng.uniform(0.8, 1.2)
                    Tv[b, i, k] = Tv[b, q, k ^ 1] = rng.uniform(-0.03, 0.03)
    op = cm.op
    st = torch.as_tensor(solid)
    op.set_mask(st)
    u = rng.standard_normal((B, 2, N, 3))
    Kt, Tt = torch.tensor(Kn)[:, None], torch.tensor(Tv)[:, None]
    out.update(solid=solid, Kn=Kn, Tv=Tv, u=u, valid=op.vb.numpy()[:, 0],
               Ku=op.apply(torch.tensor(u), Kt, Tt).numpy(), sig=op.stress(torch.tensor(u), Kt, Tt).numpy(),
               w=op.energy(torch.tensor(u), Kt, Tt).numpy(), D=op.block_diag(Kt, Tt).numpy())
    # differentiable CoarseTV.run: loss = sum of squares of u and stresses against fixed weights
    Kg = torch.tensor(Kn, requires_grad=True)
    Tg = torch.tensor(Tv, requires_grad=True)
    r = cm.run(Kg, Tg, cell=st, tol=1e-12)
    Wu = rng.standard_normal(tuple(r["u"].shape))
    Ws = rng.standard_normal(tuple(r["sig"].shape))
    L = (r["u"] * torch.tensor(Wu)).sum() * 1e3 + (r["sig"] * torch.tensor(Ws)).sum() * 1e3
    L.backward()
    out.update(run_u=r["u"].detach().numpy(), run_sig=r["sig"].detach().numpy(), run_w=r["w"].detach().numpy(),
               run_F=r["F"].detach().numpy(), Wu=Wu, Ws=Ws, loss=float(L.detach()), gKn=Kg.grad.numpy(),
               gTv=Tg.grad.numpy())
    np.savez_compressed(os.path.join(HERE, "golden_sctv.npz"), **out)
    print("golden_sctv.npz:", len(out), "arrays")


def part_asm():
    """coarse3d/train3d.py Scatter and group_penalty on a 5^3 coarse model (s = 2), B = 2, two bond groups (axial and
    diagonal forward bonds, every undirected bond once), values drawn so that some group Hessians fall below the
    penalty threshold."""
    _env()
    sys.path.insert(0, os.path.join(REF, "coarse3d"))
    import numpy as np
    import torch
    import torch_lpm3d as T
    import train3d as TR
    torch.set_default_dtype(torch.float64)
    nc, s, B = 5, 2, 2
    cm = T.CoarseT(nc, s, device="cpu")
    lat = cm.lat
    groups = []
    for slots in (range(0, 6, 2), range(6, 18, 2)):
        bonds = [np.stack([np.nonzero(lat.valid[:, k])[0], np.full(int(lat.valid[:, k].sum()), k)], 1) for k in slots]
        groups.append(dict(bonds=np.concatenate(bonds)))
    sc = TR.Scatter(nc, s, groups, device="cpu")
    rng = np.random.default_rng(41)
    vals, leaves = [], []
    for g in groups:
        nb = len(g["bonds"])
        kn = torch.tensor(rng.uniform(0.02, 1.0, (B, nb)), requires_grad=True)
        tv = torch.tensor(rng.uniform(-0.2, 0.1, (B, nb)), requires_grad=True)
        vals.append((kn, tv))
        leaves += [kn, tv]
    Kn, Tv = sc(vals)
    Wk = rng.standard_normal(tuple(Kn.shape))
    Wt = rng.standard_normal(tuple(Tv.shape))
    Ls = (Kn * torch.tensor(Wk)).sum() + (Tv * torch.tensor(Wt)).sum()
    gs = torch.autograd.grad(Ls, leaves, retain_graph=True)
    pen, lmin = TR.group_penalty(cm, Kn, Tv, frac=0.05)
    gp = torch.autograd.grad(pen.sum(), leaves)
    out = dict(Kn=Kn.detach().numpy(), Tv=Tv.detach().numpy(), Wk=Wk, Wt=Wt, pen=pen.detach().numpy(),
               lmin=float(lmin))
    for i, g in enumerate(groups):
        out["bonds%d" % i] = g["bonds"]
        out["kn%d" % i] = vals[i][0].detach().numpy()
        out["tv%d" % i] = vals[i][1].detach().numpy()
        out["gs_kn%d" % i], out["gs_tv%d" % i] = gs[2 * i].numpy(), gs[2 * i + 1].numpy()
        out["gp_kn%d" % i], out["gp_tv%d" % i] = gp[2 * i].numpy(), gp[2 * i + 1].numpy()
    print("penalty", pen.detach().numpy(), "lmin", float(lmin))
    np.savez_compressed(os.path.join(HERE, "golden_asm.npz"), **out)
    print("golden_asm.npz:", len(out), "arrays")


PARTS = {"asm": part_asm, "sc": part_sc, "sq": part_sq, "grad": part_grad, "amg": part_amg, "cfg3": part_cfg3, "sctv": part_sctv}

if __name__ == "__main__":
    if not REF or not os.path.isdir(REF):
        sys.exit("set LPM_REFERENCE to the root of the reference checkout")
    if len(sys.argv) > 1 and sys.argv[1] in PARTS:
        PARTS[sys.argv[1]]()
    else:
        for p in PARTS:
            subprocess.run([sys.executable, os.path.abspath(__file__), p], check=True)
