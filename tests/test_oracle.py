"""Pins the CPU oracle (oracle/lpm_oracle.c) to golden vectors produced by the reference itself.

The oracle is the checker of the CUDA library, so it is checked first: kernels to round-off, solvers against the
reference's SuperLU answers and iteration counts, gradients against the reference's autograd.
"""
import numpy as np
import pytest

import oracle as O
from conftest import relmax
from lpm_b200 import geom as G


@pytest.fixture(scope="module")
def sc12(gsc):
    return G.LatticeGeom(12, 12, 12, 1.0), gsc["Kn"], gsc["Tv"]


def test_sc_kernels(gsc, sc12):
    lat, Kn, Tv = sc12
    u = gsc["u"]
    assert relmax(O.sc_apply(lat, u, Kn, Tv), gsc["Ku"]) < 1e-13
    assert relmax(O.sc_stress(lat, u, Kn, Tv), gsc["st"]) < 1e-13
    assert relmax(O.sc_energy(lat, u, Kn, Tv), gsc["U"]) < 1e-13
    assert relmax(O.sc_block_diag(lat, Kn, Tv), gsc["D"]) < 1e-13
    dL, F = O.sc_bond_forces(lat, u, Kn, Tv)
    assert relmax(F[::97], gsc["F_row"]) < 1e-13 and relmax(dL[::97], gsc["dL_row"]) < 1e-13


@pytest.mark.parametrize("s", [2, 3])
def test_sc_pcg_vs_superlu(gsc, sc12, s):
    """FP64 block-Jacobi PCG to 1e-12 vs the reference's SuperLU block means (coarse3d/check_torch3d.py:34-46)."""
    lat, Kn, Tv = sc12
    nc = 12 // s
    cid = G.block_index(lat.ijk, s, (nc,) * 3)
    for ld in G.LOADS:
        fixed, up, mov = G.prescribed(ld, lat.x, lat.ijk // s, (nc,) * 3, s)
        u, info = O.solve_pcg(lat, Kn, Tv, fixed, up, tol=1e-12)
        assert info["relres"] <= 1e-12
        ub = np.stack([np.bincount(cid, u[:, k]) for k in range(3)], 1) / s ** 3
        assert relmax(ub, gsc["u_%d_%s" % (s, ld)]) < 1e-9
        st = O.sc_stress(lat, u, Kn, Tv)
        sb = np.stack([np.bincount(cid, st[:, k]) for k in range(6)], 1) / s ** 3
        assert relmax(sb, gsc["s_%d_%s" % (s, ld)]) < 1e-8
        if mov is not None:
            P = O.sc_apply(lat, u, Kn, Tv)
            assert abs(P[mov, G.GDIR[ld]].sum() / gsc["F_%d_%s" % (s, ld)] - 1) < 1e-8
        key = "ufull_%d_%s" % (s, ld)
        if key in gsc:
            assert relmax(u, gsc[key]) < 1e-9


@pytest.mark.parametrize("ld", ["k_xx", "tb_sx"])
def test_sc_iteration_counts(gsc, sc12, ld):
    """Same iteration counts as lin3d.solve_pcg and cgplain.cg3 at tol 1e-8 (rounding order may shift by one)."""
    lat, Kn, Tv = sc12
    fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk // 2, (6,) * 3, 2)
    u, info = O.solve_pcg(lat, Kn, Tv, fixed, up, tol=1e-8)
    assert abs(info["iters"] - int(gsc["pcg_it_%s" % ld])) <= 1
    assert relmax(u, gsc["pcg_u_%s" % ld]) < 1e-6
    u, info = O.solve_pcg(lat, Kn, Tv, fixed, up, tol=1e-8, precond=False)
    assert abs(info["iters"] - int(gsc["cg_it_%s" % ld])) <= 1
    assert relmax(u, gsc["cg_u_%s" % ld]) < 1e-6


def test_sc_grad(ggrad):
    lat = G.LatticeGeom(4, 4, 4, 2.0)
    for pre in ("g3", "g3n"):
        gK, gT = O.sc_grad(lat, ggrad[pre + "_Kn"], ggrad[pre + "_Tv"], ggrad["g3_u"], ggrad["g3_lam"])
        assert relmax(gK, ggrad[pre + "_gK"]) < 1e-13
        assert relmax(gT, ggrad[pre + "_gT"]) < 1e-13


def test_sq_kernels(gsq):
    lat = G.Lattice2D("square", 16, 12, 1.0)
    f = O.sq_kmv(lat, gsq["u"], gsq["Kn_ns"], gsq["Tv_ns"])
    assert relmax(f, gsq["f_ns"]) < 1e-13
    assert relmax(f, gsq["Ku_csr_ns"]) < 1e-13
    assert relmax(O.sq_diag_inv(lat, gsq["Kn"], gsq["Tv"], gsq["diag_fixed"]), gsq["Binv"]) < 1e-13
    assert relmax(O.sq_stress(lat, gsq["u"], gsq["Kn"], gsq["Tv"]), gsq["stress"]) < 1e-13
    assert relmax(O.sq_energy(lat, gsq["u"], gsq["Kn"], gsq["Tv"]), gsq["energy"]) < 1e-13


def test_sq_solves(gsq):
    lat = G.Lattice2D("square", 16, 12, 1.0)
    u, info = O.sq_solve_cg(lat, gsq["Kn"], gsq["Tv"], gsq["cg_fixed"], gsq["cg_up"], tol=1e-10)
    assert abs(info["iters"] - int(gsq["cg_it"])) <= 1
    assert relmax(u.ravel(), gsq["cg_u"]) < 1e-8
    assert relmax(u.ravel(), gsq["lu_u"]) < 1e-7
    fixed = gsq["pcg_fixed"]
    fd = np.repeat(fixed[:, None], 2, 1)
    u, info = O.sq_solve_cg(lat, gsq["Kn"], gsq["Tv"], fd, gsq["pcg_up"], tol=1e-10, precond=True)
    assert abs(info["iters"] - int(gsq["pcg_it"])) <= 1
    assert relmax(u.ravel(), gsq["pcg_u"]) < 1e-8


def test_sq_grad(ggrad):
    lat = G.Lattice2D("square", 6, 5, 2.0)
    gK, gT = O.sq_grad(lat, ggrad["g2_u"], ggrad["g2_lam"])
    assert relmax(gK * lat.valid, ggrad["g2_gK"]) < 1e-13
    assert relmax(gT * lat.valid, ggrad["g2_gT"]) < 1e-13
    Ku = O.sq_kmv(lat, ggrad["g2_u"], ggrad["g2_Kn"], ggrad["g2_Tv"])
    assert relmax(Ku, ggrad["g2_Ku"]) < 1e-13
