"""Host geometry mirror vs the reference's golden arrays: connectivity bit-exact, BCs and maps to round-off."""
import numpy as np

from conftest import relmax
from lpm_b200 import geom as G


def test_sc_connectivity_full(gsc):
    lat = G.LatticeGeom(12, 12, 12, 1.0)
    assert lat.nbr.dtype == np.int64
    assert np.array_equal(lat.nbr, gsc["nbr"].astype(np.int64))
    assert np.array_equal(lat.valid, gsc["nbr"] >= 0)
    assert np.array_equal(lat.opp, np.arange(18) ^ 1)


def test_sc_connectivity_masked(gsc):
    lat = G.LatticeGeom(7, 5, 4, 1.5, origin=(0.1, -0.2, 0.3), active=gsc["m_active"])
    assert np.array_equal(lat.nbr, gsc["m_nbr"].astype(np.int64))
    assert np.array_equal(lat.ijk, gsc["m_ijk"])
    assert np.array_equal(lat.site_of, gsc["m_site_of"])
    assert np.array_equal(lat.nb_initial, gsc["m_nb_initial"])
    assert np.allclose(lat.x, gsc["m_x"], rtol=0, atol=1e-15)


def test_sq_connectivity(gsq):
    lat = G.Lattice2D("square", 16, 12, 1.0)
    assert np.array_equal(lat.nbr, gsq["nbr"].astype(np.int64))
    lm = G.Lattice2D("square", 9, 7, 0.5, origin=(0.3, 0.1), active=gsq["m_active"])
    assert np.array_equal(lm.nbr, gsq["m_nbr"].astype(np.int64))
    assert np.array_equal(lm.ij, gsq["m_ij"])
    assert np.allclose(lm.x, gsq["m_x"], rtol=0, atol=1e-15)


def test_sc_params_and_bcs(gsc):
    lat = G.LatticeGeom(12, 12, 12, 1.0)
    C = G.iso_C(gsc["E"], gsc["nu"])
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    assert relmax(Kn, gsc["Kn"]) < 1e-15 and relmax(Tv, gsc["Tv"]) < 1e-15
    lb = G.LatticeGeom(6, 6, 6, 1.0)
    for ld in G.LOADS:
        fixed, up, mov = G.prescribed(ld, lb.x, lb.ijk // 2, (3, 3, 3), 2)
        assert np.array_equal(fixed, gsc["bc_fixed_%s" % ld])
        assert np.allclose(up, gsc["bc_up_%s" % ld], rtol=0, atol=1e-18)
        m = np.zeros(lb.N, bool) if mov is None else mov
        assert np.array_equal(m, gsc["bc_mov_%s" % ld])
    assert relmax(G.cell_params_from_C66(gsc["cp_C66"], 0.7), gsc["cp_params"]) < 1e-14


def test_sq_params_and_bcs(gsq):
    lat = G.Lattice2D("square", 16, 12, 1.0)
    E = np.where(gsq["phase"] == 1, 10.0, 1.0)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.square_params_from_C(G.iso_C2d(E, 0.25, plane="stress")))
    assert relmax(Kn, gsq["Kn"]) < 1e-15 and relmax(Tv, gsq["Tv"]) < 1e-15
    lb = G.Lattice2D("square", 8, 8, 1.0)
    for L in (1, 2):
        for ld in G.LOADS2D:
            fixed, up, _ = G.prescribed2d(ld, lb.x, lb.ij // 2, 4, 4, 2, 1.0, L)
            assert np.array_equal(fixed, gsq["bc_fixed_%d_%s" % (L, ld)])
            assert np.allclose(up, gsq["bc_up_%d_%s" % (L, ld)], rtol=0, atol=1e-18)
    fd, up, _ = G.uniaxial_tension_2d(lat)
    assert np.array_equal(fd, gsq["cg_fixed"]) and np.allclose(up, gsq["cg_up"], rtol=0, atol=1e-18)


def test_generators(gsc, gsq):
    from lpm_b200 import micro
    assert np.array_equal(micro.grf_two_phase(40, 32, 6.0, 0.30, 3), gsq["gen_grf"])
    assert np.array_equal(micro.spheres(16, 16, 16, 0.25, 4.0, np.random.default_rng(7), rjit=0.0)[0],
                          gsc["gen_spheres"])
    assert np.array_equal(micro.ellipsoids(16, 16, 16, 0.3, 3.0, np.random.default_rng(8), aspect=(3.0, 3.0),
                                           rjit=0.0)[0], gsc["gen_ellip"])
    assert np.array_equal(micro.grf3(12, 12, 12, 2.0, 0.3, np.random.default_rng(9))[0], gsc["gen_grf3"])


def test_cfg3_inputs_match_reference():
    """The third configuration's coarse-parameter pipeline (GRF fine field -> Voigt cells -> two-end-mean bonds,
    coarse2d/micro.py:13-20 and coarse2d/cg.py:201-234) reproduces the reference's arrays at nc = 32 and 48."""
    from lpm_b200 import micro
    from conftest import GOLDEN
    import os
    with np.load(os.path.join(GOLDEN, "golden_cfg3.npz")) as d:
        g = {k: d[k] for k in d.files}
    for nc in (32, 48):
        pre = "n%d_" % nc
        nf = 2 * nc
        ph = micro.grf_two_phase(nf, nf, 6.0, 0.30, 3)
        assert np.array_equal(ph, g[pre + "ph"])
        Cpix = G.iso_C2d(np.where(ph == 1, 10.0, 1.0), 0.25, plane="stress")
        lat = G.SquareLattice(nc, nc, 2.0)
        cp = G.cell_params_from_C6(G.voigt_cells2d(Cpix, nf, nf, 2))
        K0, T0 = G.bond_params_from_cells2d(lat, cp)
        assert relmax(K0, g[pre + "K0"]) < 1e-15 and relmax(T0, g[pre + "T0"]) < 1e-15
