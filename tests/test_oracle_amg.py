"""Pins the AMG oracle (oracle/amg.py) to the reference's own aggregation AMG (timing/t3d/amg3d.py), run by
tests/golden/make_golden.py: geometry, numeric hierarchy, one preconditioner application and the PCG iterations."""
import numpy as np
import pytest

import amg as A
import oracle as O
from conftest import relmax
from lpm_b200 import geom as G
from lpm_b200 import micro as M

SETS = (("ring", "k_xx"), ("tb", "tb_tz"), ("lr", "lr_tx"))


@pytest.fixture(scope="module")
def hier14(gamg):
    n = int(gamg["a_n"])
    lat = G.LatticeGeom(n, n, n, 1.0)
    out, rho0 = {}, None
    for name, ld in SETS:
        fixed, up, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        geo = A.Geometry(lat, ~fixed, agg=3, coarse_max=100)
        h = A.Hierarchy(geo, gamg["a_Kn"], gamg["a_Tv"], rho0=rho0)
        rho0 = h.rho0
        out[name] = (lat, fixed, up, geo, h)
    return out


@pytest.mark.parametrize("name", [s[0] for s in SETS])
def test_amg_geometry_and_setup(gamg, hier14, name):
    lat, fixed, up, geo, h = hier14[name]
    p = "a_%s_" % name
    assert np.array_equal(np.array(geo.grids), gamg[p + "g"])
    assert np.array_equal(geo.agg_of0, gamg[p + "agg_of"])
    assert np.abs(geo.P - gamg[p + "P"]).max() < 1e-14
    assert np.abs(geo.levels[0]["Q"] - gamg[p + "Q1"]).max() < 1e-14
    assert relmax([h.rho0] + h.rho, gamg[p + "rho"]) < 1e-12
    assert relmax(h.A[0], gamg[p + "A1"]) < 1e-6  # the fixture holds A1 in FP32
    assert relmax(h.A[1], gamg[p + "A2"]) < 1e-12


@pytest.mark.parametrize("name", [s[0] for s in SETS])
def test_amg_vcycle_and_pcg(gamg, hier14, name):
    lat, fixed, up, geo, h = hier14[name]
    p = "a_%s_" % name
    assert relmax(h.vcycle(gamg[p + "vin"].copy()), gamg[p + "vout"]) < 1e-12
    b = -O.sc_apply(lat, up, gamg["a_Kn"], gamg["a_Tv"])
    b[fixed] = 0.0
    x, it, rel = h.pcg(b, 1e-8)
    assert it == int(gamg[p + "pcg_it"]) and abs(rel - float(gamg[p + "pcg_rel"])) < 1e-12
    assert relmax(up + x, gamg[p + "pcg_x"]) < 1e-12


def test_amg_iterations_48(gamg):
    """The 48^3 spheres specimen of the bench (ring BCs, k_xx): same hierarchy, rho and PCG iterations."""
    n = 48
    lat = G.LatticeGeom(n, n, n, 1.0)
    ph, _ = M.spheres(n, n, n, 0.25, 4.0, np.random.default_rng(0), rjit=0.0)
    C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    fixed, up, _ = G.prescribed("k_xx", lat.x, lat.ijk, (n,) * 3, 1)
    geo = A.Geometry(lat, ~fixed)
    assert np.array_equal(np.array(geo.grids), gamg["a48_g"])
    h = A.Hierarchy(geo, Kn, Tv)
    assert relmax([h.rho0] + h.rho, gamg["a48_rho"]) < 1e-10
    b = -O.sc_apply(lat, up, Kn, Tv)
    b[fixed] = 0.0
    x, it, rel = h.pcg(b, 1e-8)
    assert it == int(gamg["a48_it"]) and abs(rel - float(gamg["a48_rel"])) < 1e-12


def test_interface_cells(gamg):
    """geom.interface_cells restates coarse3d/geom3d.py:134-147 (the iface_s arrays of data/fine_*.npz)."""
    for s in (2, 3):
        assert np.array_equal(G.interface_cells(gamg["iface_ph12"], 12, s), gamg["iface_12_%d" % s])
