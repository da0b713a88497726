"""CPU checks of the C ABI: the library loads and exports every entry point that include/lpm_b200.h declares, and
argument validation rejects bad input before any device work."""
import ctypes
import os
import re

import pytest

from lpm_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(lpm_\w+)\s*\(", src))
    return sorted(names)


def test_library_exports_header():
    lib = L.load()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.exported_symbols())


def test_abi_version_and_strings():
    lib = L.load()
    assert lib.lpm_abi_version() == 4
    assert lib.lpm_status_string(0) == b"ok"
    assert b"argument" in lib.lpm_status_string(-1)
    assert b"workspace" in lib.lpm_status_string(-2)


def test_argument_validation():
    lib = L.load()
    bad = L.Lattice(4, 8, 8, 8, 512, None)        # dim 4
    assert lib.lpm_kmv_scratch_bytes(ctypes.byref(bad), 0, 1) < 0
    wrong_n = L.Lattice(3, 8, 8, 8, 100, None)    # full box with n != nx*ny*nz
    one = L.Batch(1, 1, 1, 0)
    assert lib.lpm_cg_workspace_bytes(ctypes.byref(wrong_n), ctypes.byref(one), 0, 0) < 0
    sq_nz = L.Lattice(2, 8, 8, 3, 192, None)      # 2D with nz != 1
    assert lib.lpm_ir_workspace_bytes(ctypes.byref(sq_nz), ctypes.byref(one), 1) < 0
    ok = L.Lattice(3, 8, 8, 8, 512, None)
    assert lib.lpm_kmv_scratch_bytes(ctypes.byref(ok), 1, 2) >= 2 * 512 * 4 * 4
    six = L.Batch(6, 6, 1, 0)
    assert lib.lpm_cg_workspace_bytes(ctypes.byref(ok), ctypes.byref(six), 1, 1) > 0
    b = L.Batch(0, 1, 1, 0)                        # nsys 0
    rc = lib.lpm_kmv_sc_f64(ctypes.byref(ok), None, None, None, 0, ctypes.byref(b), None, None, 0, None)
    assert rc == -1
    assert lib.lpm_pack_coef_f32(None, None, 10, 18, 1, None) == -1
    assert lib.lpm_build_nbr(5, 2, 2, 2, 8, None, None, None, None) == -1


def test_no_cpu_fallback():
    torch = pytest.importorskip("torch")
    from lpm_b200 import core, geom
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU behaviour")
    with pytest.raises(L.LPMError):
        core.DeviceLattice(geom.LatticeGeom(4, 4, 4), device="cpu")


def test_amg_create_validation():
    """lpm_amg_create rejects bad boxes, masks and options on the host, before any device work."""
    lib = L.load()
    lat = L.Lattice(3, 12, 12, 12, 12 ** 3, None)
    b = L.Batch(2, 2, 2, 0)
    o = L.AmgOpts()
    lib.lpm_amg_default_opts(ctypes.byref(o))
    assert (o.agg, o.coarse_max, o.nu, o.gamma, o.power_its) == (3, 1000, 1, 2, 5) and abs(o.omega - 1.32) < 1e-15
    h = ctypes.c_void_p(None)
    box = (ctypes.c_int32 * 6)(1, 1, 1, 10, 10, 10)
    of = (ctypes.c_int32 * 2)(0, 0)
    bad_box = (ctypes.c_int32 * 6)(1, 1, 1, 12, 10, 10)           # hi beyond the lattice
    assert lib.lpm_amg_create(ctypes.byref(lat), ctypes.byref(b), bad_box, 1, of, ctypes.byref(o),
                              ctypes.byref(h)) == -1
    bad_of = (ctypes.c_int32 * 2)(0, 1)                              # mask 1 names box 1 of a single box
    assert lib.lpm_amg_create(ctypes.byref(lat), ctypes.byref(b), box, 1, bad_of, ctypes.byref(o),
                              ctypes.byref(h)) == -1
    thin = (ctypes.c_int32 * 6)(0, 0, 0, 0, 0, 11)                    # a line: rank-deficient aggregates
    assert lib.lpm_amg_create(ctypes.byref(lat), ctypes.byref(b), thin, 1, of, ctypes.byref(o),
                              ctypes.byref(h)) == -3
    o2 = L.AmgOpts()
    lib.lpm_amg_default_opts(ctypes.byref(o2))
    o2.agg = 2                                                       # aggregates must be at least 3 sites wide
    assert lib.lpm_amg_create(ctypes.byref(lat), ctypes.byref(b), box, 1, of, ctypes.byref(o2),
                              ctypes.byref(h)) == -3
    assert not h.value
