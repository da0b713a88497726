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
    assert lib.lpm_abi_version() == 2
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
