"""The allocation-free K.u entry point (lpm_kmv_f64_static) against the regular one (lpm_kmv_sc_f64 /
lpm_kmv_sq_f64).

lpm_kmv_f64_static serves callers that cannot allocate device memory or hand over a scratch buffer: it keeps its
scratch in a fixed device array inside the library.  This file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from lpm_b200 import _lib as L
from lpm_b200 import core, geom as G

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda"


def _call_static(dl, u, Kn, Tv, rhs_per_set, layout=L.LAYOUT_REF):
    out = torch.empty_like(u)
    b = L.Batch(u.shape[0], rhs_per_set, 1, 0)
    rc = L.load().lpm_kmv_f64_static(dl.ref, L.ptr(u), L.ptr(Kn), L.ptr(Tv), layout, ctypes.byref(b),
                                     L.ptr(out), L.stream_ptr())
    return rc, out


@pytest.mark.parametrize("dim,layout", [(3, L.LAYOUT_REF), (3, L.LAYOUT_SOA), (2, L.LAYOUT_REF), (2, L.LAYOUT_SOA)])
def test_static_scratch_kmv_matches_regular_entry_point(dim, layout):
    """Both coefficient layouts on full boxes; with the packed (SoA) layout the regular SC call runs the single-pass
    TMA operator, so the two entry points agree within rounding (1e-13), not bit for bit."""
    rng = np.random.default_rng(dim)
    lat = G.LatticeGeom(24, 18, 13) if dim == 3 else G.Lattice2D("square", 75, 41, 1.0)
    dl = core.DeviceLattice(lat)
    nset, rps = 2, 3
    Kn = torch.as_tensor(rng.uniform(0.5, 1.5, (nset, lat.N, lat.NN)) * lat.valid, device=DEV)
    Tv = torch.as_tensor(rng.uniform(-0.05, 0.05, (nset, lat.N, lat.NN)) * lat.valid, device=DEV)
    u = torch.as_tensor(rng.standard_normal((nset * rps, lat.N, dim)), device=DEV)
    if layout == L.LAYOUT_SOA:
        Kn, Tv = core.pack(Kn, torch.float64), core.pack(Tv, torch.float64)
        ref = core.kmv(dl, u, Kn, Tv, layout=layout, rhs_per_set=rps)
    else:
        ref = core.kmv(dl, u.view(nset, rps, lat.N, dim), Kn[:, None], Tv[:, None]).reshape(nset * rps, lat.N, dim)
    for _ in range(2):                      # two calls in a row share (and reuse) the static array
        rc, out = _call_static(dl, u, Kn, Tv, rps, layout)
        assert rc == 0, L.load().lpm_status_string(rc)
        torch.cuda.synchronize()
        err = float((out - ref).abs().max() / ref.abs().max())
        assert err < 1e-13


def test_static_scratch_rejects_oversized_batches():
    lat = G.LatticeGeom(48, 48, 48)
    dl = core.DeviceLattice(lat)
    nsys = 10                               # 4 * 10 * 110592 doubles > 32 MiB
    assert 4 * nsys * lat.N * 8 > 32 * 1024 * 1024
    u = torch.zeros((nsys, lat.N, 3), dtype=torch.float64, device=DEV)
    Kn = torch.zeros((1, lat.N, 18), dtype=torch.float64, device=DEV)
    rc, _ = _call_static(dl, u, Kn, Kn, nsys)
    assert rc == -2
