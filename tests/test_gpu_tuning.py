"""The z-chunk autotuner: returns a chunking the library then uses, and K.u results do not depend on the chunking
(every site's value is computed the same way whatever the chunk boundaries)."""
import numpy as np
import pytest

import oracle as O
from conftest import relmax
from lpm_b200 import _lib, core, geom as G

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_autotune_keeps_results():
    lat = G.LatticeGeom(32, 24, 40)
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(3)
    Kn = rng.uniform(0.5, 1.5, (2, lat.N, 18)) * lat.valid
    Tv = rng.uniform(-0.05, 0.05, (2, lat.N, 18)) * lat.valid
    u = rng.standard_normal((6, lat.N, 3))
    T = lambda a, dt=torch.float64: torch.as_tensor(a, device="cuda", dtype=dt)
    K32, T32 = core.pack(T(Kn), torch.float32), core.pack(T(Tv), torch.float32)
    before = core.kmv(dl, T(u, torch.float32), K32, T32, layout=_lib.LAYOUT_SOA, rhs_per_set=3).cpu().numpy()
    z = core.autotune(dl, K32, T32, 6, 3)
    assert 8 <= z <= lat.nz or z == lat.nz
    after = core.kmv(dl, T(u, torch.float32), K32, T32, layout=_lib.LAYOUT_SOA, rhs_per_set=3).cpu().numpy()
    assert np.array_equal(before, after)
    ref = O.sc_apply(lat, u[4], Kn[1], Tv[1])
    assert relmax(after[4], ref) < 3e-6
