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
    z, v = core.autotune(dl, K32, T32, 6, 3, with_variant=True)
    assert (8 <= z <= lat.nz or z == lat.nz) and v in (0, 1)
    after = core.kmv(dl, T(u, torch.float32), K32, T32, layout=_lib.LAYOUT_SOA, rhs_per_set=3).cpu().numpy()
    assert np.array_equal(before, after)
    ref = O.sc_apply(lat, u[4], Kn[1], Tv[1])
    assert relmax(after[4], ref) < 3e-6


@pytest.mark.parametrize("shape", [(48, 48, 48), (36, 9, 5), (32, 24, 40), (16, 20, 33)])
def test_variants_and_chunkings_agree(shape):
    """Both operator variants (tiles staged in shared memory / lean, two CTAs per SM) and several z-chunkings give
    bit-identical K.u, and match the oracle; also through a mixed-precision solve."""
    lat = G.LatticeGeom(*shape)
    dl = core.DeviceLattice(lat)
    rng = np.random.default_rng(sum(shape))
    Kn = rng.uniform(0.5, 1.5, (1, lat.N, 18)) * lat.valid
    Tv = rng.uniform(-0.05, 0.05, (1, lat.N, 18)) * lat.valid
    u = rng.standard_normal((5, lat.N, 3))
    T = lambda a, dt=torch.float64: torch.as_tensor(a, device="cuda", dtype=dt)
    K32, T32 = core.pack(T(Kn), torch.float32), core.pack(T(Tv), torch.float32)
    outs = []
    for z in sorted({lat.nz, min(lat.nz, max(8, (lat.nz + 1) // 2))}):
        if (lat.nz + z - 1) // z > max(1, lat.nz // 8):
            continue
        for v in (0, 1):
            core.tune_set(dl, 5, 5, z, v)
            outs.append(core.kmv(dl, T(u, torch.float32), K32, T32, layout=_lib.LAYOUT_SOA, rhs_per_set=5).cpu().numpy())
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    for s in range(5):
        assert relmax(outs[0][s], O.sc_apply(lat, u[s], Kn[0], Tv[0])) < 3e-6
