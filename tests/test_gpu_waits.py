"""The bounded device waits of the TMA-fed operators made to run out, on purpose and safely: with the poll bound at 0
(lpm_set_tma_wait_polls) every data wait expires at once, so the pair-packed FP32 operator (k_sc_pair) and its FP64
instantiation (one system per lane group) take their abort path inside a CG solve: the block decides to stop at one barrier, lets the
copies it issued land with the full bound and returns, and the engine reports LPM_ERR_TIMEOUT.  Nothing hangs or
faults: the next solve on the same GPU, with the default bound, gives the oracle's answer."""
import numpy as np
import pytest
import torch

import oracle as O
from lpm_b200 import _lib as L
from lpm_b200 import core
from lpm_b200 import geom as G
from lpm_b200 import micro as M

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def case(n=24):
    lat = G.LatticeGeom(n, n, n, 1.0)
    ph, _ = M.spheres(n, n, n, 0.25, 3.0, np.random.default_rng(2), rjit=0.0)
    C = G.iso_C(np.where(ph == 1, 10.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    fixed, up, _ = G.prescribed("k_xy", lat.x, lat.ijk, (n,) * 3, 1)
    up = np.where(fixed[:, None], up, 0.0)
    return lat, Kn, Tv, fixed, up


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_tma_wait_expiry_aborts_and_recovers(dtype):
    lat, Kn, Tv, fixed, up = case()
    dl = core.DeviceLattice(lat, DEV)
    Kd, Td = torch.as_tensor(Kn, device=DEV)[None], torch.as_tensor(Tv, device=DEV)[None]
    Kp, Tp = core.pack(Kd, dtype), core.pack(Td, dtype)
    free = torch.as_tensor(~fixed, device=DEV, dtype=dtype)[None]
    b64 = -core.kmv(dl, torch.as_tensor(up, device=DEV)[None], Kd, Td) * free.double()[..., None]
    b = torch.cat([b64, b64], 0).to(dtype)             # two systems of one set: one pair for the FP32 operator
    fr2 = torch.cat([free, free], 0)
    tol = 1e-5 if dtype == torch.float32 else 1e-10
    kw = dict(free=fr2, check=1, layout=L.LAYOUT_SOA, rhs_per_set=2, engine=L.ENGINE_LAUNCHED)
    x0, i0 = core.cg(dl, Kp, Tp, b, tol=tol, maxit=5000, **kw)          # before: the default bound
    lib = L.load()
    prev = lib.lpm_set_tma_wait_polls(0)
    try:
        with pytest.raises(L.LPMError, match=r"code -5"):
            core.cg(dl, Kp, Tp, b, tol=1e-6, maxit=50, **kw)
    finally:
        assert lib.lpm_set_tma_wait_polls(prev) == 0
    assert prev == 1 << 22
    torch.cuda.synchronize()
    x1, i1 = core.cg(dl, Kp, Tp, b, tol=tol, maxit=5000, **kw)          # after: same GPU, default bound
    assert (i1.status == 0).all() and np.array_equal(i0.iters, i1.iters)
    assert torch.equal(x0, x1)                                          # deterministic: bit for bit
    if dtype == torch.float64:
        uo, _ = O.solve_pcg(lat, Kn, Tv, fixed, up, tol=1e-12)
        xo = uo - up
        for s in range(2):
            assert np.linalg.norm(x1[s].cpu().numpy() - xo) / np.linalg.norm(xo) < 1e-6, s
