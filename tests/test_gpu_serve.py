"""Serving on the GPU: every result is the same alone and in a mixed stream (2D and 3D sizes, 1-5 load cases, staggered
arrivals), and matches the FP64 PCG solution to the mixed-precision bar (1e-6 relative displacement)."""
import time

import numpy as np
import pytest

from lpm_b200 import core, geom as G, micro, serve

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def spec3(n, seed, loads):
    lat = G.LatticeGeom(n, n, n, 1.0)
    ph, _ = micro.spheres(n, n, n, 0.25, 3.0, np.random.default_rng(seed), rjit=0.0)
    C = G.iso_C(np.where(ph == 1, 8.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    free, up = [], []
    for ld in loads:
        fixed, u, _ = G.prescribed(ld, lat.x, lat.ijk, (n,) * 3, 1)
        free.append(np.repeat(~fixed[:, None], 3, 1))
        up.append(np.where(fixed[:, None], u, 0.0))
    return serve.Request(3, (n,) * 3, Kn, Tv, np.array(free), np.array(up))


def spec2(nx, ny, seed, nloads):
    lat = G.SquareLattice(nx, ny, 1.0)
    ph = micro.grf_two_phase(nx, ny, 4.0, 0.3, seed)
    C = G.iso_C2d(np.where(ph == 1, 10.0, 1.0), 0.25, plane="stress")
    Kn, Tv = G.bond_params_two_end_mean(lat, G.square_params_from_C(C))
    free, up = [], []
    for k in range(nloads):
        fd, u, _ = G.uniaxial_tension_2d(lat, strain=1e-3 * (k + 1))
        free.append(~fd)
        up.append(u)
    return serve.Request(2, (nx, ny), Kn, Tv, np.array(free), np.array(up))


def spec3_custom(n, seed):
    """A 3D request with a boundary mask outside the standard load set (bottom and top faces and the x = 0 face held,
    the top face pulled along z): it is served by a block-Jacobi bucket."""
    lat = G.LatticeGeom(n, n, n, 1.0)
    ph, _ = micro.spheres(n, n, n, 0.25, 3.0, np.random.default_rng(seed), rjit=0.0)
    C = G.iso_C(np.where(ph == 1, 8.0, 1.0), 0.2)
    Kn, Tv = G.bond_params_two_end_mean(lat, G.sc_params_from_C(C, 0.5))
    i, k = lat.ijk[:, 0], lat.ijk[:, 2]
    fixed = (k == 0) | (k == n - 1) | (i == 0)
    up = np.zeros((lat.N, 3))
    up[(k == n - 1) & (i > 0), 2] = 1e-3 * (n - 1)
    return serve.Request(3, (n,) * 3, Kn, Tv, np.repeat(~fixed[:, None], 3, 1)[None], up[None])


def fp64_reference(r):
    lat = G.LatticeGeom(*r.shape, 1.0) if r.dim == 3 else G.SquareLattice(*r.shape, 1.0)
    dl = core.DeviceLattice(lat)
    T = lambda a: torch.as_tensor(a, device="cuda")
    Kn, Tv = T(r.Kn), T(r.Tv)
    free = T(r.free.astype(np.float64))
    up = T(r.up) * (1 - free)
    b = -core.kmv(dl, up, Kn, Tv) * free
    M = core.block_jacobi(dl, Kn, Tv, torch.float64)
    x, info = core.cg(dl, Kn, Tv, b, Minv=M, free=free, tol=1e-12, maxit=50000, check=1, poll=50)
    assert (info.status == 0).all()
    return (up + x).cpu().numpy()


def run(reqs, gaps, keys=None):
    srv = serve.Server(budget_bytes=8 << 30, rmax=6, max_slots=3)
    try:
        for r, g in zip(reqs, gaps):
            srv.submit(r)
            time.sleep(g)
        done = srv.wait_all(len(reqs), timeout=600)
        if keys is not None:
            keys.extend(srv.bucket_log)
        return done
    finally:
        srv.close()


def test_alone_equals_in_the_mix():
    def make():
        return [spec3(24, 1, ["k_xx", "k_yy", "k_xy"]), spec2(40, 32, 2, 2), spec3(24, 3, ["k_zz", "tb_tz"]),
                spec3(16, 4, G.LOADS[:5]), spec2(40, 32, 5, 1), spec3(24, 6, ["lr_tx"]), spec3_custom(24, 7)]
    mixed = make()
    keys = []
    run(mixed, [0.0, 0.01, 0.02, 0.0, 0.03, 0.0, 0.0], keys)
    # standard load boxes in AMG buckets, the custom mask in a block-Jacobi bucket of the same size
    assert {(3, 24, 24, 24, "amg"), (3, 16, 16, 16, "amg"), (3, 24, 24, 24), (2, 40, 32, 1)} <= set(keys)
    for r in mixed:
        assert r.status == 0 and (r.relres <= 1e-8).all(), (r.key, r.relres)
    alone = make()
    for r in alone:
        run([r], [0.0])
    for a, m in zip(alone, mixed):
        d = np.abs(a.u - m.u).max() / np.abs(a.u).max()
        assert d <= 1e-12, (m.key, d)          # same bucket geometry: identical up to rounding
        ref = fp64_reference(m)
        err = np.linalg.norm((m.u - ref).ravel()) / np.linalg.norm(ref.ravel())
        assert err < 1e-6, (m.key, err)
    st = serve.latency_stats(mixed)
    assert st["p99_ms"] >= st["p50_ms"] > 0
