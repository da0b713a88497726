"""The assembled-matrix 2D solve (lin2d.solve_disp, coarse2d/lin2d.py:166-180) through its own signature: the CSR K
probed from the GPU operator equals the reference's assembled stiffness (golden K u), and the device Jacobi-PCG gives
the reference's SuperLU displacements (golden lu_u) and SciPy SuperLU's answers for further loads, an external force
and a reused cache.  Bar: 1e-9 relative (CG to 1e-12 against a direct solve)."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

from conftest import relmax
from lpm_b200 import lin2d

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def superlu(K, fdofs, ufix, f_ext=None):
    n = K.shape[0]
    fixed = np.zeros(n, bool)
    fixed[fdofs] = True
    u = np.zeros(n)
    u[fdofs] = ufix
    rhs = -K[~fixed][:, fixed] @ u[fixed]
    if f_ext is not None:
        rhs = rhs + f_ext[~fixed]
    u[~fixed] = spla.splu(K[~fixed][:, ~fixed].tocsc()).solve(rhs)
    return u


def test_stiffness_matches_reference_assembly(gsq):
    lat = lin2d.Lattice2D("square", 16, 12, 1.0)
    K, B, H = lat.stiffness(gsq["Kn_ns"], gsq["Tv_ns"])
    assert K.shape == (2 * lat.N, 2 * lat.N) and B is None and H is None
    assert relmax(K @ gsq["u"], gsq["Ku_csr_ns"]) < 1e-13


def test_solve_disp_matches_superlu(gsq):
    lat = lin2d.Lattice2D("square", 16, 12, 1.0)
    K, _, _ = lat.stiffness(gsq["Kn"], gsq["Tv"])
    fd = gsq["cg_fixed"].ravel()
    fdofs = np.nonzero(fd)[0]
    ub = gsq["cg_up"].ravel()
    u, cache = lin2d.solve_disp(K, fdofs, ub[fdofs])
    assert rel_l2(u, gsq["lu_u"]) < 1e-9
    assert np.array_equal(u[fdofs], ub[fdofs])
    # a second load on the same K and fixed set through the returned cache, and an external force
    rng = np.random.default_rng(3)
    uf2 = rng.standard_normal(fdofs.size) * 1e-3
    f_ext = rng.standard_normal(K.shape[0]) * 1e-4
    u2, cache2 = lin2d.solve_disp(K, fdofs, uf2, f_ext=f_ext, lu_cache=cache)
    assert cache2 is cache
    assert rel_l2(u2, superlu(K, fdofs, uf2, f_ext)) < 1e-9


def test_solve_disp_larger_lattice():
    """A 64 x 48 two-phase lattice, particle-fixed left column and pulled right column (the 2D fine-reference
    pattern of coarse2d/cg.py:64-76)."""
    from lpm_b200 import micro
    nx, ny = 64, 48
    lat = lin2d.Lattice2D("square", nx, ny, 1.0)
    ph = micro.grf_two_phase(nx, ny, 6.0, 0.3, 2)
    C = lin2d.iso_C(np.where(ph == 1, 10.0, 1.0), 0.25, plane="stress")
    Kn, Tv = lin2d.bond_params_two_end_mean(lat, lin2d.square_params_from_C(C))
    K, _, _ = lat.stiffness(Kn, Tv)
    left, right = lat.ij[:, 0] == 0, lat.ij[:, 0] == nx - 1
    fp = np.flatnonzero(left | right)
    fdofs = np.concatenate([2 * fp, 2 * fp + 1])
    up = np.zeros((lat.N, 2))
    up[right, 0] = 1e-3 * (nx - 1)
    u, _ = lin2d.solve_disp(K, fdofs, up.ravel()[fdofs])
    assert rel_l2(u, superlu(K, fdofs, up.ravel()[fdofs])) < 1e-9
