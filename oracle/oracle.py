"""CPU oracle of the LPM linear solve -- TEST INFRASTRUCTURE ONLY.

NumPy front end over ``oracle/lpm_oracle.c`` (FP64, OpenMP), a restatement of the reference's Numba kernels and CPU
solvers.  Used by ``tests/`` (as the checker of the CUDA library), ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py``.  The product path never imports this module.

Parity of the oracle itself is pinned in ``tests/test_oracle.py`` against golden vectors produced by the reference
(``tests/golden/make_golden.py``).
"""
import ctypes
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import build as _build  # noqa: E402

_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_int64)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_I64 = ctypes.c_int64


def lib():
    global _lib
    if _lib is None:
        path = _build.build(quiet=True)
        L = ctypes.CDLL(path)
        sig = {
            "orc_set_threads": [ctypes.c_int],
            "orc_get_threads": [],
            "orc_sc_shell_sums": [_I64, _L, _D, _D, _D, _D, _D],
            "orc_sc_bond_forces": [_I64, _L, _D, _D, _D, _D, _D, _D],
            "orc_sc_apply": [_I64, _L, _D, _D, _D, _D, _D],
            "orc_sc_stress": [_I64, _L, _D, _D, _D, _D, ctypes.c_double, _D, _D],
            "orc_sc_energy": [_I64, _L, _D, _D, _D, _D, _D],
            "orc_sc_block_diag": [_I64, _L, _D, _D, _D, _D],
            "orc_block_jacobi3": [_I64, _D, _U8, _D],
            "orc_sc_pcg": [_I64, _L, _D, _D, _D, _D, _U8, _D, _D, ctypes.c_double, ctypes.c_int, _D],
            "orc_sc_cg": [_I64, _L, _D, _D, _D, _U8, _D, _D, ctypes.c_double, ctypes.c_int, _D],
            "orc_sc_grad": [_I64, _L, _D, _D, _D, _D, _D, _D, _D],
            "orc_sq_kmv": [_I64, _L, _D, _D, _D, _D, _D, _D],
            "orc_sq_diag_inv": [_I64, _L, _D, _D, _D, _U8, _D],
            "orc_sq_pcg_mf": [_I64, _L, _D, _D, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_int, _D],
            "orc_sq_cg_mf": [_I64, _L, _D, _D, _D, _D, _D, _D, ctypes.c_double, ctypes.c_int, _D],
            "orc_sq_stress": [_I64, _L, _D, _D, _D, _D, ctypes.c_double, _D, _D],
            "orc_sq_energy": [_I64, _L, _D, _D, _D, _D, _D],
            "orc_sq_grad": [_I64, _L, _D, _D, _D, _D, _D],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int if name in ("orc_sc_pcg", "orc_sc_cg", "orc_sq_pcg_mf", "orc_sq_cg_mf",
                                                  "orc_get_threads") else None
        _lib = L
    return _lib


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return int(lib().orc_get_threads())


def _d(a):
    return a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _nbr(lat):
    return np.ascontiguousarray(lat.nbr, dtype=np.int64)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


# ---------------------------------------------------------------------------------------------------------------- 3D
def sc_apply(lat, u, Kn, Tv):
    """K u (N, 3) -- coarse3d/lin3d.py:126-149."""
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(lat.N, 3)
    out = np.empty((lat.N, 3))
    lib().orc_sc_apply(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(u), _d(out))
    return out


def sc_shell_sums(lat, u, Tv):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    S, TS = np.empty((lat.N, 2)), np.empty((lat.N, 2))
    u, Tv = _f64(u).reshape(lat.N, 3), _f64(Tv)
    lib().orc_sc_shell_sums(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Tv), _d(u), _d(S), _d(TS))
    return S, TS


def sc_bond_forces(lat, u, Kn, Tv):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(lat.N, 3)
    dL, F = np.empty((lat.N, 18)), np.empty((lat.N, 18))
    lib().orc_sc_bond_forces(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(u), _d(dL), _d(F))
    return dL, F


def sc_stress(lat, u, Kn, Tv):
    nbr, nd, l0 = _nbr(lat), _f64(lat.ndir), _f64(lat.l0)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(lat.N, 3)
    out = np.empty((lat.N, 6))
    lib().orc_sc_stress(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(l0), _d(Kn), _d(Tv), float(lat.V), _d(u), _d(out))
    return out


def sc_energy(lat, u, Kn, Tv):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(lat.N, 3)
    out = np.empty(lat.N)
    lib().orc_sc_energy(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(u), _d(out))
    return out


def sc_block_diag(lat, Kn, Tv):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv = _f64(Kn), _f64(Tv)
    D = np.empty((lat.N, 3, 3))
    lib().orc_sc_block_diag(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(D))
    return D


def block_jacobi3(D, free):
    D = _f64(D)
    fr = _u8(free)
    M = np.empty_like(D)
    lib().orc_block_jacobi3(len(D), _d(D), fr.ctypes.data_as(_U8), _d(M))
    return M


def sc_pcg(lat, Kn, Tv, M, free, b, x, tol, maxit):
    """In-place block-Jacobi PCG (coarse3d/lin3d.py:464-518).  Returns (iters, relres)."""
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    Kn, Tv, M, b, fr = _f64(Kn), _f64(Tv), _f64(M), _f64(b), _u8(free)
    rel = ctypes.c_double(0.0)
    it = lib().orc_sc_pcg(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(M), fr.ctypes.data_as(_U8),
                          _d(b), _d(x), float(tol), int(maxit), ctypes.byref(rel))
    return it, rel.value


def sc_cg(lat, Kn, Tv, free, b, x, tol, maxit):
    """In-place plain CG (timing/t3d/cgplain.py:11-55).  Returns (iters, relres)."""
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    Kn, Tv, b, fr = _f64(Kn), _f64(Tv), _f64(b), _u8(free)
    rel = ctypes.c_double(0.0)
    it = lib().orc_sc_cg(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), fr.ctypes.data_as(_U8), _d(b), _d(x),
                         float(tol), int(maxit), ctypes.byref(rel))
    return it, rel.value


def sc_grad(lat, Kn, Tv, u, lam):
    """Positive per-slot derivatives of lam . K u w.r.t. Kn, Tv (code-force operator)."""
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, u, lam = _f64(Kn), _f64(Tv), _f64(u).reshape(lat.N, 3), _f64(lam).reshape(lat.N, 3)
    gK, gT = np.empty((lat.N, 18)), np.empty((lat.N, 18))
    lib().orc_sc_grad(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(u), _d(lam), _d(gK), _d(gT))
    return gK, gT


def solve_pcg(lat, Kn, Tv, fixed, u_presc, tol=1e-10, maxit=20000, M=None, x0=None, precond=True):
    """Mirror of coarse3d/lin3d.py:521-532 (precond=False: the plain CG of timing/t3d/cgplain.py)."""
    free = ~np.asarray(fixed, bool)
    up = np.zeros((lat.N, 3))
    up[~free] = np.asarray(u_presc)[~free]
    b = -sc_apply(lat, up, Kn, Tv)
    b[~free] = 0.0
    x = np.zeros((lat.N, 3)) if x0 is None else np.ascontiguousarray(np.where(free[:, None], x0, 0.0))
    if precond:
        if M is None:
            M = block_jacobi3(sc_block_diag(lat, Kn, Tv), free)
        it, rr = sc_pcg(lat, Kn, Tv, M, free, b, x, tol, maxit)
    else:
        it, rr = sc_cg(lat, Kn, Tv, free, b, x, tol, maxit)
    return up + x, dict(iters=int(it), relres=float(rr))


# ---------------------------------------------------------------------------------------------------------------- 2D
def sq_kmv(lat, u, Kn, Tv):
    """K u (2N,) -- timing/t2d/solver2d.py:269-305."""
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(-1)
    g, f = np.zeros((lat.N, 8)), np.empty(2 * lat.N)
    lib().orc_sq_kmv(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(u), _d(g), _d(f))
    return f


def sq_diag_inv(lat, Kn, Tv, fixed):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, fx = _f64(Kn), _f64(Tv), _u8(fixed)
    B = np.empty((lat.N, 2, 2))
    lib().orc_sq_diag_inv(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), fx.ctypes.data_as(_U8), _d(B))
    return B


def sq_cg_mf(lat, Kn, Tv, mask, b, x, tol, maxit):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    Kn, Tv, mask, b = _f64(Kn), _f64(Tv), _f64(mask).reshape(-1), _f64(b).reshape(-1)
    rel = ctypes.c_double(0.0)
    it = lib().orc_sq_cg_mf(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(mask), _d(b), _d(x), float(tol),
                            int(maxit), ctypes.byref(rel))
    return it, rel.value


def sq_pcg_mf(lat, Kn, Tv, Binv, mask, b, x, tol, maxit):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    assert x.dtype == np.float64 and x.flags.c_contiguous
    Kn, Tv, Binv, mask, b = _f64(Kn), _f64(Tv), _f64(Binv), _f64(mask).reshape(-1), _f64(b).reshape(-1)
    rel = ctypes.c_double(0.0)
    it = lib().orc_sq_pcg_mf(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(Binv), _d(mask), _d(b), _d(x),
                             float(tol), int(maxit), ctypes.byref(rel))
    return it, rel.value


def sq_stress(lat, u, Kn, Tv):
    nbr, nd, l0 = _nbr(lat), _f64(lat.ndir), _f64(lat.l0)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(-1)
    out = np.empty((lat.N, 3))
    lib().orc_sq_stress(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(l0), _d(Kn), _d(Tv), float(lat.V), _d(u), _d(out))
    return out


def sq_energy(lat, u, Kn, Tv):
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    Kn, Tv, u = _f64(Kn), _f64(Tv), _f64(u).reshape(-1)
    out = np.empty(lat.N)
    lib().orc_sq_energy(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(Kn), _d(Tv), _d(u), _d(out))
    return out


def sq_grad(lat, u, lam):
    """Positive per-slot derivatives of lam^T K u w.r.t. Kn, Tv (exact-Hessian operator)."""
    nbr, nd = _nbr(lat), _f64(lat.ndir)
    u, lam = _f64(u).reshape(-1), _f64(lam).reshape(-1)
    gK, gT = np.empty((lat.N, 8)), np.empty((lat.N, 8))
    lib().orc_sq_grad(lat.N, nbr.ctypes.data_as(_L), _d(nd), _d(u), _d(lam), _d(gK), _d(gT))
    return gK, gT


def sq_solve_cg(lat, Kn, Tv, fixed_dof, u_presc, tol=1e-10, maxit=200000, precond=False):
    """Per-DOF-mask solve as timing/t2d/cg2plain.py:52-68 (precond=True: solver2d.pcg_mf with particle blocks)."""
    fd = np.asarray(fixed_dof, bool).reshape(-1)
    mask = (~fd).astype(np.float64)
    ub = np.where(fd, np.asarray(u_presc, float).reshape(-1), 0.0)
    b = -sq_kmv(lat, ub, Kn, Tv) * mask
    x = np.zeros(2 * lat.N)
    if precond:
        B = sq_diag_inv(lat, Kn, Tv, fd.reshape(-1, 2).any(1))
        it, rr = sq_pcg_mf(lat, Kn, Tv, B, mask, b, x, tol, maxit)
    else:
        it, rr = sq_cg_mf(lat, Kn, Tv, mask, b, x, tol, maxit)
    return (x + ub).reshape(-1, 2), dict(iters=int(it), relres=float(rr))
