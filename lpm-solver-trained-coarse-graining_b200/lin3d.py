"""NumPy-facing 3D SC solve on the GPU (drop-in for the solver entry points of coarse3d/lin3d.py and
timing/t3d/cgplain.py).

Arrays come in and go out as NumPy (as with the reference's Numba kernels); the work runs in liblpm_b200.so on the
current CUDA device.

  Lattice3D(nx, ny, nz, h, origin, active)   .apply, .stress, .energy_per_particle, .block_diag   (lin3d.py:29-51)
  solve_pcg(lat, Kn, Tv, fixed, u_presc, tol, maxit, M, x0)   block-Jacobi PCG            (lin3d.py:521-532)
  solve_cg(lat, Kn, Tv, fixed, u_presc, tol, maxit)            plain CG                     (cgplain.py:11-55)
  solve_mixed(lat, Kn, Tv, fixed, u_presc, tol)                FP32 PCG + FP64 refinement
The assembled-matrix paths of the reference (CSR assembly, SuperLU solve_direct) are direct-solver code outside the
matrix-free hot path and are not provided.
"""
import numpy as np
import torch

from . import _lib
from . import core
from .geom import (DIR_OF_SLOT, FWD_SLOTS, LOADS, NSLOT, SC_OFFS, SC_SHELL, VOIGT_PAIRS, LatticeGeom,  # noqa: F401
                   affine_disp, bond_params_two_end_mean, iso_C, sc_params_from_C, unit_strain)

_F64 = torch.float64


def _dev():
    if not torch.cuda.is_available():
        raise _lib.LPMError("lin3d runs on the GPU; no CUDA device is available (there is no CPU fallback)")
    return torch.device("cuda", torch.cuda.current_device())


def _t(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=_dev())


class Lattice3D(LatticeGeom):
    """SC lattice geometry (geom.LatticeGeom) with GPU kernels (coarse3d/lin3d.py:29-51)."""

    def __init__(self, nx, ny, nz, h=1.0, origin=(0.0, 0.0, 0.0), active=None):
        super().__init__(nx, ny, nz, h, origin, active)
        self._dl = None

    @property
    def device_lattice(self):
        if self._dl is None:
            self._dl = core.DeviceLattice(self, _dev())
        return self._dl

    def apply(self, u, Kn, Tv):
        return core.kmv(self.device_lattice, _t(u).reshape(self.N, 3), _t(Kn), _t(Tv)).cpu().numpy()

    def stress(self, u, Kn, Tv):
        """computeStress(): (N, 6) in the code order xx, yy, zz, yz, xz, xy."""
        return core.stress(self.device_lattice, _t(u).reshape(self.N, 3), _t(Kn), _t(Tv)).cpu().numpy()

    def energy_per_particle(self, u, Kn, Tv):
        return core.energy(self.device_lattice, _t(u).reshape(self.N, 3), _t(Kn), _t(Tv)).cpu().numpy()

    def block_diag(self, Kn, Tv):
        _, D = core.block_jacobi(self.device_lattice, _t(Kn), _t(Tv), _F64, want_D=True)
        return D[0].cpu().numpy()


def _as_lattice(lat):
    if isinstance(lat, Lattice3D):
        return lat
    full = Lattice3D.__new__(Lattice3D)
    full.__dict__.update(lat.__dict__)
    full._dl = None
    return full


def _solve(lat, Kn, Tv, fixed, u_presc, tol, maxit, precond, M=None, x0=None):
    lat = _as_lattice(lat)
    dl = lat.device_lattice
    free = ~np.asarray(fixed, bool)
    up = np.zeros((lat.N, 3))
    up[~free] = np.asarray(u_presc, float).reshape(lat.N, 3)[~free]
    Kt, Tt = _t(Kn), _t(Tv)
    b = -core.kmv(dl, _t(up), Kt, Tt) * _t(free)[:, None]
    Minv = None
    if precond:
        Minv = _t(M).reshape(1, lat.N, 3, 3) if M is not None else core.block_jacobi(dl, Kt, Tt, _F64)
    x0t = None if x0 is None else _t(np.where(free[:, None], x0, 0.0))
    layout, Kc, Tc = _lib.LAYOUT_REF, Kt, Tt
    if lat.full:
        layout, Kc, Tc = _lib.LAYOUT_SOA, core.pack(Kt[None], _F64), core.pack(Tt[None], _F64)
    x, info = core.cg(dl, Kc, Tc, b[None], x=None if x0t is None else x0t[None], Minv=Minv, free=_t(free)[None],
                      tol=tol, maxit=maxit, check=1, layout=layout, rhs_per_set=1)
    return up + x[0].cpu().numpy(), dict(iters=int(info.iters[0]), relres=float(info.relres[0]),
                                          status=int(info.status[0]))


def solve_pcg(lat, Kn, Tv, fixed, u_presc, tol=1e-10, maxit=20000, M=None, x0=None):
    """u with u = u_presc on fixed particles and K_ff u_f = -K_fp u_p, block-Jacobi PCG stopped when
    |r| <= tol |b| (tested every iteration).  Returns (u (N, 3), dict(iters, relres, status))."""
    return _solve(lat, Kn, Tv, fixed, u_presc, tol, maxit, True, M, x0)


def solve_cg(lat, Kn, Tv, fixed, u_presc, tol=1e-4, maxit=200000):
    """The same problem by unpreconditioned CG from zero (the solverCG algorithm of timing/t3d/cgplain.py)."""
    return _solve(lat, Kn, Tv, fixed, u_presc, tol, maxit, False)


def solve_mixed(lat, Kn, Tv, fixed, u_presc, tol=1e-8, inner_tol=1e-3, maxit=20000):
    """The same problem with FP32 block-Jacobi PCG inside FP64 iterative refinement (FP64 true residual <= tol)."""
    lat = _as_lattice(lat)
    dl = lat.device_lattice
    free = ~np.asarray(fixed, bool)
    up = np.zeros((lat.N, 3))
    up[~free] = np.asarray(u_presc, float).reshape(lat.N, 3)[~free]
    Kt, Tt = _t(Kn), _t(Tv)
    b = -core.kmv(dl, _t(up), Kt, Tt) * _t(free)[:, None]
    x, info = core.ir(dl, Kt, Tt, b, free=_t(free), tol=tol, inner_tol=inner_tol, maxit=maxit)
    return up + x.cpu().numpy(), dict(iters=int(info.iters[0]), relres=float(info.relres[0]),
                                      status=int(info.status[0]), outer=info.outer)
