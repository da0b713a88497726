"""NumPy-facing 2D square-lattice solves on the GPU (matrix-free replacements for the solve entry points of
coarse2d/lin2d.py, timing/t2d/solver2d.py and timing/t2d/cg2plain.py).

  Lattice2D(kind="square", nx, ny, h, origin, active)   .kmv, .stress, .energy_per_particle   (lin2d.py:29-163)
  solve_mf(lat, Kn, Tv, fixed_dofs, u_fixed, tol, maxit, precond)   per-DOF mask CG / 2x2 block-Jacobi PCG
      (cg2plain.cg_mf + solve_cg, solver2d.pcg_mf + solve_mf; stopping rule |r| <= tol |b|, initial test included)
  solve_mixed(lat, Kn, Tv, fixed_dofs, u_fixed, tol)                FP32 CG + FP64 refinement
The assembled-matrix path (lin2d.stiffness + solve_disp via SuperLU) is direct-solver code outside the matrix-free hot
path and is not provided.
"""
import numpy as np
import torch

from . import core
from .geom import (SQ_OFFS, SQ_SHELL, affine_disp, bond_params_two_end_mean, iso_C2d as iso_C,  # noqa: F401
                   square_params_from_C)
from .geom import Lattice2D as _GeomLattice2D
from .lin3d import _dev, _t

_F64 = torch.float64


class Lattice2D(_GeomLattice2D):
    """Square lattice geometry with GPU kernels."""

    def __init__(self, kind, nx, ny, h, origin=(0.0, 0.0), active=None):
        super().__init__(kind, nx, ny, h, origin, active)
        self._dl = None

    @property
    def device_lattice(self):
        if self._dl is None:
            self._dl = core.DeviceLattice(self, _dev())
        return self._dl

    def kmv(self, u, Kn, Tv):
        """K u (2N,), the exact Hessian of sum_i U_i (solver2d._kmv)."""
        return core.kmv(self.device_lattice, _t(u).reshape(self.N, 2), _t(Kn), _t(Tv)).cpu().numpy().ravel()

    def stress(self, u, Kn, Tv):
        """Particle stress (N, 3) xx yy xy (lin2d.Lattice2D.stress for an intact lattice)."""
        return core.stress(self.device_lattice, _t(u).reshape(self.N, 2), _t(Kn), _t(Tv)).cpu().numpy()

    def energy_per_particle(self, u, Kn, Tv):
        return core.energy(self.device_lattice, _t(u).reshape(self.N, 2), _t(Kn), _t(Tv)).cpu().numpy()


def _prep(lat, Kn, Tv, fixed_dofs, u_fixed):
    if not isinstance(lat, Lattice2D):
        l2 = Lattice2D.__new__(Lattice2D)
        l2.__dict__.update(lat.__dict__)
        l2._dl = None
        lat = l2
    n = 2 * lat.N
    fixed = np.zeros(n, bool)
    fixed[np.asarray(fixed_dofs)] = True
    ub = np.zeros(n)
    ub[np.asarray(fixed_dofs)] = u_fixed
    dl = lat.device_lattice
    Kt, Tt = _t(Kn), _t(Tv)
    free = _t(~fixed).reshape(lat.N, 2)
    b = -core.kmv(dl, _t(ub).reshape(lat.N, 2), Kt, Tt) * free
    return lat, dl, Kt, Tt, free, b, ub


def solve_mf(lat, Kn, Tv, fixed_dofs, u_fixed, tol=1e-10, maxit=200000, precond=False):
    """u (2N,) with prescribed DOFs and K_ff u_f = -K_fp u_p.  Returns (u, dict(iters, relres, status))."""
    lat, dl, Kt, Tt, free, b, ub = _prep(lat, Kn, Tv, fixed_dofs, u_fixed)
    Minv = core.block_jacobi(dl, Kt, Tt, _F64) if precond else None
    x, info = core.cg(dl, Kt, Tt, b, Minv=Minv, free=free, tol=tol, maxit=maxit, check=1, precheck=True)
    return ub + x.cpu().numpy().ravel(), dict(iters=int(info.iters[0]), relres=float(info.relres[0]),
                                               status=int(info.status[0]))


def solve_mixed(lat, Kn, Tv, fixed_dofs, u_fixed, tol=1e-10, inner_tol=1e-3, maxit=200000, precond=False):
    """The same problem with FP32 (P)CG inside FP64 iterative refinement (FP64 true residual <= tol)."""
    lat, dl, Kt, Tt, free, b, ub = _prep(lat, Kn, Tv, fixed_dofs, u_fixed)
    x, info = core.ir(dl, Kt, Tt, b, free=free, tol=tol, inner_tol=inner_tol, maxit=maxit, precond=precond)
    return ub + x.cpu().numpy().ravel(), dict(iters=int(info.iters[0]), relres=float(info.relres[0]),
                                               status=int(info.status[0]), outer=info.outer)
