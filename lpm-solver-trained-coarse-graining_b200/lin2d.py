"""NumPy-facing 2D square-lattice solves on the GPU (matrix-free replacements for the solve entry points of
coarse2d/lin2d.py, timing/t2d/solver2d.py and timing/t2d/cg2plain.py).

  Lattice2D(kind="square", nx, ny, h, origin, active)   .kmv, .stress, .energy_per_particle   (lin2d.py:29-163)
  solve_mf(lat, Kn, Tv, fixed_dofs, u_fixed, tol, maxit, precond)   per-DOF mask CG / 2x2 block-Jacobi PCG
      (cg2plain.cg_mf + solve_cg, solver2d.pcg_mf + solve_mf; stopping rule |r| <= tol |b|, initial test included)
  solve_mixed(lat, Kn, Tv, fixed_dofs, u_fixed, tol)                FP32 CG + FP64 refinement
  Lattice2D.stiffness(Kn, Tv) -> (K, None, None)   assembled SciPy CSR K (lin2d.py:113-118), probed from the GPU operator
  solve_disp(K, fixed_dofs, u_fixed, f_ext, lu_cache) -> (u, cache)   the assembled-matrix solve (lin2d.py:166-180):
      Jacobi-PCG on the device on the CSR of K instead of a SuperLU factorisation
"""
import ctypes

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib as L
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

    def stiffness(self, Kn, Tv, alive=None):
        """Assembled K (2N x 2N SciPy CSR, DOF 2p + a) of the exact-Hessian operator, as lin2d.Lattice2D.stiffness.

        The operator couples particles at most two sites apart in each direction, so the 25 residue classes of
        (i mod 5, j mod 5) times the 2 components give 50 probe vectors that each meet one column per row: one batched
        FP64 K.u of 50 systems on the GPU, scattered into the 5 x 5 stencil pattern on the host.  The reference also
        returns its bond matrix B and bond Hessian H (used by the fracture scripts, outside this path); they are not
        formed here and come back as None.  `alive` (bond deletion) belongs to the fracture path and is not supported.
        """
        if alive is not None:
            raise NotImplementedError("bond deletion (alive) is part of the fracture scripts, not of the solve path")
        N, nx, ny = self.N, self.nx, self.ny
        ii, jj = self.ij[:, 0], self.ij[:, 1]
        colour = (ii % 5) + 5 * (jj % 5)
        probes = np.zeros((50, N, 2))
        for a in range(2):
            probes[colour * 2 + a, np.arange(N), a] = 1.0
        Y = core.kmv(self.device_lattice, _t(probes), _t(Kn), _t(Tv)).cpu().numpy()     # (50, N, 2), one set
        rows, cols, vals = [], [], []
        for dy in range(-2, 3):
            for dx in range(-2, 3):
                qi, qj = ii + dx, jj + dy
                inside = (qi >= 0) & (qi < nx) & (qj >= 0) & (qj < ny)
                q = self.site_of[np.where(inside, qj * nx + qi, 0)]
                ok = inside & (q >= 0)
                p = np.flatnonzero(ok)
                q = q[ok]
                cq = colour[q]
                for a in range(2):          # column DOF 2q + a
                    for b in range(2):      # row DOF 2p + b
                        rows.append(2 * p + b)
                        cols.append(2 * q + a)
                        vals.append(Y[cq * 2 + a, p, b])
        rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
        keep = vals != 0.0
        K = sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(2 * N, 2 * N))
        K.sort_indices()
        return K, None, None


class CsrSystem:
    """Device copy of an assembled K (CSR) for solve_disp; it plays the role of the reference's SuperLU factor
    (`lu_cache`): passing it back with the same K skips the upload."""

    def __init__(self, K, device):
        K = sp.csr_matrix(K)
        K.sort_indices()
        self.shape, self.nnz = K.shape, K.nnz
        self.rowptr = torch.as_tensor(K.indptr.astype(np.int64), device=device)
        self.col = torch.as_tensor(K.indices.astype(np.int32), device=device)
        self.val = torch.as_tensor(K.data.astype(np.float64), device=device)
        self.device = device
        self.last = None       # (iters, relres, status) of the last solve

    def matches(self, K):
        return tuple(K.shape) == tuple(self.shape) and K.nnz == self.nnz

    def solve(self, b, mask, tol=1e-12, maxit=None, poll=32):
        """x with K_ff x_f = b_f (b, mask: length-n host arrays); zero on fixed rows."""
        n = self.shape[0]
        lib = L.load()
        bd = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float64), device=self.device)
        md = torch.as_tensor(np.ascontiguousarray(mask, dtype=np.uint8), device=self.device)
        x = torch.empty(n, dtype=torch.float64, device=self.device)
        ws = core._scratch(lib.lpm_csr_workspace_bytes(n), self.device)
        it = torch.zeros(1, dtype=torch.int32, device=self.device)
        rel = torch.zeros(1, dtype=torch.float64, device=self.device)
        st = torch.zeros(1, dtype=torch.int32, device=self.device)
        opts = L.CgOpts(float(tol), int(maxit if maxit is not None else 10 * n), 1, int(poll), 0, None, None, 0, 0)
        L.check(lib.lpm_csr_pcg_f64(n, L.ptr(self.rowptr), L.ptr(self.col), L.ptr(self.val), L.ptr(md), L.ptr(bd),
                                    L.ptr(x), ctypes.byref(opts), L.ptr(ws), ws.numel(), L.ptr(it), L.ptr(rel),
                                    L.ptr(st), L.stream_ptr(self.device)), "lpm_csr_pcg_f64")
        self.last = (int(it.item()), float(rel.item()), int(st.item()))
        if self.last[2] == L.STATUS_BREAKDOWN:
            raise FloatingPointError("solve_disp: K_ff is not positive definite (CG breakdown)")
        return x.cpu().numpy()


def solve_disp(K, fixed_dofs, u_fixed, f_ext=None, lu_cache=None, tol=1e-12, maxit=None):
    """Solve K u = f with u prescribed on fixed_dofs (coarse2d/lin2d.py:166-180).  Returns (u (n,), cache).

    Same arguments and return contract as the reference: K is an assembled SciPy sparse matrix (2N x 2N), u_fixed
    the values on fixed_dofs, f_ext an optional external force on the free DOFs, and the returned cache is passed back
    to skip the set-up for the same K.  The reference factors K_ff with SuperLU; here K stays on the GPU as CSR and
    K_ff u_f = f_f - K_fp u_p is solved by FP64 Jacobi-PCG to |r| <= tol |b| (default 1e-12; SuperLU's answer is
    matched to about 1e-9 relative).  The right-hand side is formed on the host with one SciPy product, as the
    reference forms it.  Non-convergence within maxit (default 10 n) raises RuntimeError.
    """
    n = K.shape[0]
    fixed = np.zeros(n, bool)
    fixed[np.asarray(fixed_dofs)] = True
    u = np.zeros(n)
    u[np.asarray(fixed_dofs)] = u_fixed
    rhs = -(K @ u)
    if f_ext is not None:
        rhs = rhs + np.asarray(f_ext, dtype=np.float64)
    rhs[fixed] = 0.0
    dev = _dev()
    if lu_cache is None or not isinstance(lu_cache, CsrSystem) or not lu_cache.matches(K):
        lu_cache = CsrSystem(K, dev)
    x = lu_cache.solve(rhs, ~fixed, tol=tol, maxit=maxit)
    if lu_cache.last[2] != L.STATUS_OK:
        raise RuntimeError("solve_disp: CG did not reach %.1e in %d iterations (relres %.3e)"
                           % (tol, lu_cache.last[0], lu_cache.last[1]))
    u[~fixed] = x[~fixed]
    return u, lu_cache


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
