"""Batched, differentiable linearised 3D SC LPM on the B200 CUDA library (drop-in for coarse3d/torch_lpm3d.py).

Same operator, stress, energy and boundary conditions as the reference (coarse3d/torch_lpm3d.py:36-263); every
operator evaluation, preconditioner, solve, gradient and adjoint runs in liblpm_b200.so kernels:

  SCT(lat, device, dtype)   .apply / .stress / .energy (autograd-capable), .block_diag, .precond, .pcg, .solve
  LinSolve.apply(Kn, Tv, op, up, free, tol)   forward PCG, backward adjoint PCG + per-bond gradient kernel
  LoadSet, CoarseT(nc, s, ...).run(Kn, Tv, tol, differentiable), FineRefT(n, s, ...).run(Kn, Tv, tol)

Shapes follow the reference: u (..., N, 3); Kn, Tv (..., N, 18) broadcast against u's leading dimensions; free
(..., N) float.  The VJPs of apply / stress / energy are exact for any bond parameters; LinSolve's adjoint assumes
symmetric bond parameters, as the reference's own adjoint does (K symmetric).  There is no CPU path: CPU tensors raise.
"""
import numpy as np
import torch

from . import core
from . import geom as G
from .operator import LatticeOperator, LinSolve, inv3  # noqa: F401

_F64 = torch.float64


class SCT(LatticeOperator):
    """Matrix-free SC operator on a fixed lattice geometry (geom.LatticeGeom) (coarse3d/torch_lpm3d.py:36-148)."""

    def __init__(self, lat, device="cuda", dtype=_F64):
        if lat.dim != 3:
            raise ValueError("SCT needs a simple-cubic lattice")
        super().__init__(lat, device, dtype)


# ---------------------------------------------------------------------------------------------------------------
# coarse model with the load cases (training / evaluation) and the fine reference (data generation)
# ---------------------------------------------------------------------------------------------------------------
class LoadSet:
    """BCs of the load cases on a lattice whose particles belong to blocks IJK (coarse3d/torch_lpm3d.py:181-194)."""

    def __init__(self, lat, IJK, nc, s, h, device, dtype, loads=G.LOADS):
        self.loads = loads
        fr, ups, mov = [], [], []
        for ld in loads:
            fixed, up, moving = G.prescribed(ld, lat.x, IJK, nc, s, h)
            fr.append(~fixed)
            ups.append(up)
            mov.append(np.zeros(lat.N, bool) if moving is None else moving)
        self.free = torch.as_tensor(np.array(fr), device=device, dtype=dtype)
        self.up = torch.as_tensor(np.array(ups), device=device, dtype=dtype)
        self.moving = torch.as_tensor(np.array(mov), device=device, dtype=dtype)


def _gdir(ld):
    return G.GDIR.get(ld, G.GDIR_EXTRA.get(ld))


class CoarseT:
    """Coarse SC model: nc^3 particles at the block centres, spacing s h (coarse3d/torch_lpm3d.py:197-227)."""

    def __init__(self, nc, s, h=1.0, device="cuda", dtype=_F64, loads=G.LOADS):
        self.nc, self.s, self.h = nc, s, h
        self.lat = G.LatticeGeom(nc, nc, nc, s * h)
        self.op = SCT(self.lat, device, dtype)
        self.N = self.lat.N
        self.loads = loads
        self.bc = LoadSet(self.lat, self.lat.ijk, (nc, nc, nc), s, h, device, dtype, loads)
        self.freecell = self.bc.free.bool()
        surf = [G.free_surface_cells(ld, (nc, nc, nc)) if _gdir(ld) is not None else np.zeros(self.N, bool)
                for ld in loads]
        self.surf = torch.as_tensor(np.array(surf), device=device)
        self.V = (s * h) ** 3

    def run(self, Kn, Tv, tol=1e-10, differentiable=True):
        """Kn, Tv (B, N, 18) -> dict u (B,L,N,3), sig (B,L,N,6), w (B,L,N) energy density, F (B,L) reaction."""
        Kn4, Tv4 = Kn[:, None], Tv[:, None]
        B = Kn.shape[0]
        up, free = self.bc.up[None], self.bc.free[None]
        if differentiable:
            u = LinSolve.apply(Kn4, Tv4, self.op, up.expand(B, -1, -1, -1), free.expand(B, -1, -1), tol)
        else:
            with torch.no_grad():
                u, _, _ = self.op.solve(Kn4, Tv4, up.expand(B, -1, -1, -1), free.expand(B, -1, -1), tol)
        sig = self.op.stress(u, Kn4, Tv4)
        w = self.op.energy(u, Kn4, Tv4) / self.V
        P = self.op.apply(u, Kn4, Tv4)
        F = torch.stack([(P[:, l, :, _gdir(ld)] * self.bc.moving[l]).sum(-1) if _gdir(ld) is not None
                         else torch.zeros(B, device=Kn.device, dtype=Kn.dtype) for l, ld in enumerate(self.loads)], 1)
        return dict(u=u, sig=sig, w=w, F=F)


class FineRefT:
    """Fine reference for an n^3 voxel box and block size s: block means of u, stress, energy density and grip
    reactions for the load cases, all samples of a batch at once (coarse3d/torch_lpm3d.py:230-263).

    precision="fp64" runs the reference's FP64 block-Jacobi PCG; "mixed" runs FP32 PCG inside FP64 refinement to the
    same FP64 true-residual tolerance; "amg" the same refinement with the aggregation-AMG preconditioner."""

    def __init__(self, n, s, h=1.0, device="cuda", dtype=_F64, loads=G.LOADS, precision="fp64"):
        self.n, self.s, self.h = n, s, h
        self.nc = n // s
        self.lat = G.LatticeGeom(n, n, n, h)
        self.op = SCT(self.lat, device, dtype)
        IJK = self.lat.ijk // s
        self.bc = LoadSet(self.lat, IJK, (self.nc,) * 3, s, h, device, dtype, loads)
        self.loads = loads
        cid = (IJK[:, 2] * self.nc + IJK[:, 1]) * self.nc + IJK[:, 0]
        self.cid = torch.as_tensor(cid, device=device)
        self.Nc = self.nc ** 3
        self.precision = precision

    def bmean(self, f):
        out = torch.zeros(f.shape[:-2] + (self.Nc, f.shape[-1]), device=f.device, dtype=f.dtype)
        out.index_add_(f.dim() - 2, self.cid, f)
        return out / self.s ** 3

    @torch.no_grad()
    def run(self, Kn, Tv, tol=1e-10):
        Kn4, Tv4 = Kn[:, None], Tv[:, None]
        B = Kn.shape[0]
        up = self.bc.up[None].expand(B, -1, -1, -1)
        free = self.bc.free[None].expand(B, -1, -1)
        if self.precision in ("mixed", "amg"):
            solve = self.op.solve_mixed if self.precision == "mixed" else self.op.solve_amg
            u, info = solve(Kn4, Tv4, up, free, tol=tol)
            it, rel = int(info.iters.max()), float(info.relres.max())
        else:
            u, it, rel = self.op.solve(Kn4, Tv4, up, free, tol)
        sig = self.op.stress(u, Kn4, Tv4)
        U = self.op.energy(u, Kn4, Tv4)
        P = self.op.apply(u, Kn4, Tv4)
        F = torch.stack([(P[:, l, :, _gdir(ld)] * self.bc.moving[l]).sum(-1) if _gdir(ld) is not None
                         else torch.zeros(B, device=Kn.device, dtype=Kn.dtype) for l, ld in enumerate(self.loads)], 1)
        return dict(u=self.bmean(u), sig=self.bmean(sig), w=self.bmean(U[..., None])[..., 0] / self.h ** 3,
                    F=F, iters=it, relres=rel)
