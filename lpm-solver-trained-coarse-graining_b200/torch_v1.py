"""Per-specimen voids on the B200 CUDA library (drop-in for cement3d/torch_v1.py: SCTV, CoarseTV, FineRefTV).

The lattice is the full n^3 grid and every specimen of a batch carries its own solid mask; a bond exists only if it is
geometric and both of its ends are solid (cement3d/torch_v1.py:37-45).  Void particles stay in the numbering, have no
bonds and are fixed at u = 0 by the models.  Shell sums run over existing bonds only, the stress uses the opp-flag
surface rule of the removed neighbours, and without a mask everything is the plain SC operator (SCT), bit for bit.

On the device each specimen's bond validity is an int32 bond table built by lpm_solid_nbr from its mask; the
specimen's operator calls (K u, stress, energy, their VJPs, block Jacobi, PCG, the adjoint and the per-bond gradient)
then run on the table kernels, one launch sequence per specimen.  Shapes follow the reference: u (B|1, L, N, 3);
Kn, Tv (B|1, 1, N, 18); free (B|1, L, N); solid (B, N) bool.
"""
import numpy as np
import torch

from . import core
from . import geom as G
from .operator import LatticeOperator, LinSolve
from .torch_lpm3d import SCT, LoadSet, _gdir

_F64 = torch.float64


def _nn6(ndir):
    """(18, 6) products n_a n_b in Voigt order xx yy zz yz xz xy."""
    pairs = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
    return torch.stack([ndir[:, a] * ndir[:, b] for a, b in pairs], 1)


class SCTV:
    """SC operator with per-specimen solid masks (cement3d/torch_v1.py:18-142)."""

    def __init__(self, lat, device="cuda", dtype=_F64):
        if lat.dim != 3 or not lat.full:
            raise ValueError("SCTV needs the full simple-cubic box (voids are given by the solid masks)")
        self.lat, self.dev, self.dt = lat, torch.device(device), dtype
        self.N = lat.N
        self.base = SCT(lat, device, dtype)
        self.dl = self.base.dl
        self.gvalid = torch.as_tensor(lat.valid, device=self.dev)
        self.ndir = torch.as_tensor(lat.ndir, device=self.dev, dtype=dtype)
        self.opp = torch.as_tensor(np.arange(18) ^ 1, device=self.dev)[None, :]
        self.l0 = torch.as_tensor(lat.l0, device=self.dev, dtype=dtype)
        self.Vp = lat.V
        self.nn6 = _nn6(self.ndir)
        self.d, self.NN = 3, 18
        self.set_mask(None)

    def set_mask(self, solid):
        """solid: None (no voids) or (B, N) bool.  Sets the per-specimen operators, valid (B|1, 1, N, 18), the
        stress weights stw and the shell normal sums s0, s1 (cement3d/torch_v1.py:37-52)."""
        if solid is None:
            self.ops = None
            v = self.gvalid[None, None]
        else:
            solid = torch.as_tensor(solid, device=self.dev).bool()
            tabs = core.solid_tables(self.lat, solid)
            self.ops = [LatticeOperator(self.lat, self.dev, self.dt, dl=core.DeviceLattice(self.lat, self.dev, tabs[b]))
                        for b in range(tabs.shape[0])]
            v = (tabs >= 0)[:, None]
        self.vb = v
        self.valid = v.to(self.dt)
        full = v.sum(-1, keepdim=True) == 18
        oppv = v[..., self.opp[0]]
        of = torch.where(full | oppv, torch.full_like(self.valid, 0.5), torch.ones_like(self.valid))
        self.stw = of / self.Vp * self.l0 * self.valid
        self.s0 = self.valid[..., :6] @ self.ndir[:6]
        self.s1 = self.valid[..., 6:] @ self.ndir[6:]

    # ---------------------------------------------------------------------------------------- dispatch
    def _each(self, fn, *args):
        """fn(op_b, *args_b) for every specimen b, where a tensor argument with a leading dimension of B is sliced to
        [b:b+1] and one with a leading 1 is passed whole; results are concatenated along dim 0."""
        B = len(self.ops)
        outs = []
        for b in range(B):
            ab = [a[b:b + 1] if isinstance(a, torch.Tensor) and a.dim() >= 3 and a.shape[0] == B else a
                  for a in args]
            outs.append(fn(self.ops[b], *ab))
        return outs

    def apply(self, u, Kn, Tv):
        if self.ops is None:
            return self.base.apply(u, Kn, Tv)
        return torch.cat(self._each(lambda op, uu, k, t: op.apply(uu, k, t), u, Kn, Tv), 0)

    def forces(self, u, Kn, Tv):
        raise NotImplementedError("per-bond forces are not formed on the device; use apply / stress / energy")

    def stress(self, u, Kn, Tv):
        if self.ops is None:
            return self.base.stress(u, Kn, Tv)
        return torch.cat(self._each(lambda op, uu, k, t: op.stress(uu, k, t), u, Kn, Tv), 0)

    def energy(self, u, Kn, Tv):
        if self.ops is None:
            return self.base.energy(u, Kn, Tv)
        return torch.cat(self._each(lambda op, uu, k, t: op.energy(uu, k, t), u, Kn, Tv), 0)

    def block_diag(self, Kn, Tv):
        if self.ops is None:
            return self.base.block_diag(Kn, Tv)
        return torch.cat(self._each(lambda op, k, t: op.block_diag(k, t), Kn, Tv), 0)

    def precond(self, Kn, Tv, free):
        """Block-Jacobi inverse, zero on fixed / void particles (cement3d/torch_v1.py:95-99)."""
        if self.ops is None:
            return self.base.precond(Kn, Tv, free)
        return torch.cat(self._each(lambda op, k, t, f: op.precond(k, t, f), Kn, Tv, free), 0)

    def bond_grad(self, u, lam, Kn, Tv):
        if self.ops is None:
            return self.base.bond_grad(u, lam, Kn, Tv)
        parts = self._each(lambda op, uu, ll, k, t: op.bond_grad(uu, ll, k, t), u, lam, Kn, Tv)
        return torch.cat([p[0] for p in parts], 0), torch.cat([p[1] for p in parts], 0)

    def _solve_sets(self, b, Kn, Tv, free, tol, maxit, check, x0=None, M=None):
        if self.ops is None:
            return self.base._solve_sets(b, Kn, Tv, free, tol, maxit, check, x0=x0, M=M)
        parts = self._each(lambda op, bb, k, t, f, xx, mm: op._solve_sets(bb, k, t, f, tol, maxit, check, x0=xx, M=mm),
                           b, Kn, Tv, free, x0, M)
        x = torch.cat([p[0] for p in parts], 0)
        info = core.SolveInfo(*(np.concatenate([getattr(p[1], f) for p in parts]) for f in ("iters", "relres",
                                                                                             "status")))
        return x, info

    def pcg(self, b, Kn, Tv, M, free, tol=1e-10, maxit=20000, x0=None, check=10):
        """Batched PCG with per-system freezing (cement3d/torch_v1.py:101-133).  Returns (x, iterations, max rel)."""
        with torch.no_grad():
            x, info = self._solve_sets(b, Kn, Tv, free, tol, maxit, check, x0=x0, M=M)
        info.raise_on_breakdown()
        self.last_iters = int(info.iters.max())
        return x, int(info.iters.max()), float(info.relres.max())

    def solve(self, Kn, Tv, up, free, tol=1e-10, maxit=20000, M=None):
        """u = up on fixed particles and (K u)_free = 0 (cement3d/torch_v1.py:135-141)."""
        with torch.no_grad():
            b = -self.apply(up, Kn, Tv) * free[..., None]
            x, it, rel = self.pcg(b, Kn, Tv, M, free, tol, maxit)
        return up + x, it, rel

    def solve_mixed(self, Kn, Tv, up, free, tol=1e-8, inner_tol=1e-3, maxit=20000):
        """FP32 PCG inside FP64 iterative refinement to |b - K x| <= tol |b|, per specimen.  Returns (u, SolveInfo)."""
        if self.ops is None:
            return self.base.solve_mixed(Kn, Tv, up, free, tol, inner_tol, maxit)
        parts = self._each(lambda op, k, t, uu, f: op.solve_mixed(k, t, uu, f, tol, inner_tol, maxit), Kn, Tv, up,
                           free)
        u = torch.cat([p[0] for p in parts], 0)
        info = core.SolveInfo(*(np.concatenate([getattr(p[1], f) for p in parts]) for f in ("iters", "relres",
                                                                                             "status")))
        return u, info


class CoarseTV:
    """Coarse SC model (nc^3 grid, spacing s h) with per-specimen cell masks (cement3d/torch_v1.py:145-186)."""

    def __init__(self, nc, s, h=1.0, device="cuda", dtype=_F64, loads=G.LOADS):
        self.nc, self.s, self.h = nc, s, h
        self.lat = G.LatticeGeom(nc, nc, nc, s * h)
        self.op = SCTV(self.lat, device, dtype)
        self.N = self.lat.N
        self.loads = loads
        self.bc = LoadSet(self.lat, self.lat.ijk, (nc, nc, nc), s, h, device, dtype, loads)
        self.freecell = self.bc.free.bool()
        surf = [G.free_surface_cells(ld, (nc, nc, nc)) if _gdir(ld) is not None else np.zeros(self.N, bool)
                for ld in loads]
        self.surf = torch.as_tensor(np.array(surf), device=device)
        self.V = (s * h) ** 3
        self.dt = dtype

    def masks(self, cell):
        """cell (B, N) bool or None -> free (B|1, L, N), up (B|1, L, N, 3)."""
        if cell is None:
            return self.bc.free[None], self.bc.up[None]
        cm = cell.to(self.dt)[:, None]
        return self.bc.free[None] * cm, self.bc.up[None] * cm[..., None]

    def run(self, Kn, Tv, cell=None, tol=1e-10, differentiable=True, maxit=20000):
        """Kn, Tv (B, N, 18), cell (B, N) bool -> dict u, sig, w, F (cement3d/torch_v1.py:163-186)."""
        self.op.set_mask(cell)
        Kn = Kn * self.op.valid[:, 0]
        Tv = Tv * self.op.valid[:, 0]
        Kn4, Tv4 = Kn[:, None], Tv[:, None]
        free, up = self.masks(cell)
        B = Kn.shape[0]
        if differentiable:
            u = LinSolve.apply(Kn4, Tv4, self.op, up.expand(B, -1, -1, -1), free.expand(B, -1, -1), tol)
        else:
            with torch.no_grad():
                u, it, rel = self.op.solve(Kn4, Tv4, up, free, tol, maxit=maxit)
                self.info = (it, rel)
        sig = self.op.stress(u, Kn4, Tv4)
        w = self.op.energy(u, Kn4, Tv4) / self.V
        P = self.op.apply(u, Kn4, Tv4)
        F = torch.stack([(P[:, l, :, _gdir(ld)] * self.bc.moving[l]).sum(-1) if _gdir(ld) is not None
                         else torch.zeros(B, device=Kn.device, dtype=Kn.dtype) for l, ld in enumerate(self.loads)], 1)
        return dict(u=u, sig=sig, w=w, F=F)


class FineRefTV:
    """Fine reference with voids: block sums / means for the s^3 blocks (stress and energy: sum / s^3, voids count
    as zero; displacement: mean over the block's solid particles) and grip reactions (cement3d/torch_v1.py:189-231).
    precision "fp64" (block-Jacobi PCG) or "mixed" (FP32 PCG in FP64 refinement to the same tolerance)."""

    def __init__(self, n, s, h=1.0, device="cuda", dtype=_F64, loads=G.LOADS, precision="fp64"):
        self.n, self.s, self.h = n, s, h
        self.nc = n // s
        self.lat = G.LatticeGeom(n, n, n, h)
        self.op = SCTV(self.lat, device, dtype)
        IJK = self.lat.ijk // s
        self.bc = LoadSet(self.lat, IJK, (self.nc,) * 3, s, h, device, dtype, loads)
        self.loads = loads
        cid = (IJK[:, 2] * self.nc + IJK[:, 1]) * self.nc + IJK[:, 0]
        self.cid = torch.as_tensor(cid, device=device)
        self.Nc = self.nc ** 3
        self.dt = dtype
        self.precision = precision

    def bsum(self, f):
        out = torch.zeros(f.shape[:-2] + (self.Nc, f.shape[-1]), device=f.device, dtype=f.dtype)
        out.index_add_(f.dim() - 2, self.cid, f)
        return out

    @torch.no_grad()
    def run(self, Kn, Tv, solid=None, tol=1e-10, maxit=40000):
        self.op.set_mask(solid)
        Kn = Kn * self.op.valid[:, 0]
        Tv = Tv * self.op.valid[:, 0]
        Kn4, Tv4 = Kn[:, None], Tv[:, None]
        if solid is None:
            free, up = self.bc.free[None], self.bc.up[None]
            sm = torch.ones(1, 1, self.lat.N, device=Kn.device, dtype=self.dt)
        else:
            sm = torch.as_tensor(solid, device=Kn.device).to(self.dt)[:, None]
            free, up = self.bc.free[None] * sm, self.bc.up[None] * sm[..., None]
        B = Kn.shape[0]
        up = up.expand(B, -1, -1, -1)
        free = free.expand(B, -1, -1)
        if self.precision == "mixed":
            u, info = self.op.solve_mixed(Kn4, Tv4, up, free, tol=tol, maxit=maxit)
            it, rel = int(info.iters.max()), float(info.relres.max())
        else:
            u, it, rel = self.op.solve(Kn4, Tv4, up, free, tol, maxit=maxit)
        u = u * sm[..., None]
        sig = self.op.stress(u, Kn4, Tv4)
        U = self.op.energy(u, Kn4, Tv4)
        P = self.op.apply(u, Kn4, Tv4)
        F = torch.stack([(P[:, l, :, _gdir(ld)] * self.bc.moving[l]).sum(-1) if _gdir(ld) is not None
                         else torch.zeros(B, device=Kn.device, dtype=Kn.dtype) for l, ld in enumerate(self.loads)], 1)
        cnt = self.bsum(sm[..., None])
        um = self.bsum(u) / cnt.clamp_min(1.0)
        return dict(u=um, sig=self.bsum(sig) / self.s ** 3,
                    w=self.bsum(U[..., None])[..., 0] / self.s ** 3 / self.h ** 3, F=F, iters=it, relres=rel)
