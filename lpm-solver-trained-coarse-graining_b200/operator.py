"""Lattice operator objects with autograd, shared by the 3D (torch_lpm3d) and 2D (torch_lpm) drop-in modules.

Every evaluation runs in liblpm_b200.so: K u, stress, energy and their vector-Jacobian products, block-Jacobi
preconditioners, batched PCG, the adjoint solve and the per-bond gradient.  The VJPs of apply / stress / energy are
exact for any bond parameters; the LinSolve adjoint reuses K for K^T, i.e. assumes symmetric bond parameters, as the
reference's adjoint does.
"""
import numpy as np
import torch

from . import _lib
from . import core

_F64 = torch.float64


def inv3(D):
    """Inverse of (..., d, d) blocks (mirror of the reference helper coarse3d/torch_lpm3d.py:22-33)."""
    return torch.linalg.inv(D)


def _sum_to(g, K, lead):
    """Reduce a per-coefficient-set gradient (nset, N, NN) to the shape of K (broadcast over `lead`)."""
    kshape = tuple(K.shape)
    n = int(np.prod(kshape[:-2])) if len(kshape) > 2 else 1
    if g.shape[0] == n:
        return g.reshape(kshape)
    full = g.reshape(tuple(lead) + kshape[-2:])
    kl = (1,) * (len(lead) - (len(kshape) - 2)) + kshape[:-2]
    dims = tuple(i for i, (a, b) in enumerate(zip(kl, lead)) if a == 1 and b != 1)
    if dims:
        full = full.sum(dims, keepdim=True)
    return full.reshape(kshape)


class _Apply(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, Kn, Tv, dl):
        ctx.save_for_backward(u, Kn, Tv)
        ctx.dl = dl
        return core.kmv(dl, u, Kn, Tv)

    @staticmethod
    def backward(ctx, g):
        u, Kn, Tv = ctx.saved_tensors
        dl = ctx.dl
        g = g.contiguous()
        du = dK = dT = None
        lead = torch.broadcast_shapes(u.shape[:-2], Kn.shape[:-2])
        if dl.dim == 3:
            # one pass: du = K^T g (the code-force operator is not symmetric for non-symmetric parameters)
            du, gK, gT = core.post_vjp(dl, "apply", u, g, Kn, Tv)
            du = du.to(u.dtype)
        else:
            # the square lattice's operator is an exact Hessian: K^T = K
            if ctx.needs_input_grad[0]:
                du = core.kmv(dl, g.to(u.dtype), Kn.to(u.dtype), Tv.to(u.dtype))
            gK, gT = core.bond_grad(dl, u, g, Kn, Tv) if (ctx.needs_input_grad[1] or ctx.needs_input_grad[2]) \
                else (None, None)
        if ctx.needs_input_grad[1]:
            dK = _sum_to(gK, Kn, lead).to(Kn.dtype)
        if ctx.needs_input_grad[2]:
            dT = _sum_to(gT, Tv, lead).to(Tv.dtype)
        return du if ctx.needs_input_grad[0] else None, dK, dT, None


class _Post(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u, Kn, Tv, dl, which):
        ctx.save_for_backward(u, Kn, Tv)
        ctx.dl, ctx.which = dl, which
        out = core.stress(dl, u, Kn, Tv) if which == "stress" else core.energy(dl, u, Kn, Tv)
        return out.to(u.dtype)

    @staticmethod
    def backward(ctx, g):
        u, Kn, Tv = ctx.saved_tensors
        du, gK, gT = core.post_vjp(ctx.dl, ctx.which, u, g.contiguous(), Kn, Tv)
        lead = u.shape[:-2]
        dK = _sum_to(gK, Kn, lead).to(Kn.dtype) if ctx.needs_input_grad[1] else None
        dT = _sum_to(gT, Tv, lead).to(Tv.dtype) if ctx.needs_input_grad[2] else None
        return du.to(u.dtype) if ctx.needs_input_grad[0] else None, dK, dT, None, None


def _lead_expand(u, Kn):
    """u may carry fewer leading dimensions than Kn (e.g. a shared up (1, L, N, 3) against Kn (B, 1, N, 18))."""
    lead = torch.broadcast_shapes(u.shape[:-2], Kn.shape[:-2])
    if tuple(u.shape[:-2]) != tuple(lead):
        u = u.expand(tuple(lead) + tuple(u.shape[-2:]))
    return u


class LatticeOperator:
    """Matrix-free LPM operator on a fixed lattice geometry (geom.LatticeGeom or geom.Lattice2D), on the GPU.

    SC lattice: code-force operator (coarse3d/torch_lpm3d.py:63-83); square lattice: exact-Hessian operator
    (timing/t2d/solver2d.py:269-305, coarse2d/torch_lpm.py:173-191)."""

    def __init__(self, lat, device="cuda", dtype=_F64, dl=None):
        self.lat, self.dev, self.dt = lat, torch.device(device), dtype
        self.dl = core.DeviceLattice(lat, device) if dl is None else dl
        self.N = lat.N
        self.ndir = torch.as_tensor(lat.ndir, device=self.dev, dtype=dtype)
        self.valid = torch.as_tensor(lat.valid, device=self.dev, dtype=dtype)
        self.shell = torch.as_tensor(lat.shell, device=self.dev)
        self.d, self.NN = lat.dim, lat.NN

    # ------------------------------------------------------------------------------------------- kernels
    def apply(self, u, Kn, Tv):
        """K u (..., N, d) (coarse3d/torch_lpm3d.py:81-83)."""
        u = _lead_expand(u, Kn)
        if torch.is_grad_enabled() and (u.requires_grad or Kn.requires_grad or Tv.requires_grad):
            return _Apply.apply(u, Kn, Tv, self.dl)
        return core.kmv(self.dl, u.to(self.dt), Kn.to(self.dt), Tv.to(self.dt))

    def stress(self, u, Kn, Tv):
        """Particle stress (..., N, 6) xx yy zz yz xz xy, or (..., N, 3) xx yy xy (coarse3d/torch_lpm3d.py:85-87)."""
        u = _lead_expand(u, Kn)
        if torch.is_grad_enabled() and (u.requires_grad or Kn.requires_grad or Tv.requires_grad):
            return _Post.apply(u, Kn, Tv, self.dl, "stress")
        return core.stress(self.dl, u, Kn, Tv).to(u.dtype)

    def energy(self, u, Kn, Tv):
        """Particle energy (..., N) (coarse3d/torch_lpm3d.py:89-92)."""
        u = _lead_expand(u, Kn)
        if torch.is_grad_enabled() and (u.requires_grad or Kn.requires_grad or Tv.requires_grad):
            return _Post.apply(u, Kn, Tv, self.dl, "energy")
        return core.energy(self.dl, u, Kn, Tv).to(u.dtype)

    def block_diag(self, Kn, Tv):
        """d x d diagonal blocks of K (..., N, d, d) (coarse3d/torch_lpm3d.py:94-102)."""
        lead = Kn.shape[:-2]
        _, D = core.block_jacobi(self.dl, Kn, Tv, _F64, want_D=True)
        return D.reshape(tuple(lead) + (self.N, self.d, self.d)).to(self.dt)

    def precond(self, Kn, Tv, free):
        """Block-Jacobi inverse (..., N, d, d), zero on fixed particles (coarse3d/torch_lpm3d.py:104-106)."""
        lead = Kn.shape[:-2]
        M = core.block_jacobi(self.dl, Kn, Tv, _F64).reshape(tuple(lead) + (self.N, self.d, self.d))
        return (M * free[..., None, None]).to(self.dt)

    # ----------------------------------------------------------------------------------------------- PCG
    def _solve_sets(self, b, Kn, Tv, free, tol, maxit, check, x0=None, M=None):
        """PCG on every system of b with the preconditioner per coefficient set (or the given per-system M)."""
        lead = torch.broadcast_shapes(b.shape[:-2], Kn.shape[:-2], free.shape[:-1])
        b = b.expand(tuple(lead) + (self.N, self.d)).to(self.dt)
        if M is None:
            Kc, rps = core.coef_sets(Kn.to(self.dt), self.dl, lead)
            Tc, _ = core.coef_sets(Tv.to(self.dt), self.dl, lead)
            Minv = core.block_jacobi(self.dl, Kc, Tc, self.dt)
        else:
            nsys = int(np.prod(lead)) if lead else 1
            Kc = Kn.to(self.dt).expand(tuple(lead) + (self.N, self.NN)).reshape(nsys, self.N, self.NN)
            Tc = Tv.to(self.dt).expand(tuple(lead) + (self.N, self.NN)).reshape(nsys, self.N, self.NN)
            Minv = M.to(self.dt).expand(tuple(lead) + (self.N, self.d, self.d)).reshape(nsys, self.N, self.d, self.d)
        nsys = int(np.prod(lead)) if lead else 1
        rps = nsys // Kc.shape[0]
        layout = _lib.LAYOUT_REF
        if self.dl.nbr is None and self.d == 3:   # full SC boxes run on the packed (SoA) layout, the fused operator
            Kc, Tc, layout = core.pack(Kc, self.dt), core.pack(Tc, self.dt), _lib.LAYOUT_SOA
        x, info = core.cg(self.dl, Kc, Tc, b.reshape(nsys, self.N, self.d),
                          x=None if x0 is None else x0.expand(tuple(lead) + (self.N, self.d)).reshape(nsys, self.N, self.d),
                          Minv=Minv, free=free.expand(tuple(lead) + (self.N,)).reshape(nsys, self.N), tol=tol,
                          maxit=maxit, check=check, layout=layout, rhs_per_set=rps)
        x = x.reshape(tuple(lead) + (self.N, self.d))
        return x, info

    def bond_grad(self, u, lam, Kn, Tv):
        """Per-slot d(lam . K(Kn, Tv) u)/d(Kn, Tv), summed over the systems sharing each coefficient set."""
        return core.bond_grad(self.dl, u, lam, Kn, Tv)

    def pcg(self, b, Kn, Tv, M, free, tol=1e-10, maxit=20000, x0=None, check=10):
        """Solve K_ff x = b for all systems (coarse3d/torch_lpm3d.py:109-140).  Returns (x, iterations, max rel)."""
        with torch.no_grad():
            x, info = self._solve_sets(b, Kn, Tv, free, tol, maxit, check, x0=x0, M=M)
        info.raise_on_breakdown()
        return x, int(info.iters.max()), float(info.relres.max())

    def solve(self, Kn, Tv, up, free, tol=1e-10, maxit=20000, M=None, check=10):
        """u = up on fixed particles and (K u)_free = 0 (coarse3d/torch_lpm3d.py:142-148)."""
        with torch.no_grad():
            b = -self.apply(up, Kn, Tv) * free[..., None]
            x, info = self._solve_sets(b, Kn, Tv, free, tol, maxit, check, M=M)
        info.raise_on_breakdown()
        return up + x, int(info.iters.max()), float(info.relres.max())

    def solve_mixed(self, Kn, Tv, up, free, tol=1e-8, inner_tol=1e-3, maxit=20000):
        """FP32 inner PCG with FP64 iterative refinement to |b - K x| <= tol |b| (FP64 true residual)."""
        with torch.no_grad():
            lead = torch.broadcast_shapes(up.shape[:-2], Kn.shape[:-2], free.shape[:-1])
            b = -self.apply(up, Kn, Tv) * free[..., None]
            b = b.expand(tuple(lead) + (self.N, self.d))
            x, info = core.ir(self.dl, Kn.to(_F64), Tv.to(_F64), b, free=free.expand(tuple(lead) + (self.N,)),
                              tol=tol, inner_tol=inner_tol, maxit=maxit)
        info.raise_on_breakdown()
        return up + x, info

    def solve_amg(self, Kn, Tv, up, free, tol=1e-8, inner_tol=1e-4, maxit=20000, **amg_cfg):
        """Mixed-precision solve preconditioned by the aggregation AMG (``amg.AmgBatch``, settings of
        timing/t3d/problems.py:19 unless overridden): full simple-cubic boxes whose free sets are boxes, as every load case
        of geom.prescribed.  One hierarchy per (specimen, free box), rebuilt for the coefficients of every call; the
        aggregation geometry is cached per batch shape and set of masks.  Returns (up + x, SolveInfo)."""
        from . import amg as GA
        if self.d != 3 or self.dl.nbr is not None:
            raise ValueError("solve_amg needs a full simple-cubic box")
        with torch.no_grad():
            lead = tuple(torch.broadcast_shapes(up.shape[:-2], Kn.shape[:-2], free.shape[:-1]))
            N, d = self.N, self.d
            b = (-self.apply(up, Kn, Tv) * free[..., None]).expand(lead + (N, d))
            Kc, rps = core.coef_sets(Kn.to(_F64), self.dl, lead)
            Tc, _ = core.coef_sets(Tv.to(_F64), self.dl, lead)
            nsys = int(np.prod(lead)) if lead else 1
            fm = (free.expand(lead + (N,)) != 0).reshape(nsys, N)
            per_set = fm.reshape(-1, rps, N)
            masks = per_set[0] if bool((per_set == per_set[:1]).all()) else fm
            mh = masks.cpu().numpy()
            cfg = dict(GA.AMG_CFG, **amg_cfg)
            key = (nsys, rps, mh.shape, hash(mh.tobytes()), tuple(sorted(cfg.items())))
            cache = self.__dict__.setdefault("_amg_cache", {})
            ab = cache.get(key)
            if ab is None:
                if len(cache) >= 4:
                    for v in cache.values():
                        v.close()
                    cache.clear()
                ab = cache[key] = GA.AmgBatch(self.dl, nsys, rps, mh, **cfg)
            K32, T32 = core.pack(Kc, torch.float32), core.pack(Tc, torch.float32)
            ab.setup(K32, T32, core.block_jacobi(self.dl, Kc, Tc, torch.float32))
            x, info = ab.ir(Kc, Tc, b.reshape(nsys, N, d), tol=tol, inner_tol=inner_tol, maxit=maxit)
        info.raise_on_breakdown()
        return up + x.reshape(lead + (N, d)), info


class LinSolve(torch.autograd.Function):
    """u = solve(Kn, Tv) with the exact adjoint gradient w.r.t. Kn, Tv (coarse3d/torch_lpm3d.py:151-175; for the
    square lattice the exact-Hessian gradient of coarse2d/torch_lpm.py:34-51 through assemble).

    Forward: block-Jacobi PCG.  Backward: adjoint PCG K_ff lam = g_f with the same K, then the per-bond gradient
    kernel gives -d(lam . K(Kn, Tv) u)/d(Kn, Tv), summed over broadcast load cases."""

    @staticmethod
    def forward(ctx, Kn, Tv, op, up, free, tol):
        with torch.no_grad():
            b = -op.apply(up, Kn, Tv) * free[..., None]
            x, info = op._solve_sets(b, Kn, Tv, free, tol, 20000, 10)
            info.raise_on_breakdown()
            u = up + x
        ctx.save_for_backward(Kn, Tv, u)
        ctx.op, ctx.free, ctx.tol = op, free, tol
        ctx.info = (int(info.iters.max()), float(info.relres.max()))
        return u

    @staticmethod
    def backward(ctx, g):
        Kn, Tv, u = ctx.saved_tensors
        op, free = ctx.op, ctx.free
        with torch.no_grad():
            lam, info = op._solve_sets(g * free[..., None], Kn, Tv, free, ctx.tol, 20000, 10)
            info.raise_on_breakdown()
            gK, gT = op.bond_grad(u, lam, Kn, Tv)
            lead = u.shape[:-2]
            dK = -_sum_to(gK, Kn, lead).to(Kn.dtype)
            dT = -_sum_to(gT, Tv, lead).to(Tv.dtype)
        return dK, dT, None, None, None, None


