"""Bond-parameter assembly upstream of the 3D solve, on the CUDA library (drop-in for the two pieces of
coarse3d/train3d.py that every training step runs before and beside the differentiable solve):

  Scatter(nc, s, groups, device)(vals) -> Kn, Tv (B, N, 18)   symmetric scatter of per-group bond values
                                                               (train3d.py:77-97), autograd-capable
  group_penalty(cm, Kn, Tv, frac) -> (pen (B,), lmin)          stability penalty of the (particle, shell) group bond
                                                               Hessians (train3d.py:119-137), autograd-capable
  forward_bond_groups(lat)                                     the axial and diagonal forward-bond groups, every
                                                               undirected bond once (the `bonds` of net3d.BondWindows)

The scatter and its adjoint are one kernel launch per group and per pass (lpm_bond_scatter_f64 /
lpm_bond_gather_sym_f64).  The penalty's eigenvalues come from lpm_group_eigmin_sc (smallest eigenpair of every
6 x 6 and 12 x 12 group Hessian by Jacobi rotations on the device); its gradient uses dlam/dH = v v^T of the
eigenvector, the rest (the sample scale, the relu square) is tensor arithmetic on (B, N) values.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import core
from . import geom as G

_F64 = torch.float64


def forward_bond_groups(lat):
    """[axial, diagonal] groups of forward bonds (even slots 0, 2, 4 and 6, ..., 16) of a full box: dict(bonds (nb, 2)
    = (particle, slot)), particles in increasing order for each slot, as coarse3d/net3d.py:99-117 lists them."""
    out = []
    for slots in (range(0, 6, 2), range(6, 18, 2)):
        bonds = [np.stack([np.nonzero(lat.valid[:, k])[0], np.full(int(lat.valid[:, k].sum()), k)], 1) for k in slots]
        out.append(dict(bonds=np.concatenate(bonds).astype(np.int64)))
    return out


class _ScatterFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sc, *flat):
        B = flat[0].shape[0]
        dev = flat[0].device
        Kn = torch.zeros((B, sc.N, 18), dtype=_F64, device=dev)
        Tv = torch.zeros_like(Kn)
        lib = L.load()
        for gi, (p, k, q) in enumerate(sc.idx):
            kn, tv = flat[2 * gi].contiguous(), flat[2 * gi + 1].contiguous()
            for v, out in ((kn, Kn), (tv, Tv)):
                L.check(lib.lpm_bond_scatter_f64(B, sc.N, p.numel(), L.ptr(p), L.ptr(k), L.ptr(q), L.ptr(v),
                                                 L.ptr(out), L.stream_ptr(dev)), "lpm_bond_scatter_f64")
        ctx.sc = sc
        ctx.B = B
        return Kn, Tv

    @staticmethod
    def backward(ctx, gK, gT):
        sc, B = ctx.sc, ctx.B
        lib = L.load()
        grads = []
        for p, k, q in sc.idx:
            for G_ in (gK, gT):
                g = torch.empty((B, p.numel()), dtype=_F64, device=G_.device)
                L.check(lib.lpm_bond_gather_sym_f64(B, sc.N, p.numel(), L.ptr(p), L.ptr(k), L.ptr(q),
                                                    L.ptr(G_.contiguous()), L.ptr(g), L.stream_ptr(G_.device)),
                        "lpm_bond_gather_sym_f64")
                grads.append(g)
        return (None,) + tuple(grads)


class Scatter:
    """Per-group bond values -> symmetric (B, N, 18) parameter arrays (coarse3d/train3d.py:77-97).  Each group's
    `bonds` (nb, 2) holds (particle p, slot k); the value lands on slot k of p and on slot k^1 of its neighbour."""

    def __init__(self, nc, s, groups, device="cuda"):
        lat = G.LatticeGeom(nc, nc, nc, s)
        self.N = lat.N
        dev = torch.device(device)
        L.require_cuda(torch.empty(0, device=dev))
        self.idx = []
        for g in groups:
            b = np.asarray(g["bonds"])
            q = lat.nbr[b[:, 0], b[:, 1]]
            self.idx.append(tuple(torch.as_tensor(np.ascontiguousarray(x, dtype=np.int32), device=dev)
                                  for x in (b[:, 0], b[:, 1], q)))

    def __call__(self, vals):
        """vals: list over groups of (kn (B, nb), tv (B, nb)) -> Kn, Tv (B, N, 18)."""
        flat = [x.to(_F64) for kv in vals for x in kv]
        return _ScatterFn.apply(self, *flat)


class _GroupEig(torch.autograd.Function):
    """Smallest eigenvalue (B, N) of the shell-`shell` group Hessians; gradients to Kn, Tv (B, N, 18) and sc (B,)."""

    @staticmethod
    def forward(ctx, Kn, Tv, sc, dl, shell):
        B = Kn.shape[0]
        M = 6 if shell == 0 else 12
        Kc, Tc, scc = Kn.contiguous(), Tv.contiguous(), sc.contiguous()
        lam = torch.empty((B, dl.N), dtype=_F64, device=Kn.device)
        vec = torch.empty((B, dl.N, M), dtype=_F64, device=Kn.device)
        L.check(L.load().lpm_group_eigmin_sc(dl.ref, B, L.ptr(Kc), L.ptr(Tc), L.ptr(scc), shell, L.ptr(lam),
                                             L.ptr(vec), L.stream_ptr(Kn.device)), "lpm_group_eigmin_sc")
        ctx.save_for_backward(vec)
        ctx.shell, ctx.M, ctx.valid = shell, M, dl
        return lam

    @staticmethod
    def backward(ctx, g):
        (vec,) = ctx.saved_tensors
        dl, shell, M = ctx.valid, ctx.shell, ctx.M
        sl = slice(0, 6) if shell == 0 else slice(6, 18)
        vv = torch.as_tensor(dl.lat.valid[:, sl], device=vec.device, dtype=_F64)           # (N, M)
        w = vec * vv
        gK = torch.zeros(vec.shape[:2] + (18,), dtype=_F64, device=vec.device)
        gT = torch.zeros_like(gK)
        gK[..., sl] = g[..., None] * w * w                                                  # dH_aa / dkn_a
        gT[..., sl] = g[..., None] * w * w.sum(-1, keepdim=True)                            # sum_c v_a v_c
        gsc = (g * (1e3 * (vec * vec * (1 - vv)).sum(-1))).sum(-1)                          # 1e3 sc on missing slots
        return gK, gT, gsc, None, None


def group_penalty(cm, Kn, Tv, frac=0.05):
    """relu(frac - lambda_min / mean|Kn|)^2 summed over the (particle, shell) groups of every sample, and the smallest
    scaled eigenvalue (coarse3d/train3d.py:119-137).  cm: a torch_lpm3d.CoarseT (full box); Kn, Tv (B, N, 18)."""
    dl = cm.op.dl
    sc = Kn.abs().mean((1, 2))
    pen = 0.0
    lmin = []
    for shell in (0, 1):
        lam = _GroupEig.apply(Kn.to(_F64), Tv.to(_F64), sc, dl, shell) / sc[:, None]
        pen = pen + (torch.relu(frac - lam) ** 2).sum(1)
        lmin.append(lam.min())
    return pen, float(min(lmin).detach())
