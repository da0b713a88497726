"""Torch-level calls into the CUDA library: device lattices, K.u, preconditioner, batched CG, mixed-precision
refinement, gradients and post-processing.

Batching model (shared with the C ABI): ``nsys`` systems (right-hand sides) flattened from the leading dimensions of
the vector arguments; coefficient sets are matched to systems set-major (system ``s`` uses set ``s // rhs_per_set``)
and DOF masks periodically (``s % nmask``).  Broadcast patterns that do not fit are materialised.
"""
import ctypes
import math

import numpy as np
import torch

from . import _lib as L

_F64, _F32 = torch.float64, torch.float32


class DeviceLattice:
    """A host lattice (``geom.LatticeGeom`` or ``geom.Lattice2D``) described for the CUDA library.

    Full boxes use implicit neighbours; lattices with inactive sites carry an int32 neighbour table on the device.
    """

    def __init__(self, lat, device="cuda", nbr=None):
        """nbr: optional (N, NN) int32 CUDA tensor of bonds that replaces the geometric ones (-1 = no bond), e.g. one
        specimen's table from solid_tables(); the lattice then runs on the table kernels."""
        self.lat = lat
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise L.LPMError("DeviceLattice needs a CUDA device (got %s); there is no CPU fallback" % self.device)
        L.load()
        self.dim = lat.dim
        self.N = lat.N
        self.NN = lat.NN
        nz = lat.nz if lat.dim == 3 else 1
        self.nbr = None
        if nbr is not None:
            if tuple(nbr.shape) != (lat.N, lat.NN) or nbr.dtype != torch.int32 or not nbr.is_cuda:
                raise ValueError("bond table must be a CUDA int32 tensor of shape (%d, %d)" % (lat.N, lat.NN))
            self.nbr = nbr.contiguous()
        elif not lat.full:
            self.nbr = torch.as_tensor(np.ascontiguousarray(lat.nbr, dtype=np.int32), device=self.device)
        self.c = L.Lattice(lat.dim, lat.nx, lat.ny, nz, lat.N, None if self.nbr is None else self.nbr.data_ptr())
        self.l0 = torch.as_tensor(np.asarray(lat.l0, float), device=self.device, dtype=_F64)
        self.V = float(lat.V)

    @property
    def ref(self):
        return ctypes.byref(self.c)


# ----------------------------------------------------------------------------------------------------- helpers
def _batch(nsys, rps, nmask=1):
    return L.Batch(int(nsys), int(rps), int(nmask), 0)


def _flat_vec(u, dl):
    if u.shape[-2:] != (dl.N, dl.dim):
        raise ValueError("expected (..., %d, %d), got %s" % (dl.N, dl.dim, tuple(u.shape)))
    L.require_cuda(u)
    return u.reshape(-1, dl.N, dl.dim).contiguous()


def coef_sets(K, dl, lead):
    """Coefficient tensor (..., N, NN) -> ((nset, N, NN) contiguous, rhs_per_set) for systems of leading shape `lead`.

    Works without copying when K's leading shape is a prefix of `lead` followed by ones (the reference's (B, 1, N, NN)
    against (B, L, N, d)); other broadcasts are materialised.
    """
    if K.shape[-2:] != (dl.N, dl.NN):
        raise ValueError("expected coefficients (..., %d, %d), got %s" % (dl.N, dl.NN, tuple(K.shape)))
    L.require_cuda(K)
    kl = tuple(K.shape[:-2])
    lead = tuple(lead)
    nsys = int(np.prod(lead)) if lead else 1
    kl_full = (1,) * (len(lead) - len(kl)) + kl
    if len(kl_full) > len(lead):
        raise ValueError("coefficient batch %s does not broadcast to %s" % (kl, lead))
    ok = all(a == b or a == 1 for a, b in zip(kl_full, lead))
    if not ok:
        raise ValueError("coefficient batch %s does not broadcast to %s" % (kl, lead))
    # find the split point: kl_full == lead[:j] + (1,)*(rest)
    j = len(lead)
    while j > 0 and kl_full[j - 1] == 1:
        j -= 1
    if kl_full[:j] == lead[:j]:
        nset = int(np.prod(lead[:j])) if j else 1
        return K.reshape(nset, dl.N, dl.NN).contiguous(), nsys // nset
    Kx = K.expand(lead + (dl.N, dl.NN)).reshape(nsys, dl.N, dl.NN).contiguous()
    return Kx, 1


def dof_masks(free, dl, lead):
    """Particle (..., N) or DOF (..., N, d) free masks (any dtype, nonzero = free) -> ((nmask, N, d) uint8, nmask)."""
    if free is None:
        return None, 1
    f = free
    if f.dim() >= 2 and f.shape[-1] == dl.dim and f.shape[-2] == dl.N:
        per_dof = True
    elif f.shape[-1] == dl.N:
        per_dof = False
    else:
        raise ValueError("free mask of shape %s does not match N = %d" % (tuple(f.shape), dl.N))
    fl = tuple(f.shape[:-2] if per_dof else f.shape[:-1])
    lead = tuple(lead)
    fl_full = (1,) * (len(lead) - len(fl)) + fl
    j = 0
    while j < len(fl_full) and fl_full[j] == 1:
        j += 1
    if fl_full[j:] == lead[j:]:
        nmask = int(np.prod(lead[j:])) if j < len(lead) else 1
        m = f.reshape((nmask, dl.N, dl.dim) if per_dof else (nmask, dl.N))
    else:
        m = f.expand(lead + tuple(f.shape[len(fl):]))
        nmask = int(np.prod(lead))
        m = m.reshape((nmask, dl.N, dl.dim) if per_dof else (nmask, dl.N))
    m = (m != 0).to(torch.uint8)
    if not per_dof:
        m = m[..., None].expand(nmask, dl.N, dl.dim)
    return m.contiguous(), nmask


def _prof_ptr(prof):
    """prof: a ctypes (c_double * 4) array accumulating [K.u ms, K.u launches, full-batch K.u ms, full-batch launches]
    (see lpm_cg_opts.prof), or None."""
    return None if prof is None else ctypes.cast(prof, ctypes.POINTER(ctypes.c_double))


def new_prof():
    return (ctypes.c_double * 4)(0.0, 0.0, 0.0, 0.0)


def _scratch(nbytes, device):
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


def autotune(dl, K32, T32, nsys, rhs_per_set, with_variant=False):
    """Time the variants and z-chunk candidates of the pair-packed FP32 operator for this batch shape (packed FP32
    coefficients K32/T32 (nset, NN, N)); the fastest is recorded in the library for later launches and returned
    (zchunk, or (zchunk, variant) with with_variant)."""
    lib = L.load()
    scr = _scratch(lib.lpm_kmv_scratch_bytes(dl.ref, L.LPM_F32, int(nsys)), K32.device)
    z, v = ctypes.c_int32(0), ctypes.c_int32(0)
    b = _batch(nsys, rhs_per_set)
    L.check(lib.lpm_autotune_kmv(dl.ref, ctypes.byref(b), L.ptr(K32), L.ptr(T32), L.ptr(scr), scr.numel(),
                                 ctypes.byref(z), ctypes.byref(v), L.stream_ptr(K32.device)), "lpm_autotune_kmv")
    return (int(z.value), int(v.value)) if with_variant else int(z.value)


def tune_set(dl, nsys, rhs_per_set, zchunk, variant):
    """Pin the pair-packed operator's z-chunk and variant for this batch shape (instead of autotune)."""
    b = _batch(nsys, rhs_per_set)
    L.check(L.load().lpm_tune_kmv_set(dl.ref, ctypes.byref(b), int(zchunk), int(variant)), "lpm_tune_kmv_set")


def pack(K, dtype=_F32):
    """(nset, N, NN) FP64 -> (nset, NN, N) in `dtype` (the packed SoA layout of the solver)."""
    L.require_cuda(K)
    K = K.to(_F64).contiguous()
    nset, N, NN = K.shape
    out = torch.empty((nset, NN, N), dtype=dtype, device=K.device)
    fn = L.load().lpm_pack_coef_f32 if dtype == _F32 else L.load().lpm_pack_coef_f64
    L.check(fn(L.ptr(K), L.ptr(out), N, NN, nset, L.stream_ptr(K.device)), "lpm_pack_coef")
    return out


# ------------------------------------------------------------------------------------------------------- K . u
def kmv(dl, u, Kn, Tv, layout=L.LAYOUT_REF, rhs_per_set=None):
    """K u for u (..., N, d); Kn/Tv (nset, N, NN) [layout REF] or (nset, NN, N) [layout SOA], same dtype as u."""
    lead = u.shape[:-2]
    uf = _flat_vec(u, dl)
    nsys = uf.shape[0]
    if layout == L.LAYOUT_REF:
        Kc, rps = coef_sets(Kn, dl, lead)
        Tc, rps2 = coef_sets(Tv, dl, lead)
        if rps != rps2:
            raise ValueError("Kn and Tv batch shapes differ")
    else:
        Kc, Tc = Kn.contiguous(), Tv.contiguous()
        rps = rhs_per_set or nsys // Kc.shape[0]
    if Kc.dtype != uf.dtype or Tc.dtype != uf.dtype:
        raise TypeError("u, Kn and Tv must share a dtype (got %s, %s, %s)" % (uf.dtype, Kc.dtype, Tc.dtype))
    lib = L.load()
    prec = L.LPM_F64 if uf.dtype == _F64 else L.LPM_F32
    nb = lib.lpm_kmv_scratch_bytes(dl.ref, prec, nsys)
    scr = _scratch(nb, uf.device)
    out = torch.empty_like(uf)
    name = "lpm_kmv_%s_%s" % ("sc" if dl.dim == 3 else "sq", "f64" if prec == L.LPM_F64 else "f32")
    b = _batch(nsys, rps)
    L.check(getattr(lib, name)(dl.ref, L.ptr(uf), L.ptr(Kc), L.ptr(Tc), layout, ctypes.byref(b), L.ptr(out),
                               L.ptr(scr), scr.numel(), L.stream_ptr(uf.device)), name)
    return out.reshape(u.shape)


# ------------------------------------------------------------------------------------------------ preconditioner
def block_jacobi(dl, Kn, Tv, dtype=_F64, want_D=False):
    """Inverse diagonal blocks (nset, N, d, d) in `dtype` (and the FP64 blocks D if want_D) of K per coefficient set."""
    L.require_cuda(Kn)
    Kn = Kn.to(_F64).reshape(-1, dl.N, dl.NN).contiguous()
    Tv = Tv.to(_F64).reshape(-1, dl.N, dl.NN).contiguous()
    nset = Kn.shape[0]
    M = torch.empty((nset, dl.N, dl.dim, dl.dim), dtype=dtype, device=Kn.device)
    D = torch.empty((nset, dl.N, dl.dim, dl.dim), dtype=_F64, device=Kn.device) if want_D else None
    lib = L.load()
    fn = lib.lpm_block_jacobi_f64 if dtype == _F64 else lib.lpm_block_jacobi_f32
    L.check(fn(dl.ref, L.ptr(Kn), L.ptr(Tv), L.LAYOUT_REF, nset, L.ptr(M), L.ptr(D), L.stream_ptr(Kn.device)),
            "lpm_block_jacobi")
    return (M, D) if want_D else M


# --------------------------------------------------------------------------------------------------- batched CG
class SolveInfo:
    """Per-system outcome of a batched solve (host numpy arrays)."""

    def __init__(self, iters, relres, status, outer=None):
        self.iters = iters
        self.relres = relres
        self.status = status
        self.outer = outer

    def raise_on_breakdown(self):
        if (self.status == L.STATUS_BREAKDOWN).any():
            raise FloatingPointError("LPM solve broke down (p.Ap <= 0 or non-finite values: unstable bond parameters)")

    def __repr__(self):
        return "SolveInfo(iters=%s, relres=%s, status=%s, outer=%s)" % (self.iters, self.relres, self.status,
                                                                         self.outer)


def cg(dl, Kn, Tv, b, x=None, Minv=None, free=None, tol=1e-10, maxit=20000, check=1, poll=None, precheck=False,
       layout=L.LAYOUT_REF, rhs_per_set=None, prof=None, engine=L.ENGINE_AUTO, pack2d=True):
    """Batched (P)CG on the free DOFs.  b (..., N, d) zero on fixed DOFs; x start (zero if None), returned updated.

    dtype of b decides the precision (float64 or float32); Kn/Tv/Minv must match it.  With rhs_per_set given, Kn/Tv
    are the coefficient sets themselves ((nset, N, NN) for the reference layout, packed for SoA), systems
    s*rhs_per_set .. (s+1)*rhs_per_set-1 using set s.  engine: L.ENGINE_AUTO / ENGINE_LAUNCHED / ENGINE_PERSISTENT
    (one cooperative kernel per solve, small batches).  pack2d: reference-layout coefficients of a full 2D box are
    packed (SoA) once before the iterations, where a warp's per-slot reads are contiguous (10 x 128^2 FP64 plain CG:
    25.7 instead of 32.2 us per iteration); pack2d=False keeps the reference layout.  Returns (x, SolveInfo).
    """
    lead = b.shape[:-2]
    bf = _flat_vec(b, dl)
    nsys = bf.shape[0]
    dt = bf.dtype
    if layout == L.LAYOUT_REF and rhs_per_set is None:
        Kc, rps = coef_sets(Kn, dl, lead)
        Tc, _ = coef_sets(Tv, dl, lead)
    else:                                   # coefficient sets given explicitly, rhs_per_set systems each
        Kc, Tc = Kn.contiguous(), Tv.contiguous()
        rps = rhs_per_set or nsys // Kc.shape[0]
    if Kc.dtype != dt or Tc.dtype != dt:
        raise TypeError("coefficients must have the dtype of b (%s)" % dt)
    if pack2d and layout == L.LAYOUT_REF and dl.dim == 2 and dl.nbr is None:
        Kc, Tc, layout = pack(Kc.reshape(-1, dl.N, dl.NN), dt), pack(Tc.reshape(-1, dl.N, dl.NN), dt), L.LAYOUT_SOA
    if Minv is not None:
        Minv = Minv.to(dt).reshape(-1, dl.N, dl.dim, dl.dim).contiguous()
        if Minv.shape[0] * rps != nsys and Minv.shape[0] != 1:
            raise ValueError("Minv sets %d do not match %d systems / %d per set" % (Minv.shape[0], nsys, rps))
    m, nmask = dof_masks(free, dl, lead)
    x0_zero = x is None
    xf = torch.zeros_like(bf) if x is None else _flat_vec(x, dl).to(dt).clone()
    lib = L.load()
    prec = L.LPM_F64 if dt == _F64 else L.LPM_F32
    b_ = _batch(nsys, rps, nmask)
    ws = _scratch(lib.lpm_cg_workspace_bytes(dl.ref, ctypes.byref(b_), prec, int(Minv is not None)), bf.device)
    it = torch.zeros(nsys, dtype=torch.int32, device=bf.device)
    rel = torch.zeros(nsys, dtype=_F64, device=bf.device)
    st = torch.zeros(nsys, dtype=torch.int32, device=bf.device)
    opts = L.CgOpts(float(tol), int(maxit), int(check), int(poll or max(check, 10)), int(bool(precheck)),
                    _prof_ptr(prof), None, int(engine), 0)
    fn = lib.lpm_cg_batched_f64 if prec == L.LPM_F64 else lib.lpm_cg_batched_f32
    L.check(fn(dl.ref, L.ptr(Kc), L.ptr(Tc), layout, ctypes.byref(b_), L.ptr(Minv), L.ptr(m), L.ptr(bf), L.ptr(xf),
               int(x0_zero), ctypes.byref(opts), L.ptr(ws), ws.numel(), L.ptr(it), L.ptr(rel), L.ptr(st),
               L.stream_ptr(bf.device)), "lpm_cg_batched")
    info = SolveInfo(it.cpu().numpy(), rel.cpu().numpy(), st.cpu().numpy())
    return xf.reshape(b.shape), info


def ir(dl, Kn64, Tv64, b, x=None, free=None, tol=1e-8, inner_tol=1e-3, maxit=20000, max_outer=20, check=1,
       poll=10, precond=True, packed=None, prof=None, engine=L.ENGINE_AUTO):
    """Mixed-precision solve: FP32 inner PCG, FP64 iterative refinement to |b - K x| <= tol |b| (FP64 operator).

    b (..., N, d) float64, zero on fixed DOFs.  `packed` may pass a precomputed (Kn32, Tv32, Minv32) triple.
    engine selects the inner solves' CG engine (see cg).
    Returns (x, SolveInfo) with total inner iterations and the final FP64 relative residual per system.
    """
    lead = b.shape[:-2]
    bf = _flat_vec(b.to(_F64), dl)
    nsys = bf.shape[0]
    Kc, rps = coef_sets(Kn64.to(_F64), dl, lead)
    Tc, _ = coef_sets(Tv64.to(_F64), dl, lead)
    if packed is None:
        K32, T32 = pack(Kc, _F32), pack(Tc, _F32)
        M32 = block_jacobi(dl, Kc, Tc, _F32) if precond else None
    else:
        K32, T32, M32 = packed
    m, nmask = dof_masks(free, dl, lead)
    xf = torch.zeros_like(bf) if x is None else _flat_vec(x, dl).to(_F64).clone()
    lib = L.load()
    lay64 = L.LAYOUT_REF
    if dl.dim == 3 and dl.nbr is None:      # full SC box: the FP64 residuals run on the TMA operator (packed SoA)
        Kc, Tc, lay64 = pack(Kc, _F64), pack(Tc, _F64), L.LAYOUT_SOA
    b_ = _batch(nsys, rps, nmask)
    ws = _scratch(lib.lpm_ir_workspace_bytes(dl.ref, ctypes.byref(b_), int(M32 is not None)), bf.device)
    it = torch.zeros(nsys, dtype=torch.int32, device=bf.device)
    rel = torch.zeros(nsys, dtype=_F64, device=bf.device)
    st = torch.zeros(nsys, dtype=torch.int32, device=bf.device)
    outer = ctypes.c_int32(0)
    opts = L.IrOpts(float(tol), float(inner_tol), int(maxit), int(max_outer), int(check), int(poll),
                    _prof_ptr(prof), int(x is None), int(engine))
    L.check(lib.lpm_ir_batched(dl.ref, L.ptr(Kc), L.ptr(Tc), lay64, L.ptr(K32), L.ptr(T32), L.ptr(M32),
                               ctypes.byref(b_), L.ptr(m), L.ptr(bf), L.ptr(xf), ctypes.byref(opts), L.ptr(ws),
                               ws.numel(), L.ptr(it), L.ptr(rel), L.ptr(st), ctypes.byref(outer),
                               L.stream_ptr(bf.device)), "lpm_ir_batched")
    info = SolveInfo(it.cpu().numpy(), rel.cpu().numpy(), st.cpu().numpy(), int(outer.value))
    return xf.reshape(b.shape), info


# ------------------------------------------------------------------------------------------------------ gradients
def bond_grad(dl, u, lam, Kn, Tv):
    """Per-slot derivatives of sum_s lam_s . K u_s, summed over the systems sharing each coefficient set.

    u, lam (..., N, d) float64; Kn/Tv (..., N, NN) broadcastable.  Returns (gKn, gTv) shaped like the coefficient
    sets (nset, N, NN).  SC: code-force operator; SQ: exact Hessian.
    """
    lead = u.shape[:-2]
    uf = _flat_vec(u.to(_F64), dl)
    lf = _flat_vec(lam.to(_F64), dl)
    nsys = uf.shape[0]
    Kc, rps = coef_sets(Kn.to(_F64), dl, lead)
    Tc, _ = coef_sets(Tv.to(_F64), dl, lead)
    nset = Kc.shape[0]
    gK = torch.empty_like(Kc)
    gT = torch.empty_like(Tc)
    lib = L.load()
    scr = _scratch(lib.lpm_grad_scratch_bytes(dl.ref, nsys), uf.device)
    b_ = _batch(nsys, rps)
    fn = lib.lpm_bond_grad_sc if dl.dim == 3 else lib.lpm_bond_grad_sq
    L.check(fn(dl.ref, L.ptr(uf), L.ptr(lf), L.ptr(Kc), L.ptr(Tc), L.LAYOUT_REF, ctypes.byref(b_), L.ptr(gK),
               L.ptr(gT), 0, L.ptr(scr), scr.numel(), L.stream_ptr(uf.device)), "lpm_bond_grad")
    return gK.reshape(nset, dl.N, dl.NN), gT.reshape(nset, dl.N, dl.NN)


# -------------------------------------------------------------------------------------------------- post-process
def stress(dl, u, Kn, Tv):
    """Particle stress (..., N, 6) [SC: xx yy zz yz xz xy] or (..., N, 3) [SQ: xx yy xy], FP64."""
    lead = u.shape[:-2]
    uf = _flat_vec(u.to(_F64), dl)
    nsys = uf.shape[0]
    Kc, rps = coef_sets(Kn.to(_F64), dl, lead)
    Tc, _ = coef_sets(Tv.to(_F64), dl, lead)
    nc = 6 if dl.dim == 3 else 3
    out = torch.empty((nsys, dl.N, nc), dtype=_F64, device=uf.device)
    lib = L.load()
    scr = _scratch(lib.lpm_kmv_scratch_bytes(dl.ref, L.LPM_F64, nsys), uf.device)
    b_ = _batch(nsys, rps)
    L.check(lib.lpm_stress_f64(dl.ref, L.ptr(uf), L.ptr(Kc), L.ptr(Tc), L.LAYOUT_REF, ctypes.byref(b_), L.ptr(dl.l0),
                               dl.V, L.ptr(out), L.ptr(scr), scr.numel(), L.stream_ptr(uf.device)), "lpm_stress_f64")
    return out.reshape(tuple(lead) + (dl.N, nc))


def energy(dl, u, Kn, Tv):
    """Particle energy (..., N), FP64."""
    lead = u.shape[:-2]
    uf = _flat_vec(u.to(_F64), dl)
    nsys = uf.shape[0]
    Kc, rps = coef_sets(Kn.to(_F64), dl, lead)
    Tc, _ = coef_sets(Tv.to(_F64), dl, lead)
    out = torch.empty((nsys, dl.N), dtype=_F64, device=uf.device)
    b_ = _batch(nsys, rps)
    L.check(L.load().lpm_energy_f64(dl.ref, L.ptr(uf), L.ptr(Kc), L.ptr(Tc), L.LAYOUT_REF, ctypes.byref(b_),
                                    L.ptr(out), L.stream_ptr(uf.device)), "lpm_energy_f64")
    return out.reshape(tuple(lead) + (dl.N,))


def post_vjp(dl, which, u, G, Kn, Tv):
    """VJP of the particle energy (which="energy", G (..., N)), the stress (which="stress", G (..., N, 6|3)) or, on the
    SC lattice, of K u (which="apply", G (..., N, 3): du = K^T G, exact for non-symmetric bond parameters).

    Returns (du shaped like u, gKn, gTv (nset, N, NN) summed over the systems of each coefficient set)."""
    lead = u.shape[:-2]
    uf = _flat_vec(u.to(_F64), dl)
    nsys = uf.shape[0]
    Kc, rps = coef_sets(Kn.to(_F64), dl, lead)
    Tc, _ = coef_sets(Tv.to(_F64), dl, lead)
    Gf = G.to(_F64).reshape((nsys, dl.N) if which == "energy" else (nsys, dl.N, -1)).contiguous()
    du = torch.empty_like(uf)
    gK = torch.empty_like(Kc)
    gT = torch.empty_like(Tc)
    lib = L.load()
    scr = _scratch(lib.lpm_grad_scratch_bytes(dl.ref, nsys), uf.device)
    b_ = _batch(nsys, rps)
    if which == "apply":
        rc = lib.lpm_kmv_vjp_f64(dl.ref, L.ptr(uf), L.ptr(Gf), L.ptr(Kc), L.ptr(Tc), L.LAYOUT_REF, ctypes.byref(b_),
                                 L.ptr(du), L.ptr(gK), L.ptr(gT), 0, L.ptr(scr), scr.numel(), L.stream_ptr(uf.device))
    elif which == "energy":
        rc = lib.lpm_energy_vjp_f64(dl.ref, L.ptr(uf), L.ptr(Gf), L.ptr(Kc), L.ptr(Tc), L.LAYOUT_REF, ctypes.byref(b_),
                                    L.ptr(du), L.ptr(gK), L.ptr(gT), 0, L.ptr(scr), scr.numel(), L.stream_ptr(uf.device))
    else:
        rc = lib.lpm_stress_vjp_f64(dl.ref, L.ptr(uf), L.ptr(Gf), L.ptr(Kc), L.ptr(Tc), L.LAYOUT_REF, ctypes.byref(b_),
                                    L.ptr(dl.l0), dl.V, L.ptr(du), L.ptr(gK), L.ptr(gT), 0, L.ptr(scr), scr.numel(),
                                    L.stream_ptr(uf.device))
    L.check(rc, "lpm_%s_vjp_f64" % which)
    return du.reshape(u.shape), gK, gT


def solid_tables(lat, solid):
    """Per-specimen bond tables (B, N, NN) int32 of the full box `lat` under solid masks (B, N) (bool CUDA tensor):
    a bond exists iff it is geometric and both ends are solid (cement3d/torch_v1.py:37-45)."""
    if not lat.full:
        raise ValueError("solid masks apply to the full box (void particles stay in the numbering)")
    L.require_cuda(solid)
    B = solid.shape[0]
    if tuple(solid.shape) != (B, lat.N):
        raise ValueError("solid mask must be (B, %d)" % lat.N)
    sm = solid.to(torch.uint8).contiguous()
    out = torch.empty((B, lat.N, lat.NN), dtype=torch.int32, device=solid.device)
    nz = lat.nz if lat.dim == 3 else 1
    L.check(L.load().lpm_solid_nbr(lat.dim, lat.nx, lat.ny, nz, B, L.ptr(sm), L.ptr(out),
                                   L.stream_ptr(solid.device)), "lpm_solid_nbr")
    return out


def build_nbr(lat, device="cuda"):
    """Neighbour table of `lat` computed on the device (int64, -1 = no bond): the reference's LatticeGeom.nbr."""
    dev = torch.device(device)
    site_of = torch.as_tensor(lat.site_of, device=dev, dtype=torch.int64)
    sites = torch.as_tensor(lat.sites, device=dev, dtype=torch.int64)
    out = torch.empty((lat.N, lat.NN), dtype=torch.int64, device=dev)
    nz = lat.nz if lat.dim == 3 else 1
    L.check(L.load().lpm_build_nbr(lat.dim, lat.nx, lat.ny, nz, lat.N, L.ptr(site_of), L.ptr(sites), L.ptr(out),
                                   L.stream_ptr(dev)), "lpm_build_nbr")
    return out
