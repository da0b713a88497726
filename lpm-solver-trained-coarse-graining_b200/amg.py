"""Aggregation-AMG preconditioner on the GPU (csrc/amg.cu) and the solvers that use it.

Drop-in mirror of timing/t3d/amg3d.py: ``AMGGeom`` (aggregation of one lattice and box of free particles) and ``AMG3D``
(numeric hierarchy of one specimen, ``vcycle()`` and ``pcg()``), plus the batched form ``AmgBatch`` that preconditions
every system of a batch of specimens x load cases with one hierarchy per (specimen, free box), as
timing/t3d/problems.py:112-132 builds one per BC set.  ``AMG_CFG`` is that file's tuned setting (problems.py:19).

The hierarchy is FP32; solves run FP32 PCG inner iterations inside an FP64 iterative refinement (``lpm_ir_amg``), so
``AMG3D.pcg`` returns an FP64 answer whose true residual meets ``tol`` -- the reference's stopping rule on the FP64
system.  Iteration counts are the total inner PCG iterations.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from . import core

AMG_CFG = dict(agg=3, coarse_max=1000, nu=1, gamma=2, power_its=5)  # timing/t3d/problems.py:19


def free_box(free, lat):
    """Inclusive site bounds (lo, hi) of a particle free mask, which must be a box (amg3d.py:450-452)."""
    f = np.asarray(free, bool).reshape(-1)
    fi = np.nonzero(f)[0]
    if len(fi) == 0:
        raise ValueError("the free set is empty")
    ijk = np.asarray(lat.ijk, np.int64)
    lo, hi = ijk[fi].min(0), ijk[fi].max(0)
    if int(np.prod(hi - lo + 1)) != len(fi):
        raise ValueError("free set must be a box")
    return lo.astype(np.int32), hi.astype(np.int32)


def boxes_of_masks(free_masks, lat):
    """Distinct free boxes of (nmask, N) particle masks, in order of first appearance, and the box of every mask."""
    boxes, of = [], []
    for f in np.asarray(free_masks, bool).reshape(-1, lat.N):
        lo, hi = free_box(f, lat)
        key = tuple(lo) + tuple(hi)
        if key not in boxes:
            boxes.append(key)
        of.append(boxes.index(key))
    return np.array(boxes, np.int32).reshape(-1, 6), np.array(of, np.int32)


def _grid_sizes(L_, agg, coarse_max, max_levels):
    """Grids of every level below the finest (amg3d.AMGGeom's chunk rule "merge")."""
    g = tuple(max(1, int(v) // agg) for v in L_)
    grids = [g]
    while 6 * int(np.prod(g)) > coarse_max and len(grids) - 1 < max_levels:
        g = tuple(max(1, v // agg) for v in g)
        grids.append(g)
    return grids


class AmgBatch:
    """CUDA AMG for a batch shape: ``nsys`` systems, ``rhs_per_set`` consecutive systems per coefficient set, particle
    free masks (nmask, N) (system s uses mask s % nmask; every mask a box).  ``setup()`` builds the numeric
    hierarchies from packed FP32 coefficients; ``apply``, ``pcg`` and ``ir`` precondition with them."""

    def __init__(self, dl, nsys, rhs_per_set, free_masks, agg=3, coarse_max=1000, max_levels=8, nu=1, nu_c=None,
                 gamma=2, w_from=1, power_its=5, omega=1.32, rho0_per_box=False):
        if dl.dim != 3 or dl.nbr is not None:
            raise L.LPMError("the AMG preconditioner needs a full simple-cubic box")
        self.dl = dl
        self.nsys, self.rps = int(nsys), int(rhs_per_set)
        fm = np.asarray(free_masks, bool).reshape(-1, dl.N)
        self.nmask = fm.shape[0]
        self.boxes, self.box_of_mask = boxes_of_masks(fm, dl.lat)
        self.nset = (self.nsys + self.rps - 1) // self.rps
        o = L.AmgOpts()
        L.load().lpm_amg_default_opts(ctypes.byref(o))
        o.agg, o.coarse_max, o.max_levels, o.nu = int(agg), int(coarse_max), int(max_levels), int(nu)
        o.nu_c = int(nu if nu_c is None else nu_c)
        o.gamma, o.w_from, o.power_its, o.omega = int(gamma), int(w_from), int(power_its), float(omega)
        o.rho0_per_box = int(bool(rho0_per_box))
        self.opts = o
        self._h = ctypes.c_void_p(None)
        b = core._batch(self.nsys, self.rps, self.nmask)
        with torch.cuda.device(dl.device):
            L.check(L.load().lpm_amg_create(dl.ref, ctypes.byref(b), self.boxes.ctypes.data_as(ctypes.c_void_p),
                                            len(self.boxes), self.box_of_mask.ctypes.data_as(ctypes.c_void_p),
                                            ctypes.byref(o), ctypes.byref(self._h)), "lpm_amg_create")
        self.mask = core.dof_masks(torch.as_tensor(fm, device=dl.device), dl, (self.nmask,))[0]
        self.ready = False

    # ------------------------------------------------------------------------------------------- lifetime
    def close(self):
        if self._h is not None and self._h.value:
            L.load().lpm_amg_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------------------------------------- setup
    def setup(self, K32, T32, M32, rho0=None):
        """Numeric hierarchies: K32/T32 packed FP32 (nset, 18, N), M32 FP32 block-Jacobi inverse (nset, N, 3, 3).
        rho0 (optional, per set) replaces the finest-level estimate (amg3d.AMG3D's rho0)."""
        st = L.stream_ptr(self.dl.device)
        L.check(L.load().lpm_amg_setup(self._h, L.ptr(K32), L.ptr(T32), L.ptr(M32.contiguous()), st),
                "lpm_amg_setup")
        self.ready = True
        if rho0 is not None:
            r = np.ascontiguousarray(np.broadcast_to(np.asarray(rho0, np.float64),
                                                     (self.nset * self._nb0(),)))
            L.check(L.load().lpm_amg_set_rho0(self._h, r.ctypes.data_as(ctypes.c_void_p), st), "lpm_amg_set_rho0")

    def _nb0(self):
        return len(self.boxes) if self.opts.rho0_per_box else 1

    def rho0(self):
        r = np.zeros(self.nset * self._nb0())
        L.check(L.load().lpm_amg_get_rho0(self._h, r.ctypes.data_as(ctypes.c_void_p)), "lpm_amg_get_rho0")
        return r

    def grids(self, box=0):
        nl = ctypes.c_int32(0)
        g = (ctypes.c_int32 * 30)()
        nb = ctypes.c_int64(0)
        L.check(L.load().lpm_amg_info(self._h, int(box), ctypes.byref(nl), g, ctypes.byref(nb)), "lpm_amg_info")
        return [tuple(g[3 * l:3 * l + 3]) for l in range(nl.value)], int(nb.value)

    def level(self, box, set_, level):
        """(A (nodes, 27, 6, 6) FP32, rho) of level `level` (1-based) of hierarchy (set, box)."""
        grids, _ = self.grids(box)
        n = int(np.prod(grids[level - 1]))
        A = np.zeros((n, 27, 6, 6), np.float32)
        rho = ctypes.c_double(0.0)
        L.check(L.load().lpm_amg_get_level(self._h, int(box), int(set_), int(level), A.ctypes.data_as(ctypes.c_void_p),
                                           ctypes.byref(rho), None), "lpm_amg_get_level")
        return A, rho.value

    # ------------------------------------------------------------------------------------------ launch counts
    def _cycle_launches(self):
        """Kernel launches of one finest-level cycle (csrc/amg.cu fine_cycle), from the level structure."""
        o = self.opts
        total = 2                                   # residual and smoothing epilogues of the pair operator
        for k in range(len(self.boxes)):
            nlev = len(self.grids(k)[0])

            def vc(l):
                if l == nlev - 1:
                    return 1                        # dense coarsest level
                return 1 + (o.nu_c - 1) + 1 + 1 + coarse(l + 1) + 1 + o.nu_c

            def coarse(l):
                n = vc(l)
                if l < nlev - 1 and l + 1 >= o.w_from:
                    n += (o.gamma - 1) * (1 + vc(l))
                return n
            total += 2 + coarse(0)                  # restriction, coarse levels, prolongation of the box
        return total

    def launches(self, inner_iters, inner_solves, outer_steps):
        """Kernel launches of this library in one setup + mixed-precision solve with the given counts."""
        o = self.opts
        cyc = self._cycle_launches()
        setup = 1 + 1 + 2 * o.power_its + 2
        for k in range(len(self.boxes)):
            grids = self.grids(k)[0]
            nc = 6 * int(np.prod(grids[-1]))
            nbk = -(-nc // 32)
            setup += 27 // 3 * 3 + (len(grids) - 1) * (5 + 2 * o.power_its) + 3 + 4 * nbk
        per_iter = 3 + cyc
        per_solve = 3 + cyc
        per_outer = 4
        return setup + inner_iters * per_iter + inner_solves * per_solve + outer_steps * per_outer + 2

    # ------------------------------------------------------------------------------------------- applications
    def apply(self, r):
        """z = B r for every system: r (nsys, N, 3) FP32 CUDA tensor."""
        r = r.reshape(self.nsys, self.dl.N, 3).to(torch.float32).contiguous()
        z = torch.empty_like(r)
        L.check(L.load().lpm_amg_apply(self._h, L.ptr(r), L.ptr(z), L.stream_ptr(self.dl.device)), "lpm_amg_apply")
        return z

    def pcg(self, b, tol, maxit=2000, check=1, poll=10, tol_sys=None):
        """FP32 AMG-PCG from zero: b (nsys, N, 3) FP32.  Returns (x, SolveInfo)."""
        dev = self.dl.device
        b = b.reshape(self.nsys, self.dl.N, 3).to(torch.float32).contiguous()
        x = torch.empty_like(b)
        it = torch.zeros(self.nsys, dtype=torch.int32, device=dev)
        rel = torch.zeros(self.nsys, dtype=torch.float64, device=dev)
        st = torch.zeros(self.nsys, dtype=torch.int32, device=dev)
        ts = None if tol_sys is None else torch.as_tensor(tol_sys, dtype=torch.float64, device=dev).contiguous()
        opts = L.CgOpts(float(tol), int(maxit), int(check), int(poll), 0, None,
                        None if ts is None else ts.data_ptr())
        L.check(L.load().lpm_amg_pcg_f32(self._h, L.ptr(b), L.ptr(x), ctypes.byref(opts), L.ptr(it), L.ptr(rel),
                                         L.ptr(st), L.stream_ptr(dev)), "lpm_amg_pcg_f32")
        return x, core.SolveInfo(it.cpu().numpy(), rel.cpu().numpy(), st.cpu().numpy())

    def ir(self, Kn64, Tv64, b, tol=1e-8, inner_tol=1e-3, maxit=20000, max_outer=20, check=1, poll=10, prof=None,
           packed=False):
        """Mixed-precision solve with the AMG-PCG inner solver: Kn64/Tv64 FP64 coefficient sets (nset, N, 18) in the
        reference layout (packed=True: already packed to (nset, 18, N) by core.pack), b (nsys, N, 3) FP64 zero on
        fixed DOFs.  Returns (x, SolveInfo)."""
        dl = self.dl
        bf = b.reshape(self.nsys, dl.N, 3).to(torch.float64).contiguous()
        # FP64 residuals on the TMA operator: packed (nset, 18, N) coefficients
        if packed:
            Kc, Tc = Kn64.contiguous(), Tv64.contiguous()
        else:
            Kc = core.pack(Kn64.reshape(-1, dl.N, dl.NN), torch.float64)
            Tc = core.pack(Tv64.reshape(-1, dl.N, dl.NN), torch.float64)
        xf = torch.zeros_like(bf)
        lib = L.load()
        b_ = core._batch(self.nsys, self.rps, self.nmask)
        ws = core._scratch(lib.lpm_ir_workspace_bytes(dl.ref, ctypes.byref(b_), 0), bf.device)
        it = torch.zeros(self.nsys, dtype=torch.int32, device=bf.device)
        rel = torch.zeros(self.nsys, dtype=torch.float64, device=bf.device)
        st = torch.zeros(self.nsys, dtype=torch.int32, device=bf.device)
        outer = ctypes.c_int32(0)
        opts = L.IrOpts(float(tol), float(inner_tol), int(maxit), int(max_outer), int(check), int(poll),
                        core._prof_ptr(prof), 1, 0)
        L.check(lib.lpm_ir_amg(dl.ref, L.ptr(Kc), L.ptr(Tc), L.LAYOUT_SOA, self._h, ctypes.byref(b_),
                               L.ptr(self.mask), L.ptr(bf), L.ptr(xf), ctypes.byref(opts), L.ptr(ws), ws.numel(),
                               L.ptr(it), L.ptr(rel), L.ptr(st), ctypes.byref(outer), L.stream_ptr(bf.device)),
                "lpm_ir_amg")
        return xf.reshape(b.shape), core.SolveInfo(it.cpu().numpy(), rel.cpu().numpy(), st.cpu().numpy(),
                                                   int(outer.value))


# ------------------------------------------------------------------------------------ reference-named mirror
class AMGGeom:
    """Aggregation of one lattice and one box of free particles (amg3d.AMGGeom, timing/t3d/amg3d.py:440-497).  The
    aggregation and transfers are built on the device when an AMG3D uses this geometry."""

    def __init__(self, lat, free, agg=3, rule="merge", coarse_max=3000, max_levels=8):
        if rule != "merge":
            raise ValueError("only the aggregate rule 'merge' is implemented")
        self.lat, self.free = lat, np.asarray(free, bool)
        self.agg, self.rule, self.coarse_max, self.max_levels = agg, rule, coarse_max, max_levels
        self.lo, self.hi = free_box(self.free, lat)
        self.grids = _grid_sizes(self.hi - self.lo + 1, agg, coarse_max, max_levels)
        self.g_coarsest = self.grids[-1]

    def describe(self):
        s = ["L0 N=%d free=%d" % (self.lat.N, int(self.free.sum()))]
        for k, g in enumerate(self.grids):
            s.append("L%d %s n=%d" % (k + 1, g, 6 * int(np.prod(g))))
        return " | ".join(s)


class AMG3D:
    """Numeric hierarchy of one specimen on an AMGGeom (amg3d.AMG3D, timing/t3d/amg3d.py:522-668): ``vcycle(b)`` is
    the preconditioner, ``pcg(b, tol)`` the solver.  Kn, Tv: (N, 18) FP64 (NumPy or CUDA tensors)."""

    def __init__(self, geom, Kn, Tv, nu=1, omega=1.32, power_its=10, Minv0=None, nu_c=None, gamma=1,
                 fine_additive=False, w_from=1, rho0=None, device="cuda"):
        if fine_additive:
            raise ValueError("the additive finest-level correction is not implemented (multiplicative only)")
        self.geom = geom
        self.dl = core.DeviceLattice(geom.lat, device)
        dev = self.dl.device
        self.Kn = torch.as_tensor(np.asarray(Kn) if not torch.is_tensor(Kn) else Kn, dtype=torch.float64,
                                  device=dev).reshape(1, geom.lat.N, 18).contiguous()
        self.Tv = torch.as_tensor(np.asarray(Tv) if not torch.is_tensor(Tv) else Tv, dtype=torch.float64,
                                  device=dev).reshape(1, geom.lat.N, 18).contiguous()
        self.batch = AmgBatch(self.dl, 1, 1, geom.free[None], agg=geom.agg, coarse_max=geom.coarse_max,
                              max_levels=geom.max_levels, nu=nu, nu_c=nu_c, gamma=gamma, w_from=w_from,
                              power_its=power_its, omega=omega)
        K32, T32 = core.pack(self.Kn, torch.float32), core.pack(self.Tv, torch.float32)
        if Minv0 is None:
            M32 = core.block_jacobi(self.dl, self.Kn, self.Tv, torch.float32)
        else:
            M32 = torch.as_tensor(np.asarray(Minv0) if not torch.is_tensor(Minv0) else Minv0, dtype=torch.float32,
                                  device=dev).reshape(1, geom.lat.N, 3, 3)
        self.batch.setup(K32, T32, M32, rho0=rho0)
        self.rho0 = float(self.batch.rho0()[0])
        self.rho = [self.batch.level(0, 0, l)[1] for l in range(1, len(geom.grids))]

    def vcycle(self, b):
        """b (N, 3), zero on fixed particles -> z (N, 3) (same container type as b)."""
        tb = torch.as_tensor(np.asarray(b) if not torch.is_tensor(b) else b, device=self.dl.device)
        z = self.batch.apply(tb.reshape(1, -1, 3).to(torch.float32))[0].to(torch.float64)
        return z if torch.is_tensor(b) else z.cpu().numpy()

    def pcg(self, b, tol, maxit=2000):
        """K_ff x = b (b (N, 3) zero on fixed) to ||b - K x|| <= tol ||b|| in FP64.  Returns (x, iterations,
        relres)."""
        tb = torch.as_tensor(np.asarray(b) if not torch.is_tensor(b) else b, dtype=torch.float64,
                             device=self.dl.device)
        x, info = self.batch.ir(self.Kn, self.Tv, tb.reshape(1, -1, 3), tol=tol, maxit=maxit)
        x = x[0]
        return (x if torch.is_tensor(b) else x.cpu().numpy()), int(info.iters[0]), float(info.relres[0])
