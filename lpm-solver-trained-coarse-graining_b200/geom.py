"""Lattice geometry, connectivity, boundary conditions and material maps (host side, NumPy).

Everything here is set-up work that runs once per lattice size or per specimen; the per-iteration work lives in the
CUDA library.  The arrays produced match the reference bit for bit where they are integer (connectivity) and to
round-off where they are floating point:

* simple-cubic lattice: ``coarse3d/geom3d.py:16-65`` (``SC_OFFS``, ``SC_SHELL``, ``LatticeGeom``)
* square lattice:       ``coarse2d/lin2d.py:21-74`` (``SQ_OFFS``, ``Lattice2D``), ``coarse2d/torch_lpm.py:59-89``
* load cases / BCs:     ``coarse3d/geom3d.py:25-106``, ``coarse2d/torch_lpm.py:92-111``, ``timing/t2d/el_prob.py:44-63``
* material maps:        ``coarse3d/geom3d.py:153-227``, ``coarse2d/lin2d.py:186-219``, ``coarse2d/cg.py:201-234``

Slot conventions (shared with the kernels in ``csrc/lpm_lattice.cuh``): slots come in reverse pairs ``(k, k^1)``;
shell 0 holds the axial bonds, shell 1 the diagonal ones; ``ndir[k] = -offs[k] / |offs[k]|`` so that
``dL_ik = ndir[k] . (u_i - u_q)`` with ``q = i + offs[k]``.
"""
import numpy as np

# ----------------------------------------------------------------------------------------------------------------------
# simple-cubic lattice (18 slots)
# ----------------------------------------------------------------------------------------------------------------------
SC_OFFS = np.array([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
                    (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0),
                    (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
                    (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1)], np.int64)
SC_SHELL = np.where(np.abs(SC_OFFS).sum(1) == 1, 0, 1).astype(np.int64)
NSLOT = 18
DIR_OF_SLOT = np.arange(NSLOT) // 2
FWD_SLOTS = np.arange(0, NSLOT, 2)

EPS = 1e-3
LOADS = ["k_xx", "k_yy", "k_zz", "k_yz", "k_xz", "k_xy", "tb_tz", "tb_sx", "lr_tx"]
RING = LOADS[:6]
PLATES = LOADS[6:]
BCSET = {ld: "ring" for ld in RING}
BCSET.update(tb_tz="tb", tb_sx="tb", lr_tx="lr")
GDIR = {"tb_tz": 2, "tb_sx": 0, "lr_tx": 0}
VOIGT_PAIRS = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]
# y-direction uniaxial tension between the J = 0 and J = ncy-1 block layers.  The reference has grips on K (tb_*) and
# I (lr_tx) only; this one completes the three uniaxial tensions of the 192^3 workload.
EXTRA_LOADS = ["fb_ty"]
GDIR_EXTRA = {"fb_ty": 1}


def _site_coords(nx, ny, nz):
    s = np.arange(nx * ny * nz, dtype=np.int64)
    return s % nx, (s // nx) % ny, s // (nx * ny)


class LatticeGeom:
    """Regular SC lattice of ``nx*ny*nz`` voxel sites with spacing ``h`` and an optional active-site mask.

    Site id of voxel ``(i, j, k)`` is ``(k*ny + j)*nx + i``; only active sites are numbered (in site order).
    Attributes mirror ``coarse3d/geom3d.py:35-65``: ``nbr (N,18) int64`` (-1 = no bond), ``valid``, ``ndir``, ``l0``,
    ``opp``, ``ijk``, ``x``, ``V``, ``site_of``, ``sites``, ``nb_initial``.
    """

    dim = 3

    def __init__(self, nx, ny, nz, h=1.0, origin=(0.0, 0.0, 0.0), active=None):
        self.nx, self.ny, self.nz, self.h = int(nx), int(ny), int(nz), h
        nsite = self.nx * self.ny * self.nz
        act = np.ones(nsite, bool) if active is None else np.asarray(active, bool).reshape(-1)
        if act.size != nsite:
            raise ValueError("active mask has %d entries, lattice has %d sites" % (act.size, nsite))
        self.full = bool(act.all())
        self.active = act
        self.sites = np.flatnonzero(act)
        self.site_of = np.full(nsite, -1, np.int64)
        self.site_of[self.sites] = np.arange(self.sites.size, dtype=np.int64)
        ci, cj, ck = _site_coords(self.nx, self.ny, self.nz)
        ii, jj, kk = ci[self.sites], cj[self.sites], ck[self.sites]
        self.ijk = np.ascontiguousarray(np.stack([ii, jj, kk], 1))
        self.x = (self.ijk + 0.5) * h + np.asarray(origin, float)[None, :]
        self.N = int(self.sites.size)
        self.V = h ** 3
        self.offs, self.shell, self.NN = SC_OFFS, SC_SHELL, NSLOT
        self.opp = np.arange(NSLOT) ^ 1
        length = np.sqrt((SC_OFFS ** 2).sum(1).astype(float))
        self.l0 = length * h
        self.ndir = np.ascontiguousarray(-SC_OFFS / length[:, None])
        qi = ii[:, None] + SC_OFFS[None, :, 0]
        qj = jj[:, None] + SC_OFFS[None, :, 1]
        qk = kk[:, None] + SC_OFFS[None, :, 2]
        inside = (qi >= 0) & (qi < self.nx) & (qj >= 0) & (qj < self.ny) & (qk >= 0) & (qk < self.nz)
        qsite = np.where(inside, (qk * self.ny + qj) * self.nx + qi, 0)
        q = self.site_of[qsite]
        ok = inside & (q >= 0)
        self.nbr = np.ascontiguousarray(np.where(ok, q, -1).astype(np.int64))
        self.valid = ok
        self.nb_initial = ok.sum(1)


# ----------------------------------------------------------------------------------------------------------------------
# square lattice (8 slots)
# ----------------------------------------------------------------------------------------------------------------------
SQ_OFFS = np.array([(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, -1), (1, -1), (-1, 1)], np.int64)
SQ_SHELL = np.where(np.abs(SQ_OFFS).sum(1) == 1, 0, 1).astype(np.int64)
SQ_NSLOT = 8


class Lattice2D:
    """Regular square lattice of ``nx*ny`` pixel sites, spacing ``h``; particle id ``j*nx + i`` over active sites.

    Mirrors ``coarse2d/lin2d.py:29-74`` for ``kind="square"`` (the only lattice of the 2D hot path).
    """

    dim = 2

    def __init__(self, kind, nx, ny, h, origin=(0.0, 0.0), active=None):
        if kind != "square":
            raise NotImplementedError("only the square lattice is on the GPU path (got %r)" % (kind,))
        self.kind, self.nx, self.ny, self.h = kind, int(nx), int(ny), h
        nsite = self.nx * self.ny
        act = np.ones(nsite, bool) if active is None else np.asarray(active, bool).reshape(-1)
        if act.size != nsite:
            raise ValueError("active mask has %d entries, lattice has %d sites" % (act.size, nsite))
        self.full = bool(act.all())
        self.active = act
        self.sites = np.flatnonzero(act)
        self.site_of = np.full(nsite, -1, np.int64)
        self.site_of[self.sites] = np.arange(self.sites.size, dtype=np.int64)
        s = self.sites
        ii, jj = s % self.nx, s // self.nx
        self.ij = np.stack([ii, jj], 1)
        self.x = np.stack([(ii + 0.5) * h + origin[0], (jj + 0.5) * h + origin[1]], 1)
        self.V = h * h
        self.N = int(s.size)
        self.offs, self.shell = SQ_OFFS, SQ_SHELL
        self.NN = SQ_NSLOT
        self.opp = np.arange(SQ_NSLOT) ^ 1
        length = np.sqrt((SQ_OFFS ** 2).sum(1).astype(float))
        self.l0 = length * h
        self.ndir = -SQ_OFFS / length[:, None]
        qi = ii[:, None] + SQ_OFFS[None, :, 0]
        qj = jj[:, None] + SQ_OFFS[None, :, 1]
        inside = (qi >= 0) & (qi < self.nx) & (qj >= 0) & (qj < self.ny)
        q = self.site_of[np.where(inside, qj * self.nx + qi, 0)]
        ok = inside & (q >= 0)
        self.nbr = np.where(ok, q, -1)
        self.valid = ok
        self.nb_initial = ok.sum(1)


class SquareLattice(Lattice2D):
    """Full square lattice with the constructor order of ``coarse2d/torch_lpm.py:59-89`` (nx, ny, h, kind, origin)."""

    def __init__(self, nx, ny, h, kind="square", origin=(0.0, 0.0)):
        super().__init__(kind, nx, ny, h, origin)


# ----------------------------------------------------------------------------------------------------------------------
# load cases (3D): coarse3d/geom3d.py:67-106
# ----------------------------------------------------------------------------------------------------------------------
def unit_strain(k):
    """Strain tensor of Voigt component ``k`` (engineering shear: gamma = 1 gives eps_ab = 1/2)."""
    a, b = VOIGT_PAIRS[k]
    e = np.zeros((3, 3))
    e[a, b] += 0.5
    e[b, a] += 0.5
    return e


def affine_disp(x, eps, x0=None):
    """u = eps (x - x0) row-wise; works for 2D and 3D points."""
    x = np.asarray(x, float)
    x0 = np.zeros(x.shape[1]) if x0 is None else np.asarray(x0, float)
    return (x - x0[None, :]) @ np.asarray(eps, float).T


def prescribed(load, x, IJK, nc, s, h=1.0):
    """BCs of a 3D load case on whole blocks: ``(fixed (N,) bool, u_presc (N,3), moving grip (N,) bool or None)``.

    ``IJK`` is the block index of every particle and ``nc = (ncx, ncy, ncz)`` the number of blocks.  Ring loads
    prescribe the affine KUBC field on the outer block layer; plate loads clamp one grip and translate the other.
    """
    ncx, ncy, ncz = nc
    I, J, K = IJK[:, 0], IJK[:, 1], IJK[:, 2]
    u = np.zeros((len(x), 3))
    if load in RING:
        fixed = (I < 1) | (I >= ncx - 1) | (J < 1) | (J >= ncy - 1) | (K < 1) | (K >= ncz - 1)
        centre = 0.5 * np.array([ncx, ncy, ncz], float) * s * h
        u[fixed] = affine_disp(x[fixed], EPS * unit_strain(RING.index(load)), centre)
        return fixed, u, None
    if load in ("tb_tz", "tb_sx"):
        clamp, grip = K < 1, K >= ncz - 1
        travel = EPS * (ncz - 1) * s * h
        d = (0.0, 0.0, travel) if load == "tb_tz" else (travel, 0.0, 0.0)
    elif load == "lr_tx":
        clamp, grip = I < 1, I >= ncx - 1
        d = (EPS * (ncx - 1) * s * h, 0.0, 0.0)
    elif load == "fb_ty":
        clamp, grip = J < 1, J >= ncy - 1
        d = (0.0, EPS * (ncy - 1) * s * h, 0.0)
    else:
        raise ValueError("unknown load case %r" % (load,))
    u[grip] = np.asarray(d)
    return clamp | grip, u, grip


def free_surface_cells(load, nc):
    """Free cells of a plate case that lie on a free lateral face (``coarse3d/geom3d.py:109-120``)."""
    ncx, ncy, ncz = nc
    I, J, K = _site_coords(ncx, ncy, ncz)
    if load.startswith("tb"):
        grip = (K < 1) | (K >= ncz - 1)
        face = (I < 1) | (I >= ncx - 1) | (J < 1) | (J >= ncy - 1)
    else:
        grip = (I < 1) | (I >= ncx - 1)
        face = (J < 1) | (J >= ncy - 1) | (K < 1) | (K >= ncz - 1)
    return face & ~grip


def interface_cells(phase, n, s):
    """Cells of size s whose block holds a voxel with a 6-neighbour of the other phase (coarse3d/geom3d.py:134-147)."""
    p = np.asarray(phase).reshape(n, n, n)
    b = np.zeros(p.shape, bool)
    for ax in range(3):
        d = np.diff(p, axis=ax) != 0
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(1, None)
        hi[ax] = slice(None, -1)
        b[tuple(lo)] |= d
        b[tuple(hi)] |= d
    nc = n // s
    return b.reshape(nc, s, nc, s, nc, s).any(axis=(1, 3, 5)).ravel()


def cell_ijk(nc):
    I, J, K = _site_coords(*nc)
    return np.stack([I, J, K], 1)


def block_index(ijk, s, nc):
    B = ijk // s
    return (B[:, 2] * nc[1] + B[:, 1]) * nc[0] + B[:, 0]


# ----------------------------------------------------------------------------------------------------------------------
# load cases (2D): coarse2d/torch_lpm.py:92-111 (== timing/t2d/el_prob.py:44-63 and coarse2d/cg.py:40-61 for L = 1)
# ----------------------------------------------------------------------------------------------------------------------
LOADS2D = ["ring_xx", "ring_yy", "ring_xy", "tb_ty", "tb_sx", "lr_tx"]
BCSET2D = {"ring_xx": "ring", "ring_yy": "ring", "ring_xy": "ring", "tb_ty": "tb", "tb_sx": "tb", "lr_tx": "lr"}
_RING2D = {"ring_xx": ((1.0, 0.0), (0.0, 0.0)), "ring_yy": ((0.0, 0.0), (0.0, 1.0)), "ring_xy": ((0.0, 0.5), (0.5, 0.0))}


def prescribed2d(load, x, IJ, ncx, ncy, s, h, L=1):
    """BCs of a 2D load case on whole blocks with ``L`` block layers: ``(fixed, u_presc (N,2), moving or None)``."""
    I, J = IJ[:, 0], IJ[:, 1]
    u = np.zeros((len(x), 2))
    if load in _RING2D:
        fixed = (I < L) | (I >= ncx - L) | (J < L) | (J >= ncy - L)
        centre = 0.5 * np.array([ncx, ncy], float) * s * h
        u[fixed] = affine_disp(x[fixed], EPS * np.array(_RING2D[load]), centre)
        return fixed, u, None
    if load in ("tb_ty", "tb_sx"):
        clamp, grip = J < L, J >= ncy - L
        travel = EPS * (ncy - L) * s * h
        d = (0.0, travel) if load == "tb_ty" else (travel, 0.0)
    elif load == "lr_tx":
        clamp, grip = I < L, I >= ncx - L
        d = (EPS * (ncx - L) * s * h, 0.0)
    else:
        raise ValueError("unknown load case %r" % (load,))
    u[grip] = np.asarray(d)
    return clamp | grip, u, grip


def uniaxial_tension_2d(lat, strain=1e-3):
    """Per-DOF BCs of the 2D plain-CG workload: u_x = 0 on column i = 0, particle (0, 0) also pinned in y, and
    u_x = strain*(nx-1)*h on column i = nx-1 (grip distance as in ``timing/t2d/el_prob.py:59-61``).

    Returns ``(fixed_dof (N,2) bool, u_presc (N,2), moving (N,) bool)``.
    """
    i, j = lat.ij[:, 0], lat.ij[:, 1]
    fixed = np.zeros((lat.N, 2), bool)
    u = np.zeros((lat.N, 2))
    left, right = i == 0, i == lat.nx - 1
    fixed[left, 0] = True
    fixed[right, 0] = True
    fixed[left & (j == 0), 1] = True
    u[right, 0] = strain * (lat.nx - 1) * lat.h
    return fixed, u, right


# ----------------------------------------------------------------------------------------------------------------------
# materials -> bond parameters
# ----------------------------------------------------------------------------------------------------------------------
def iso_C(E, nu):
    """Isotropic 3D stiffness as (C11, C12, C44) (``coarse3d/geom3d.py:153-159``)."""
    E = np.asarray(E, float)
    nu = np.asarray(nu, float)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return np.stack([lam + 2 * mu, lam, mu], -1)


def iso_C2d(E, nu, plane="strain"):
    """Isotropic 2D stiffness (C11, C12, C66), plane strain or plane stress (``coarse2d/lin2d.py:186-194``)."""
    E = np.asarray(E, float)
    nu = np.asarray(nu, float)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu)) if plane == "strain" else E * nu / (1 - nu * nu)
    mu = E / (2 * (1 + nu))
    return np.stack([lam + 2 * mu, lam, mu], -1)


def sc_params_from_C(C, r):
    """SC lattice parameters (Kn1, Kn2, Tv) = r (C11-C12-C44, C44, (C12-C44)/18) (``coarse3d/geom3d.py:162-165``)."""
    C11, C12, C44 = C[..., 0], C[..., 1], C[..., 2]
    return np.stack([r * (C11 - C12 - C44), r * C44, r * (C12 - C44) / 18.0], -1)


def square_params_from_C(C):
    """Square lattice parameters (Kn1, Kn2, Tv) = ((C11-C12)/2, C44/2, (C12-C44)/12) (``coarse2d/lin2d.py:197-200``)."""
    C11, C12, C44 = C[..., 0], C[..., 1], C[..., 2]
    return np.stack([0.5 * (C11 - C12), 0.5 * C44, (C12 - C44) / 12.0], -1)


def bond_params_two_end_mean(lat, ppar):
    """Per-particle (Kn_axial, Kn_diag, Tv) -> per directed bond ``Kn, Tv (N, NN)``: mean of the two end particles,
    zero on missing bonds (``coarse3d/geom3d.py:168-176``, ``coarse2d/lin2d.py:210-219``)."""
    ppar = np.asarray(ppar, float)
    q = np.where(lat.valid, lat.nbr, 0)
    axial = (lat.shell == 0)[None, :]
    kn_own = np.where(axial, ppar[:, 0:1], ppar[:, 1:2])
    kn_far = np.where(axial, ppar[q, 0], ppar[q, 1])
    Kn = 0.5 * (kn_own + kn_far) * lat.valid
    Tv = 0.5 * (ppar[:, 2:3] + ppar[q, 2]) * lat.valid
    return np.ascontiguousarray(Kn), np.ascontiguousarray(Tv)


def iso_C66(C3):
    """(N, 3) (C11, C12, C44) -> (N, 6, 6) Voigt matrices (``coarse3d/geom3d.py:204-211``)."""
    C3 = np.asarray(C3, float)
    C = np.zeros((len(C3), 6, 6))
    C[:, :3, :3] = C3[:, 1, None, None]
    for a in range(3):
        C[:, a, a] = C3[:, 0]
        C[:, 3 + a, 3 + a] = C3[:, 2]
    return C


def cell_params_from_C66(C, r):
    """Anisotropic generalisation of the SC map (``coarse3d/geom3d.py:183-201``): 9 direction Kn + one Tv per cell."""
    c = lambda a, b: C[:, a - 1, b - 1]
    T = (c(1, 2) - c(6, 6) + c(1, 3) - c(5, 5) + c(2, 3) - c(4, 4)) / 3.0
    cols = [c(1, 1) - c(5, 5) - c(6, 6) - T, c(2, 2) - c(4, 4) - c(6, 6) - T, c(3, 3) - c(4, 4) - c(5, 5) - T,
            c(6, 6) + 0.5 * (c(1, 6) + c(2, 6)), c(6, 6) - 0.5 * (c(1, 6) + c(2, 6)),
            c(5, 5) + 0.5 * (c(1, 5) + c(3, 5)), c(5, 5) - 0.5 * (c(1, 5) + c(3, 5)),
            c(4, 4) + 0.5 * (c(2, 4) + c(3, 4)), c(4, 4) - 0.5 * (c(2, 4) + c(3, 4)), T / 18.0]
    return r * np.stack(cols, 1)


def bond_params_from_cells(lat_c, cp):
    """Two-end mean of per-cell (9 direction Kn, Tv) -> ``Kn, Tv (Nc, 18)`` (``coarse3d/geom3d.py:214-220``)."""
    q = np.where(lat_c.valid, lat_c.nbr, 0)
    Kn = 0.5 * (cp[:, DIR_OF_SLOT] + cp[q, DIR_OF_SLOT[None, :]]) * lat_c.valid
    Tv = 0.5 * (cp[:, 9:10] + cp[q, 9]) * lat_c.valid
    return np.ascontiguousarray(Kn), np.ascontiguousarray(Tv)


def voigt_cells(Cvox, n, s):
    """Block (Voigt) average of voxel (C11, C12, C44) -> (Nc, 6, 6) (``coarse3d/geom3d.py:223-227``)."""
    nc = n // s
    C = np.asarray(Cvox, float).reshape(nc, s, nc, s, nc, s, 3).mean(axis=(1, 3, 5)).reshape(-1, 3)
    return iso_C66(C)


# 2D coarse maps (coarse2d/cg.py:201-234)
SQ_SLOT_COL = np.array([0, 0, 1, 1, 2, 2, 3, 3])


def cell_params_from_C6(C6):
    """Per-cell (Kn_x, Kn_y, Kn_diag+, Kn_diag-, Tv) from (C11, C22, C12, C66, C16, C26)."""
    C11, C22, C12, C66, C16, C26 = [C6[:, k] for k in range(6)]
    return np.stack([0.5 * (C11 - C12), 0.5 * (C22 - C12), 0.5 * C66 + 0.25 * (C16 + C26),
                     0.5 * C66 - 0.25 * (C16 + C26), (C12 - C66) / 12.0], 1)


def bond_params_from_cells2d(lat_c, cp):
    q = np.where(lat_c.valid, lat_c.nbr, 0)
    Kn = 0.5 * (cp[:, SQ_SLOT_COL] + cp[q, SQ_SLOT_COL[None, :]]) * lat_c.valid
    Tv = 0.5 * (cp[:, 4:5] + cp[q, 4]) * lat_c.valid
    return Kn, Tv


def C6_from_C3(C3):
    z = np.zeros(len(C3))
    return np.stack([C3[:, 0], C3[:, 0], C3[:, 1], C3[:, 2], z, z], 1)


def voigt_cells2d(Cpix, nx, ny, s):
    C = np.asarray(Cpix, float).reshape(ny // s, s, nx // s, s, 3).mean(axis=(1, 3)).reshape(-1, 3)
    return C6_from_C3(C)
