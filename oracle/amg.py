"""Aggregation-AMG preconditioned CG of the SC lattice, restated in NumPy -- TEST INFRASTRUCTURE ONLY.

The checker of the CUDA AMG (csrc/amg.cu): a restatement of timing/t3d/amg3d.py (and of the two helpers it takes from
timing/t3d/gmg.py), FP64, with the finest operator from the C oracle (oracle/lpm_oracle.c).  Used by tests/ only; the
product path never imports it.  Pinned in tests/test_oracle.py against tests/golden/golden_amg.npz, which the
reference itself produced (tests/golden/make_golden.py, part "amg").

  chunk_index        amg3d.py:45-51      aggregate chunks per axis, rule "merge" (remainder joins the last chunk)
  tentative          gmg.py:70-142       per-aggregate modified Gram-Schmidt of the near-null-space rows
  rigid_modes        gmg.py:145-162      6 rigid-body modes about the mean of the free particles
  Geometry           amg3d.py:440-497    aggregation and tentative prolongators of every level (one box of free
                                         particles)
  galerkin0          amg3d.py:175-197    level-1 operator P^T K_ff P, here by probing K_ff with P restricted to 27
                                         colour classes of aggregates (aggregates at least 3 sites wide; the operator
                                         reaches 2 sites, so each probe meets one aggregate of its colour per row)
  st_galerkin        amg3d.py:253-295    Q^T A Q on 27-point 6x6-block stencils
  power_rho          amg3d.py:506-519    rho(D^-1 A) by power iteration from rng(0) (or, to check the CUDA
                                         hierarchy, from its counter-based start vectors: hash_normals)
  Hierarchy          amg3d.py:522-668    numeric setup, V/W-cycle (vcycle, _coarse, _vc) and PCG
"""
import math

import numpy as np
import scipy.linalg as sla

import oracle as O

OFF27 = np.array([(d % 3 - 1, (d // 3) % 3 - 1, d // 9 - 1) for d in range(27)], np.int64)


def chunk_index(L, a):
    """Chunk id of positions 0..L-1 along one axis and the number of chunks (amg3d.py:45-51, rule "merge")."""
    nch = max(1, L // a)
    return np.minimum(np.arange(L) // a, nch - 1), nch


def grid_ijk(g):
    gx, gy, gz = g
    k, j, i = np.meshgrid(np.arange(gz), np.arange(gy), np.arange(gx), indexing="ij")
    return np.stack([i.ravel(), j.ravel(), k.ravel()], 1).astype(np.int64)


def rigid_modes(X):
    """(3n, 6) rigid-body modes of the points X (n, 3) about their mean, rows interleaved by DOF (gmg.py:145-162)."""
    c = X - X.mean(0)
    n = len(X)
    B = np.zeros((3 * n, 6))
    for d in range(3):
        B[d::3, d] = 1.0
    B[0::3, 3], B[1::3, 3] = -c[:, 1], c[:, 0]
    B[1::3, 4], B[2::3, 4] = -c[:, 2], c[:, 1]
    B[0::3, 5], B[2::3, 5] = c[:, 2], -c[:, 0]
    return B


def tentative(agg_of_row, nagg, B, tol=1e-8):
    """Modified Gram-Schmidt of the rows of B (n, m) of every aggregate (gmg.py:70-142).

    Returns Q (n, m), the orthonormal columns restricted to each row's aggregate, and R (nagg, m, m).  Rows of one
    aggregate are taken in increasing row order.  Every column must be kept (no rank deficiency), as amg3d asserts.
    """
    n, m = B.shape
    order = np.argsort(agg_of_row, kind="stable")
    counts = np.bincount(agg_of_row, minlength=nagg)
    start = np.concatenate([[0], np.cumsum(counts)])
    Q = np.zeros((n, m))
    R = np.zeros((nagg, m, m))
    for k in np.unique(counts):
        if k == 0:
            continue
        aggs = np.nonzero(counts == k)[0]
        rows = order[start[aggs][:, None] + np.arange(k)[None, :]]  # (G, k)
        blk = B[rows]                                                # (G, k, m)
        scale = np.sqrt((blk ** 2).sum(1)).max(1)                   # (G,)
        q = np.zeros_like(blk)
        r = np.zeros((len(aggs), m, m))
        for c in range(m):
            v = blk[:, :, c].copy()
            for d in range(c):
                pr = (q[:, :, d] * v).sum(1)
                r[:, d, c] = pr
                v -= pr[:, None] * q[:, :, d]
            nrm = np.sqrt((v * v).sum(1))
            assert np.all((nrm > tol * scale) & (nrm > 0.0)), "rank-deficient aggregate"
            r[:, c, c] = nrm
            q[:, :, c] = v / nrm[:, None]
        Q[rows.ravel()] = q.reshape(-1, m)
        R[aggs] = r
    return Q, R


class Geometry:
    """Aggregation and tentative prolongators of all levels for one lattice and one box of free particles
    (amg3d.py:440-497)."""

    def __init__(self, lat, free, agg=3, coarse_max=1000, max_levels=8):
        self.lat, self.free = lat, np.asarray(free, bool)
        self.agg, self.coarse_max = agg, coarse_max
        fi = np.nonzero(self.free)[0]
        ijk = np.asarray(lat.ijk, np.int64)
        lo, hi = ijk[fi].min(0), ijk[fi].max(0)
        L = hi - lo + 1
        assert int(np.prod(L)) == len(fi), "free set must be a box"
        self.lo, self.L = lo, L
        ch = [chunk_index(int(L[d]), agg) for d in range(3)]
        g = tuple(int(c[1]) for c in ch)
        rel = ijk[fi] - lo
        agg_of = -np.ones(lat.N, np.int64)
        agg_of[fi] = (ch[2][0][rel[:, 2]] * g[1] + ch[1][0][rel[:, 1]]) * g[0] + ch[0][0][rel[:, 0]]
        nagg = g[0] * g[1] * g[2]
        B = rigid_modes(np.asarray(lat.x, np.float64)[fi])
        Qr, R = tentative(np.repeat(agg_of[fi], 3), nagg, B)
        P = np.zeros((lat.N, 3, 6))
        P[fi] = Qr.reshape(len(fi), 3, 6)
        self.g0, self.agg_of0, self.P = g, agg_of, P
        self.levels = []
        Bn = R
        while 6 * nagg > coarse_max and len(self.levels) < max_levels:
            chn = [chunk_index(g[d], agg) for d in range(3)]
            gc = tuple(int(c[1]) for c in chn)
            nij = grid_ijk(g)
            a_of = (chn[2][0][nij[:, 2]] * gc[1] + chn[1][0][nij[:, 1]]) * gc[0] + chn[0][0][nij[:, 0]]
            ncg = gc[0] * gc[1] * gc[2]
            Qn, Rn = tentative(np.repeat(a_of, 6), ncg, Bn.reshape(-1, 6))
            self.levels.append(dict(g=g, gc=gc, agg_of=a_of, Q=Qn.reshape(nagg, 6, 6)))
            g, nagg, Bn = gc, ncg, Rn
        self.grids = [self.g0] + [L_["gc"] for L_ in self.levels]


# ------------------------------------------------------------------------------------------- level operators
def restrict(P, agg_of, nagg, r):
    """rc[I] = sum_{i in I} P_i^T r_i (amg3d.py:298-310); items with agg_of < 0 are skipped."""
    ok = agg_of >= 0
    rc = np.zeros((nagg, P.shape[2]))
    np.add.at(rc, agg_of[ok], np.einsum("iac,ia->ic", P[ok], r[ok]))
    return rc


def prolong_add(P, agg_of, e, x):
    """x_i += P_i e[agg(i)] (amg3d.py:313-326)."""
    ok = agg_of >= 0
    x[ok] += np.einsum("iac,ic->ia", P[ok], e[agg_of[ok]])


def st_mv(A, g, x):
    """y = A x on a 27-point 6x6-block stencil of grid g (amg3d.py:232-250)."""
    ijk = grid_ijk(g)
    y = np.zeros_like(x)
    for d in range(27):
        j = ijk + OFF27[d]
        ok = np.all((j >= 0) & (j < np.array(g)), 1)
        J = (j[ok, 2] * g[1] + j[ok, 1]) * g[0] + j[ok, 0]
        y[ok] += np.einsum("nrc,nc->nr", A[ok, d], x[J])
    return y


def st_galerkin(A, g, Q, agg_of, gc):
    """Ac[I, dd] = sum_{n in I, m in J} Q_n^T A_nm Q_m (amg3d.py:253-295)."""
    ijk = grid_ijk(g)
    cijk = grid_ijk(gc)
    Ac = np.zeros((gc[0] * gc[1] * gc[2], 27, 6, 6))
    for d in range(27):
        j = ijk + OFF27[d]
        ok = np.nonzero(np.all((j >= 0) & (j < np.array(g)), 1))[0]
        m = (j[ok, 2] * g[1] + j[ok, 1]) * g[0] + j[ok, 0]
        I, J = agg_of[ok], agg_of[m]
        dv = cijk[J] - cijk[I] + 1
        dd = (dv[:, 2] * 3 + dv[:, 1]) * 3 + dv[:, 0]
        blk = np.einsum("nar,nab,nbc->nrc", Q[ok], A[ok, d], Q[m])
        np.add.at(Ac, (I, dd), blk)
    return Ac


def dense_from_stencil(A, g):
    n = A.shape[0]
    ijk = grid_ijk(g)
    D = np.zeros((n, 6, n, 6))
    for d in range(27):
        j = ijk + OFF27[d]
        ok = np.all((j >= 0) & (j < np.array(g)), 1)
        I = np.nonzero(ok)[0]
        J = (j[ok, 2] * g[1] + j[ok, 1]) * g[0] + j[ok, 0]
        D[I, :, J, :] = A[I, d]
    return D.reshape(6 * n, 6 * n)


def bj(M, r, w):
    return w * np.einsum("nab,nb->na", M, r)


def _mix64(z):
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def hash_normals(level, shape):
    """The counter-based normals that the CUDA power iterations start from (csrc/amg.cu start_normal): element e of
    level `level` (0 = finest) from the splitmix64 finaliser and Box-Muller, rounded to FP32 as the device does."""
    n = int(np.prod(shape))
    with np.errstate(over="ignore"):
        e = np.arange(n, dtype=np.uint64)
        k = (np.uint64(level + 1) << np.uint64(56)) ^ (e << np.uint64(1))
        u1 = ((_mix64(k) >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
        u2 = ((_mix64(k | np.uint64(1)) >> np.uint64(11)).astype(np.float64) + 0.5) * 2.0 ** -53
    z = np.sqrt(-2.0 * np.log(u1)) * np.cos(6.283185307179586 * u2)
    return z.astype(np.float32).astype(np.float64).reshape(shape)


def power_rho(mv, Minv, shape, its, seed=0, start=None):
    """rho(D^-1 A) by `its` power steps from rng(seed) normals (or the given start) pre-multiplied by Minv
    (amg3d.py:506-519)."""
    x0 = np.random.default_rng(seed).standard_normal(shape) if start is None else start
    x = bj(Minv, x0, 1.0)
    lam = 1.0
    for _ in range(its):
        x = x / np.linalg.norm(x)
        y = bj(Minv, mv(x), 1.0)
        lam = float(np.linalg.norm(y))
        x = y
    return lam


def galerkin0(geo, Kn, Tv):
    """A1 (nagg, 27, 6, 6) = P^T K_ff P by 162 probes of the finest operator."""
    lat, P, agg_of, g = geo.lat, geo.P, geo.agg_of0, geo.g0
    nagg = g[0] * g[1] * g[2]
    aijk = grid_ijk(g)
    A1 = np.zeros((nagg, 27, 6, 6))
    ok = agg_of >= 0
    for col in range(27):
        cx, cy, cz = col % 3, (col // 3) % 3, col // 9
        sel = np.zeros(lat.N, bool)
        sel[ok] = ((aijk[agg_of[ok], 0] % 3 == cx) & (aijk[agg_of[ok], 1] % 3 == cy) &
                   (aijk[agg_of[ok], 2] % 3 == cz))
        # the colour-col neighbour J of every aggregate I: offset in {-1, 0, 1} with (I + off) % 3 == colour
        off = (np.array([cx, cy, cz])[None, :] - aijk) % 3
        off = np.where(off == 2, -1, off)
        jn = aijk + off
        valid = np.all((jn >= 0) & (jn < np.array(g)), 1)
        dd = ((off[:, 2] + 1) * 3 + off[:, 1] + 1) * 3 + off[:, 0] + 1
        for c in range(6):
            v = np.where(sel[:, None], P[:, :, c], 0.0)
            y = O.sc_apply(lat, v, Kn, Tv)
            y[~geo.free] = 0.0
            rc = restrict(P, agg_of, nagg, y)
            A1[np.nonzero(valid)[0], dd[valid], :, c] = rc[valid]
    return A1


class Hierarchy:
    """Numeric hierarchy of one specimen on a Geometry (amg3d.py:522-668): vcycle() is the preconditioner, pcg() the
    solver.  Defaults are timing/t3d/problems.py:19 (AMG_CFG) apart from the geometry's agg and coarse_max."""

    def __init__(self, geo, Kn, Tv, nu=1, omega=1.32, power_its=5, Minv0=None, nu_c=None, gamma=2, w_from=1,
                 rho0=None, start="numpy"):
        self.geo, self.Kn, self.Tv = geo, np.asarray(Kn, np.float64), np.asarray(Tv, np.float64)
        self.nu, self.omega = nu, omega
        self.nu_c = nu if nu_c is None else nu_c
        self.gamma, self.w_from = gamma, w_from
        lat = geo.lat
        self.N = lat.N
        free = geo.free
        if Minv0 is None:
            Minv0 = O.block_jacobi3(O.sc_block_diag(lat, self.Kn, self.Tv), free)
        else:
            Minv0 = Minv0 * free[:, None, None]
        self.M0 = Minv0
        st = (lambda lvl, shape: None) if start == "numpy" else hash_normals
        self.rho0 = power_rho(self.apply0, self.M0, (self.N, 3), power_its, start=st(0, (self.N, 3))) \
            if rho0 is None else rho0
        self.A = [galerkin0(geo, self.Kn, self.Tv)]
        self.Minv, self.rho = [], []
        for k, Lg in enumerate(geo.levels):
            A = self.A[-1]
            Mi = np.linalg.inv(A[:, 13])
            self.Minv.append(Mi)
            self.rho.append(power_rho(lambda x, A=A, g=Lg["g"]: st_mv(A, g, x), Mi, (A.shape[0], 6), power_its,
                                      start=st(k + 1, (A.shape[0], 6))))
            self.A.append(st_galerkin(A, Lg["g"], Lg["Q"], Lg["agg_of"], Lg["gc"]))
        D = dense_from_stencil(self.A[-1], geo.grids[-1])
        self.cho = sla.cho_factor(0.5 * (D + D.T), lower=False, check_finite=False)

    def apply0(self, x):
        y = O.sc_apply(self.geo.lat, x, self.Kn, self.Tv)
        y[~self.geo.free] = 0.0
        return y

    def _coarse(self, lvl, rc):
        ec = self._vc(lvl, rc)
        k = lvl - 1
        if k == len(self.A) - 1:
            return ec
        for _ in range(self.gamma - 1 if lvl >= self.w_from else 0):
            ec = ec + self._vc(lvl, rc - st_mv(self.A[k], self.geo.grids[k], ec))
        return ec

    def _vc(self, lvl, b):
        k = lvl - 1
        A = self.A[k]
        if k == len(self.A) - 1:
            return sla.cho_solve(self.cho, b.reshape(-1), check_finite=False).reshape(-1, 6)
        g = self.geo.grids[k]
        Lg = self.geo.levels[k]
        w = self.omega / self.rho[k]
        Mi = self.Minv[k]
        x = bj(Mi, b, w)
        for _ in range(self.nu_c - 1):
            x = x + bj(Mi, b - st_mv(A, g, x), w)
        r = b - st_mv(A, g, x)
        ncg = int(np.prod(Lg["gc"]))
        ec = self._coarse(lvl + 1, restrict(Lg["Q"], Lg["agg_of"], ncg, r))
        prolong_add(Lg["Q"], Lg["agg_of"], ec, x)
        for _ in range(self.nu_c):
            x = x + bj(Mi, b - st_mv(A, g, x), w)
        return x

    def vcycle(self, b):
        """Finest level: b (N, 3), zero on fixed particles -> z (N, 3) (amg3d.py:609-637, multiplicative)."""
        geo = self.geo
        w = self.omega / self.rho0
        nagg = int(np.prod(geo.g0))
        x = bj(self.M0, b, w)
        for _ in range(self.nu - 1):
            x = x + bj(self.M0, b - self.apply0(x), w)
        r = b - self.apply0(x)
        ec = self._coarse(1, restrict(geo.P, geo.agg_of0, nagg, r))
        prolong_add(geo.P, geo.agg_of0, ec, x)
        for _ in range(self.nu):
            x = x + bj(self.M0, b - self.apply0(x), w)
        return x

    def pcg(self, b, tol, maxit=2000):
        """K_ff x = b from x0 = 0, stop at ||r|| <= tol ||b|| (amg3d.py:639-668).  Returns x, iterations, relres."""
        x = np.zeros_like(b)
        r = b.copy()
        bn = math.sqrt(float((b * b).sum()))
        if bn == 0.0:
            return x, 0, 0.0
        z = self.vcycle(r)
        p = z.copy()
        rz = float((r * z).sum())
        it, rn = 0, bn
        for it in range(1, maxit + 1):
            Ap = self.apply0(p)
            alpha = rz / float((p * Ap).sum())
            x += alpha * p
            r -= alpha * Ap
            rn = math.sqrt(float((r * r).sum()))
            if rn <= tol * bn:
                break
            z = self.vcycle(r)
            rz2 = float((r * z).sum())
            p = z + (rz2 / rz) * p
            rz = rz2
        return x, it, rn / bn
