"""Seeded two-phase microstructures for the synthetic workloads (host side, NumPy).

Restates the reference generators with the same sequence of random draws, so a seed gives the same image:
  grf_two_phase   2D thresholded Gaussian random field           (coarse2d/micro.py:5-20)
  spheres         3D random sequential addition of spheres       (coarse3d/micro3d.py:84-132)
  ellipsoids      3D RSA of randomly oriented ellipsoids         (coarse3d/micro3d.py:76-81, 135-145)
  grf3            3D thresholded Gaussian random field           (coarse3d/micro3d.py:148-157)
Voxel / pixel order is the lattice order (x fastest).
"""
import numpy as np


def _gauss_smooth_2d(noise, corr):
    ny, nx = noise.shape
    k2 = np.fft.fftfreq(ny)[:, None] ** 2 + np.fft.fftfreq(nx)[None, :] ** 2
    return np.real(np.fft.ifft2(np.fft.fft2(noise) * np.exp(-2.0 * (np.pi * corr) ** 2 * k2)))


def grf_two_phase(nx, ny, corr, phi, seed, pad=None):
    """Phase-1 indicator (ny*nx,) int64 of a Gaussian field with correlation length ~corr, area fraction ~phi;
    generated on a padded grid and cropped (not periodic)."""
    rng = np.random.default_rng(seed)
    p = int(4 * corr) + 4 if pad is None else pad
    field = _gauss_smooth_2d(rng.standard_normal((ny + 2 * p, nx + 2 * p)), corr)[p:p + ny, p:p + nx]
    return (field > np.quantile(field, 1.0 - phi)).astype(np.int64).ravel()


def _voxel_centres(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([i, j, k], -1) + 0.5


def random_rotation(rng):
    """Uniform random rotation from the QR factorisation of a Gaussian matrix (sign-fixed, det +1)."""
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))[None, :]
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def rsa(nx, ny, nz, phi, rng, sample_shape, max_tries=20000):
    """Random sequential addition until volume fraction phi (or max_tries).

    sample_shape(rng) -> (semi-axes (3,), rotation (3,3)).  During the first 70 % of the attempts a candidate must not
    touch (6-neighbourhood) an existing inclusion; later overlaps are accepted.  Returns (phase (nz,ny,nx) bool,
    number of inclusions).
    """
    img = np.zeros((nz, ny, nx), bool)
    centres = _voxel_centres(nx, ny, nz)
    target = phi * img.size
    occupied, placed, tries = 0, 0, 0
    upper = np.array([nx, ny, nz])
    while occupied < target and tries < max_tries:
        tries += 1
        axes, rot = sample_shape(rng)
        reach = axes.max()
        c = rng.uniform([-reach * 0.5] * 3, upper + reach * 0.5)
        lo = np.maximum(np.floor(c - reach - 1).astype(int), 0)
        hi = np.minimum(np.ceil(c + reach + 1).astype(int), upper)
        if np.any(hi <= lo):
            continue
        local = (centres[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] - c) @ rot
        inside = ((local / axes) ** 2).sum(-1) <= 1.0
        if not inside.any():
            continue
        box = img[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]]
        if tries < 0.7 * max_tries:
            grown = inside.copy()
            grown[1:] |= inside[:-1]
            grown[:-1] |= inside[1:]
            grown[:, 1:] |= inside[:, :-1]
            grown[:, :-1] |= inside[:, 1:]
            grown[:, :, 1:] |= inside[:, :, :-1]
            grown[:, :, :-1] |= inside[:, :, 1:]
            if (grown & box).any():
                continue
        fresh = inside & ~box
        if not fresh.any():
            continue
        box |= inside
        occupied += int(fresh.sum())
        placed += 1
    return img, placed


def spheres(nx, ny, nz, phi, rmean, rng, rjit=0.4):
    def shape(r_):
        r = rmean * (1 + rjit * (2 * r_.random() - 1))
        return np.array([r, r, r]), np.eye(3)

    img, n = rsa(nx, ny, nz, phi, rng, shape)
    return img.astype(np.int64).ravel(), dict(kind="spheres", rmean=rmean, ninc=n)


def ellipsoids(nx, ny, nz, phi, rmean, rng, aspect=(1.0, 2.0), rjit=0.4):
    """Randomly oriented ellipsoids with the volume of a sphere of radius r: semi-axes
    r (al^(2/3) be^(1/3), al^(-1/3) be^(1/3), al^(-1/3) be^(-2/3)), al ~ U(aspect), be ~ U(1, sqrt(al))."""
    def shape(r_):
        r = rmean * (1 + rjit * (2 * r_.random() - 1))
        al = r_.uniform(*aspect)
        be = r_.uniform(1.0, np.sqrt(al))
        axes = r * np.array([al ** (2 / 3) * be ** (1 / 3), al ** (-1 / 3) * be ** (1 / 3),
                             al ** (-1 / 3) * be ** (-2 / 3)])
        return axes, random_rotation(r_)

    img, n = rsa(nx, ny, nz, phi, rng, shape)
    return img.astype(np.int64).ravel(), dict(kind="ellipsoids", rmean=rmean, ninc=n, aspect=aspect)


def prolate_ellipsoids(nx, ny, nz, phi, r, rng, aspect=3.0, max_tries=20000):
    """Randomly oriented prolate ellipsoids a:b:b = aspect:1:1 with the volume of a sphere of radius r (large boxes
    need more than the default 20000 attempts to reach phi)."""
    axes = r * np.array([aspect ** (2 / 3), aspect ** (-1 / 3), aspect ** (-1 / 3)])

    def shape(r_):
        return axes, random_rotation(r_)

    img, n = rsa(nx, ny, nz, phi, rng, shape, max_tries=max_tries)
    return img.astype(np.int64).ravel(), dict(kind="prolate", r=r, ninc=n, aspect=aspect)


def grf3(nx, ny, nz, corr, phi, rng):
    p = int(4 * corr) + 4
    f = rng.standard_normal((nz + 2 * p, ny + 2 * p, nx + 2 * p))
    k2 = (np.fft.fftfreq(f.shape[0])[:, None, None] ** 2 + np.fft.fftfreq(f.shape[1])[None, :, None] ** 2 +
          np.fft.rfftfreq(f.shape[2])[None, None, :] ** 2)
    f = np.fft.irfftn(np.fft.rfftn(f) * np.exp(-2.0 * (np.pi * corr) ** 2 * k2), s=f.shape, axes=(0, 1, 2))
    f = f[p:p + nz, p:p + ny, p:p + nx]
    return (f > np.quantile(f, 1.0 - phi)).astype(np.int64).ravel(), dict(kind="grf", corr=corr)
