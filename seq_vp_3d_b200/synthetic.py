"""Seeded synthetic registration pairs (stand-ins for the OASIS-like pairs the reference runs on; no dataset here).

blob_pair   config 1 generator: fixed = sum of 24 isotropic Gaussian blobs (centres uniform in the interior,
            sigma ~ U[2, 5] vox, amplitude ~ U[0.2, 1]) normalised to [0, 1] plus N(0, 0.01) noise; moving = fixed
            resampled trilinearly through a ground-truth Q1 displacement of 6 Gaussian vector bumps (sigma = 4 vox,
            peak |u| <= 1.5 vox), zero on the boundary, redrawn until its minimum nodal JD >= 0.5.
head_pair   config 2 generator: head-like phantom (ellipsoidal mask, semi-axes 0.42/0.45/0.45 of the extents, 3 nested
            tissue classes 0.2/0.5/0.8 with low-frequency-perturbed boundaries, multiplicative degree-2 bias 1 +- 0.1,
            Gaussian blur sigma = 1 vox, noise sigma = 0.02); ground truth from 40 Gaussian bumps (sigma 6-12 vox,
            peak <= 4 vox, min JD >= 0.4).
Arrays are float64, shape (nz, ny, nx); displacements (nz, ny, nx, 3) in physical units (xyz components).
"""
import numpy as np
from scipy.ndimage import gaussian_filter, map_coordinates


def _nodal_jd(u, spacing):
    """Finite-difference nodal JD of I + grad u (central differences), for the ground-truth acceptance test."""
    g = [np.gradient(u[..., r], spacing[2], spacing[1], spacing[0], edge_order=1) for r in range(3)]
    # g[r] = (d/dz, d/dy, d/dx) of component r
    F = np.empty(u.shape[:3] + (3, 3))
    for r in range(3):
        F[..., r, 0], F[..., r, 1], F[..., r, 2] = g[r][2], g[r][1], g[r][0]
        F[..., r, r] += 1.
    return np.linalg.det(F)


def _bumps(shape, spacing, rng, count, sigma_range, peak):
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij", sparse=True)
    u = np.zeros(shape + (3,))
    for _ in range(count):
        c = rng.uniform([0.2 * nz, 0.2 * ny, 0.2 * nx], [0.8 * nz, 0.8 * ny, 0.8 * nx])
        s = rng.uniform(*sigma_range) if np.ndim(sigma_range) else sigma_range
        v = rng.normal(size=3)
        v *= rng.uniform(0.3, 1.0) * peak / np.linalg.norm(v)
        g = np.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * s * s))
        for r in range(3):
            u[..., r] += v[r] * g * spacing[r]
    u[[0, -1]] = 0.; u[:, [0, -1]] = 0.; u[:, :, [0, -1]] = 0.
    return u


def _ground_truth(shape, spacing, rng, count, sigma_range, peak, min_jd):
    for _ in range(50):
        u = _bumps(shape, spacing, rng, count, sigma_range, peak)
        # peak |u| per node in voxels
        mag = np.sqrt(sum((u[..., r] / spacing[r]) ** 2 for r in range(3)))
        if mag.max() > peak:
            u *= peak / mag.max()
        if _nodal_jd(u, spacing).min() >= min_jd:
            return u
    raise RuntimeError("ground-truth displacement: no draw met the JD floor")


def _resample(image, u, spacing, order=1):
    """image at X + u (trilinear for order 1), boundary values clamped."""
    nz, ny, nx = image.shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    coords = [zz + u[..., 2] / spacing[2], yy + u[..., 1] / spacing[1], xx + u[..., 0] / spacing[0]]
    return map_coordinates(image, coords, order=order, mode="nearest")


def blob_pair(shape=(32, 32, 32), spacing=(1., 1., 1.), seed=0):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij", sparse=True)
    fixed = np.zeros(shape)
    for _ in range(24):
        c = rng.uniform([2, 2, 2], [nz - 3, ny - 3, nx - 3])
        s = rng.uniform(2, 5)
        a = rng.uniform(.2, 1.)
        fixed = fixed + a * np.exp(-((zz - c[0]) ** 2 + (yy - c[1]) ** 2 + (xx - c[2]) ** 2) / (2 * s * s))
    fixed = (fixed - fixed.min()) / (fixed.max() - fixed.min())
    fixed = fixed + rng.normal(size=shape) * 0.01
    u_gt = _ground_truth(shape, spacing, rng, 6, 4.0, 1.5, 0.5)
    moving = _resample(fixed, u_gt, spacing, order=1)
    return np.ascontiguousarray(fixed), np.ascontiguousarray(moving), u_gt


def head_pair(shape=(224, 192, 160), spacing=(1., 1., 1.), seed=0):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    z = (np.arange(nz) - (nz - 1) / 2) / nz
    y = (np.arange(ny) - (ny - 1) / 2) / ny
    x = (np.arange(nx) - (nx - 1) / 2) / nx
    zz, yy, xx = np.meshgrid(z, y, x, indexing="ij", sparse=True)
    # low-frequency boundary perturbation
    pert = np.zeros(shape)
    for _ in range(6):
        k = rng.integers(1, 4, size=3)
        ph = rng.uniform(0, 2 * np.pi, size=3)
        pert = pert + 0.03 * rng.uniform(.5, 1.) * (np.sin(2 * np.pi * k[0] * zz + ph[0])
                                                   * np.sin(2 * np.pi * k[1] * yy + ph[1])
                                                   * np.sin(2 * np.pi * k[2] * xx + ph[2]))
    radius = np.sqrt((zz / .42) ** 2 + (yy / .45) ** 2 + (xx / .45) ** 2) + pert
    image = np.zeros(shape)
    for level, value in ((1.0, 0.2), (0.8, 0.5), (0.55, 0.8)):
        image = np.where(radius <= level * 0.5, value, image)
    c = rng.normal(size=10) * 0.1 / 3
    bias = (1 + c[0] * zz + c[1] * yy + c[2] * xx + c[3] * zz * zz + c[4] * yy * yy + c[5] * xx * xx
            + c[6] * zz * yy + c[7] * zz * xx + c[8] * yy * xx)
    image = gaussian_filter(image * np.clip(bias, 0.9, 1.1), 1.0)
    fixed = image + rng.normal(size=shape) * 0.02
    u_gt = _ground_truth(shape, spacing, rng, 40, (6., 12.), 4.0, 0.4)
    moving = _resample(image, u_gt, spacing, order=1) + rng.normal(size=shape) * 0.02
    return np.ascontiguousarray(fixed), np.ascontiguousarray(moving), u_gt


def default_weights(shape, spacing, mu=0.03, nu=0.03, kappa=0.002):
    """The reference's default native weights: lambda = 0.1 / L*^2 (L* = geometric mean of the FOV lengths)."""
    nz, ny, nx = shape
    fov = [nx * spacing[0], ny * spacing[1], nz * spacing[2]]
    lstar = float(np.prod(fov)) ** (1 / 3)
    return dict(lam=0.1 / lstar ** 2, mu=mu, nu=nu, kappa=kappa)
