"""Synthetic phantoms used as test and benchmark inputs.

Ellipsoids are encoded as 16 floats: centre (3), semi-axes (3), rotation R
(3x3, row-major, local -> world) and density, the format of the oracle's
orc_project_ellipsoids / orc_draw_ellipsoids and of rtkb_project_ellipsoids.
"""
from __future__ import annotations

import numpy as np

# RTK's Shepp-Logan ellipsoids (src/rtkSheppLoganPhantom.cxx:25-34): semi-axes,
# centre, rotation angle about y (degrees), density.
_SHEPP_LOGAN = [
    (0.69, 0.90, 0.92, 0.0, 0.0, 0.0, 0.0, 2.0),
    (0.6624, 0.880, 0.874, 0.0, 0.0, 0.0, 0.0, -0.98),
    (0.41, 0.21, 0.16, -0.22, -0.25, 0.0, 108.0, -0.02),
    (0.31, 0.22, 0.11, 0.22, -0.25, 0.0, 72.0, -0.02),
    (0.21, 0.50, 0.25, 0.0, -0.25, 0.35, 0.0, 0.02),
    (0.046, 0.046, 0.046, 0.0, -0.25, 0.10, 0.0, 0.02),
    (0.046, 0.02, 0.023, -0.08, -0.25, -0.65, 0.0, 0.01),
    (0.046, 0.02, 0.023, 0.06, -0.25, -0.65, 90.0, 0.01),
    (0.056, 0.1, 0.04, 0.06, 0.625, -0.105, 90.0, 0.02),
    (0.056, 0.1, 0.056, 0.0, 0.625, 0.1, 0.0, -0.02),
]


def rot_y(deg: float) -> np.ndarray:
    """Local -> world rotation of QuadricShape::SetEllipsoid's y rotation
    (src/rtkQuadricShape.cxx:259-318)."""
    a = np.deg2rad(deg)
    c, s = np.cos(a), np.sin(a)
    return np.array([[c, 0.0, -s], [0.0, 1.0, 0.0], [s, 0.0, c]])


def ellipsoid(center, axes, R, density) -> np.ndarray:
    e = np.zeros(16)
    e[0:3] = center
    e[3:6] = axes
    e[6:15] = np.asarray(R, dtype=np.float64).reshape(9)
    e[15] = density
    return e


def shepp_logan(scale: float) -> np.ndarray:
    return np.stack([
        ellipsoid(np.array([cx, cy, cz]) * scale, np.array([ax, ay, az]) * scale, rot_y(ang), den)
        for ax, ay, az, cx, cy, cz, ang, den in _SHEPP_LOGAN
    ])


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def random_ellipsoids(n: int, seed: int, axis_range=(5.0, 80.0), centre_radius=100.0,
                      density_range=(0.1, 1.0)) -> np.ndarray:
    """n seeded random ellipsoids: semi-axes uniform in axis_range (mm), centres
    uniform in a sphere of radius centre_radius (mm), uniform random rotations,
    densities uniform in density_range."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        while True:
            c = rng.uniform(-centre_radius, centre_radius, size=3)
            if np.linalg.norm(c) <= centre_radius:
                break
        ax = rng.uniform(*axis_range, size=3)
        out.append(ellipsoid(c, ax, random_rotation(rng), rng.uniform(*density_range)))
    return np.stack(out)


def poisson_noise(line_integrals: np.ndarray, i0: float, mu_ref: float, seed: int) -> np.ndarray:
    """Pre-log Poisson noise (rtk::AddNoise semantics, include/rtkGgoFunctions.h:295-340):
    counts ~ Poisson(I0 exp(-mu_ref * p)), p' = -log(max(counts, 1) / I0) / mu_ref."""
    rng = np.random.default_rng(seed)
    lam = i0 * np.exp(-mu_ref * line_integrals)
    counts = np.maximum(rng.poisson(lam), 1)
    return (-np.log(counts / i0) / mu_ref).astype(line_integrals.dtype)


def fov_mask(g, vol, proj) -> np.ndarray:
    """Voxels whose projection lands on the detector for every projection (the
    region rtk::FieldOfViewImageFilter keeps), for an oracle Geometry."""
    from oracle import oracle as O

    nz, ny, nx = O.shape_of(vol)
    z, y, x = np.meshgrid(np.arange(nz) + vol.index[2], np.arange(ny) + vol.index[1], np.arange(nx) + vol.index[0],
                          indexing="ij")
    X = np.stack([x.ravel(), y.ravel(), z.ravel(), np.ones(x.size)]).astype(np.float64)
    ok = np.ones(X.shape[1], dtype=bool)
    for i in range(proj.size[2]):
        m, _ = O.bp_matrix(g, vol, proj, proj.index[2] + i, False)
        w = m[2] @ X
        u = (m[0] @ X) / w - proj.index[0]
        v = (m[1] @ X) / w - proj.index[1]
        ok &= (w != 0) & (u >= 0) & (u <= proj.size[0] - 1) & (v >= 0) & (v <= proj.size[1] - 1)
    return ok.reshape(nz, ny, nx)


def check_image_quality(recon: np.ndarray, ref: np.ndarray, err_tol: float, psnr_tol: float, ref_value: float):
    """CheckImageQuality of test/rtkTest.h:38-105: mean absolute error per pixel
    and PSNR against ref_value.  Returns (error_per_pixel, psnr, passed)."""
    d = recon.astype(np.float64) - ref.astype(np.float64)
    err = np.abs(d).mean()
    mse = (d * d).mean()
    psnr = float("inf") if mse == 0.0 else 20 * np.log10(ref_value) - 10 * np.log10(mse)
    return err, psnr, bool(err < err_tol and psnr > psnr_tol)


def acceptance_ties(g, vol, proj, tol=1e-6) -> np.ndarray:
    """Voxels that some projection maps within tol pixels of RTK's acceptance
    bounds of its optimised paths (u or v at 0 or N - 1, the ends of
    0 <= floor(u) < N - 1).  On exactly symmetric geometries (pixel and voxel
    centres aligned, angles in exact steps) such ties are frequent, and
    whether the sample counts depends on the last bit of the map's rounding,
    which differs between any two correct implementations."""
    from oracle import oracle as O

    nz, ny, nx = O.shape_of(vol)
    z, y, x = np.meshgrid(np.arange(nz) + vol.index[2], np.arange(ny) + vol.index[1], np.arange(nx) + vol.index[0],
                          indexing="ij")
    X = np.stack([x.ravel(), y.ravel(), z.ravel(), np.ones(x.size)]).astype(np.float64)
    tie = np.zeros(X.shape[1], dtype=bool)
    for i in range(proj.size[2]):
        m, _ = O.bp_matrix(g, vol, proj, proj.index[2] + i, False)
        w = m[2] @ X
        u = (m[0] @ X) / w - proj.index[0]
        v = (m[1] @ X) / w - proj.index[1]
        for c, n in ((u, proj.size[0]), (v, proj.size[1])):
            tie |= (np.abs(c) < tol) | (np.abs(c - (n - 1)) < tol)
    return tie.reshape(nz, ny, nx)
