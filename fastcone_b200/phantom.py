"""Seeded random-ellipsoid phantoms (parameters on the host, voxelisation on the GPU).

Parameter rows (16 doubles) as the C ABI's fcb_phantom_device expects: centre (3, voxels
from the volume centre volDim/2), semi-axes (3, voxels), row-major rotation R (9; body
coordinates = R^T (p - c)), density.
"""
from __future__ import annotations

import numpy as np


def random_rotation(rng) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def random_ellipsoids(n: int, vol_xyz, seed: int, axes=(0.05, 0.4), density=(0.1, 1.0),
                      centre_radius=1.0) -> np.ndarray:
    """n ellipsoids: centres uniform in the ball of radius ``centre_radius`` (1 = the unit
    ball) scaled to the volume half-widths,
    semi-axes U(axes) x half-width (the smallest), random rotation, densities U(density)."""
    rng = np.random.default_rng(seed)
    half = np.asarray(vol_xyz, np.float64) / 2.0
    hw = float(half.min())
    out = np.zeros((n, 16), np.float64)
    for k in range(n):
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        r = centre_radius * rng.random() ** (1.0 / 3.0)
        out[k, 0:3] = d * r * half
        out[k, 3:6] = rng.uniform(axes[0], axes[1], 3) * hw
        out[k, 6:15] = random_rotation(rng).ravel()
        out[k, 15] = rng.uniform(density[0], density[1])
    return out
