"""Seeded synthetic phantoms (random ellipses / ellipsoids).

The reference builds its test objects the same way: sums of homogeneous
ellipses (``Tomography_2D/Ytrtt2D_simulated_data_generation.i:109-260``) and
ellipsoids (``Tomography_3D/Ytrtt3D_simulated_data_generation.i:96-153``) on
the voxel grid.  Centres, half-axes, orientations and intensities are drawn
from ``numpy.random.default_rng(seed)``; no dataset is read.

Volumes are returned in the reference memory order: 2D ``[j, i]`` and 3D
``[k, j, i]`` (x fastest, ``plugin/trtt_common.h:239-248``).
"""
from __future__ import annotations

import math

import numpy as np


def ellipses_2d(nx: int, ny: int, n: int = 10, seed: int = 0,
                dtype=np.float64, body: bool = True) -> np.ndarray:
    """``n`` random ellipses, intensities U[0,1]; the first is a large
    centred "body" ellipse unless ``body=False``."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    x = (x - 0.5 * (nx - 1)) / (0.5 * nx)
    y = (y - 0.5 * (ny - 1)) / (0.5 * ny)
    img = np.zeros((ny, nx))
    for e in range(n):
        r = 0.6 * math.sqrt(rng.uniform())
        phi = rng.uniform(0, 2 * math.pi)
        cx, cy = r * math.cos(phi), r * math.sin(phi)
        a = rng.uniform(0.05, 0.35)
        b = rng.uniform(0.05, 0.35)
        if body and e == 0:
            cx = cy = 0.0
            a, b = rng.uniform(0.85, 0.95, size=2)
        ang = rng.uniform(0, math.pi)
        val = rng.uniform(0.0, 1.0)
        ca, sa = math.cos(ang), math.sin(ang)
        xr = (x - cx) * ca + (y - cy) * sa
        yr = -(x - cx) * sa + (y - cy) * ca
        img[(xr / a) ** 2 + (yr / b) ** 2 <= 1.0] += val
    return img.astype(dtype)


def ellipsoids_3d(nx: int, ny: int, nz: int, n: int = 20, seed: int = 0,
                  dtype=np.float32, z_shift: float = 0.0, body: bool = True) -> np.ndarray:
    """``n`` random ellipsoids, intensities U[0,1].  As in the reference's
    Shepp-Logan style generator, the first one is a large "body" ellipsoid
    (transaxial semi-axes 0.85-0.95 of the half extent, longer than the
    volume along z, centred) that the others sit in, so the volume is dense
    like a patient scan (about 60% non-zero voxels); ``body=False`` draws only
    small ellipsoids.  ``z_shift`` translates every ellipsoid along z (in
    units of the half height), as the 4D breathing phantom does between
    gates."""
    rng = np.random.default_rng(seed)
    vol = np.zeros((nz, ny, nx), dtype=np.float64)
    zz = (np.arange(nz) - 0.5 * (nz - 1)) / (0.5 * nz)
    yy = (np.arange(ny) - 0.5 * (ny - 1)) / (0.5 * ny)
    xx = (np.arange(nx) - 0.5 * (nx - 1)) / (0.5 * nx)
    for e in range(n):
        r = 0.55 * math.sqrt(rng.uniform())
        phi = rng.uniform(0, 2 * math.pi)
        cx, cy = r * math.cos(phi), r * math.sin(phi)
        cz = rng.uniform(-0.5, 0.5) + z_shift
        ax, ay, az = rng.uniform(0.06, 0.3, size=3)
        if body and e == 0:
            cx, cy, cz = 0.0, 0.0, z_shift
            ax, ay = rng.uniform(0.85, 0.95, size=2)
            az = rng.uniform(1.1, 1.3)
        ang = rng.uniform(0, math.pi)
        val = rng.uniform(0.0, 1.0)
        ca, sa = math.cos(ang), math.sin(ang)
        # bounding box in voxel indices keeps the cost proportional to size
        rad = max(ax, ay, az)
        i0 = max(0, int((cx - rad + 1) * 0.5 * nx) - 1)
        i1 = min(nx, int((cx + rad + 1) * 0.5 * nx) + 2)
        j0 = max(0, int((cy - rad + 1) * 0.5 * ny) - 1)
        j1 = min(ny, int((cy + rad + 1) * 0.5 * ny) + 2)
        k0 = max(0, int((cz - az + 1) * 0.5 * nz) - 1)
        k1 = min(nz, int((cz + az + 1) * 0.5 * nz) + 2)
        if i0 >= i1 or j0 >= j1 or k0 >= k1:
            continue
        z = zz[k0:k1, None, None] - cz
        y = yy[None, j0:j1, None] - cy
        x = xx[None, None, i0:i1] - cx
        xr = x * ca + y * sa
        yr = -x * sa + y * ca
        inside = (xr / ax) ** 2 + (yr / ay) ** 2 + (z / az) ** 2 <= 1.0
        vol[k0:k1, j0:j1, i0:i1] += val * inside
    return vol.astype(dtype)


def breathing_gates(nx: int, ny: int, nz: int, nt: int, s_scl: float,
                    amplitude_mm: float = 10.0, n: int = 20, seed: int = 0,
                    dtype=np.float32) -> np.ndarray:
    """``nt`` gates of an ellipsoid phantom translated sinusoidally along z
    by up to ``amplitude_mm`` across the respiratory cycle.  Shape
    (nt, nz, ny, nx)."""
    out = np.empty((nt, nz, ny, nx), dtype=dtype)
    half_height_mm = 0.5 * nz * s_scl
    for g in range(nt):
        shift = amplitude_mm * 0.5 * (1 - math.cos(2 * math.pi * g / nt))
        out[g] = ellipsoids_3d(nx, ny, nz, n=n, seed=seed, dtype=dtype,
                               z_shift=shift / half_height_mm)
    return out
