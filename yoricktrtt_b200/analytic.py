"""Analytic projections of ellipse (2D) and ellipsoid (3D) phantoms for the
scans of ``geometry.py``: the model-level reference of the projectors.

The reference generates simulated data by the analytic Radon transform of
ellipse phantoms, with the line integral of each ray through each ellipse in
closed form and the detector cell's thickness accounted for by integrating
the profile over the cell with Romberg's method
(``Tomography_2D/Ytrtt2D_simulated_data_generation.i:261-769``, called with
the projection angle theta - pi/2 by
``Tomography_2D/Ytrtt2D_script_reconstructions.i:46-48``).  Here the same
quantity, the integral over the detector cell of the line integrals, is
computed for any ray by intersecting the ray with each ellipse / ellipsoid (a
quadratic in the ray parameter) and summing over Gauss-Legendre nodes of the
cell.  It is what the projectors return for a phantom sampled on their grid:
a detector row sums to the phantom's mass (value x area, or x volume times
the magnification squared in cone beam).

Ray conventions (those of the projectors, ``geometry.view_xforms``): for view
angle theta the source sits at Rsc (cos theta, sin theta) in the object's
(x, y) plane, rays of a parallel beam travel along (cos theta, sin theta),
the detector's v axis runs along (sin theta, -cos theta) and its u axis
(3D) along +z; cell centres are at (i - (n-1)/2) times the cell size.
Object coordinates are millimetres from the volume centre.

An ellipse is (cx, cy, a, b, angle, value): centre, semi-axes along the
ellipse's own axes, rotation of its first axis from x (radians), and the
value inside (``Ytrtt2D_simulated_data_generation.i:261-290``: x0, y0, a, b,
alpha, mu).  An ellipsoid is an ``Ellipsoid``: centre, semi-axes, a rotation
whose rows are the ellipsoid's axes in object coordinates, and the value;
``ellipsoid`` builds one from the z-x-z Euler angles of
``Tomography_3D/Ytrtt3D_simulated_data_generation.i:46-155`` and
``read_phantom`` reads the phantom files of the cone-beam simulator
(``Tomography_3D/Simul_Data/simul.c:296-360``).
"""
from __future__ import annotations

import math
from typing import NamedTuple

import numpy as np

from .geometry import TRTT_CONE_BEAM, TRTT_FAN_BEAM, TRTT_PARALLEL_BEAM


class Ellipsoid(NamedTuple):
    center: tuple
    axes: tuple
    rot: np.ndarray  # (3, 3); row r = unit vector of semi-axis r
    value: float


def euler_zxz(phi, theta, psi):
    """Rotation of Euler angles (phi about z, theta about x, psi about z),
    radians: the matrix whose rows give an object point's coordinates along
    the ellipsoid's axes (``Ytrtt3D_simulated_data_generation.i:135-137``)."""
    cf, sf = math.cos(phi), math.sin(phi)
    ct, st = math.cos(theta), math.sin(theta)
    cp, sp = math.cos(psi), math.sin(psi)
    return np.array([[cp * cf - ct * sf * sp, cp * sf + ct * cf * sp, sp * st],
                     [-sp * cf - ct * sf * cp, -sp * sf + ct * cf * cp, cp * st],
                     [st * sf, -st * cf, ct]])


def ellipsoid(center, axes, value, phi=0.0, theta=0.0, psi=0.0):
    return Ellipsoid(tuple(float(c) for c in center), tuple(float(a) for a in axes),
                     euler_zxz(phi, theta, psi), float(value))


def read_phantom(path, half_extent, value_scale=0.1928):
    """Ellipsoids of a cone-beam simulator phantom file (``phantom`` then
    ``object <n> ellipsoid center X Y Z half-axis A B C angles THETA PHI
    VALUE`` ... ``end``; ``Tomography_3D/Simul_Data/simul.c:296-360``).
    Centres and half-axes are given in units of the volume's half extent,
    ``half_extent`` = 0.5 (n - 1) x voxel size per axis; the angles are in
    degrees (phi about z, then theta tilting the first axis towards z); the
    values are multiplied by ``value_scale`` (the simulator's water
    attenuation, 0.1928 per cm).  Cylinders and Gaussians, which no shipped
    phantom uses, are rejected."""
    hx, hy, hz = half_extent
    tok = open(path).read().split()
    if "phantom" not in tok:
        raise ValueError(f"{path}: no 'phantom' keyword")
    i = tok.index("phantom") + 1
    out = []
    while i < len(tok) and tok[i] != "end":
        if tok[i] != "object":
            i += 1
            continue
        kind = tok[i + 2]
        if kind != "ellipsoid":
            raise NotImplementedError(f"{path}: {kind} objects are not supported")
        if tok[i + 3] != "center" or tok[i + 7] != "half-axis" or tok[i + 11] != "angles":
            raise ValueError(f"{path}: malformed ellipsoid at token {i}")
        c = [float(t) for t in tok[i + 4:i + 7]]
        a = [float(t) for t in tok[i + 8:i + 11]]
        th, ph = (math.radians(float(t)) for t in tok[i + 12:i + 14])
        val = float(tok[i + 14]) * value_scale
        ct, st, cp, sp = math.cos(th), math.sin(th), math.cos(ph), math.sin(ph)
        rot = np.array([[ct * cp, ct * sp, -st], [-sp, cp, 0.0], [st * cp, st * sp, ct]])
        out.append(Ellipsoid((c[0] * hx, c[1] * hy, c[2] * hz), (a[0] * hx, a[1] * hy, a[2] * hz), rot, val))
        i += 15
    return out


def _gauss(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return 0.5 * x, 0.5 * w  # nodes in [-1/2, 1/2], weights summing to 1


def chord_2d(p, u, ellipses):
    """Sum over ellipses of value x length of the line p + t u (u unit)
    inside the ellipse.  p, u: (..., 2) arrays."""
    p = np.asarray(p, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    out = np.zeros(p.shape[:-1])
    for cx, cy, a, b, ang, val in ellipses:
        ca, sa = math.cos(ang), math.sin(ang)
        qx, qy = p[..., 0] - cx, p[..., 1] - cy
        q0 = (qx * ca + qy * sa) / a
        q1 = (-qx * sa + qy * ca) / b
        w0 = (u[..., 0] * ca + u[..., 1] * sa) / a
        w1 = (-u[..., 0] * sa + u[..., 1] * ca) / b
        A = w0 * w0 + w1 * w1
        B = 2.0 * (q0 * w0 + q1 * w1)
        Cq = q0 * q0 + q1 * q1 - 1.0
        disc = B * B - 4.0 * A * Cq
        out += val * np.sqrt(np.maximum(disc, 0.0)) / A
    return out


def chord_3d(p, u, ellipsoids):
    """Same for ``Ellipsoid``s.  p, u: (..., 3) arrays."""
    p = np.asarray(p, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    out = np.zeros(p.shape[:-1])
    for e in ellipsoids:
        m = e.rot / np.asarray(e.axes)[:, None]  # object -> unit-sphere frame
        q = (p - np.asarray(e.center)) @ m.T
        w = u @ m.T
        A = (w * w).sum(-1)
        B = 2.0 * (q * w).sum(-1)
        Cq = (q * q).sum(-1) - 1.0
        disc = B * B - 4.0 * A * Cq
        out += e.value * np.sqrt(np.maximum(disc, 0.0)) / A
    return out


def _rays(theta, v, u, mode, rsc, rsd):
    """Ray origins and unit directions for detector coordinates (v, u) (mm)
    of view theta; u is None in 2D."""
    ct, st = math.cos(theta), math.sin(theta)
    ev = np.array([st, -ct])
    if mode == TRTT_PARALLEL_BEAM:
        p2 = v[..., None] * ev
        d2 = np.broadcast_to(np.array([ct, st]), p2.shape)
    else:
        s2 = rsc * np.array([ct, st])
        det = s2 - rsd * np.array([ct, st]) + v[..., None] * ev
        p2 = np.broadcast_to(s2, det.shape)
        d2 = det - s2
    if u is None:
        d2 = d2 / np.linalg.norm(d2, axis=-1, keepdims=True)
        return p2, d2
    z0 = u if mode == TRTT_PARALLEL_BEAM else np.zeros_like(u)
    p = np.concatenate([p2, z0[..., None]], axis=-1)
    dz = np.zeros_like(u) if mode == TRTT_PARALLEL_BEAM else u
    d = np.concatenate([d2, dz[..., None]], axis=-1)
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)
    return p, d


def sinogram_2d(ellipses, scan, quad=8):
    """(nviews, nv): cell integrals of the line integrals of ``ellipses`` for
    a ``geometry.Scan2D`` (parallel or fan beam)."""
    mode = scan.mode
    if mode not in (TRTT_PARALLEL_BEAM, TRTT_FAN_BEAM):
        raise ValueError("2D scans are parallel or fan beam")
    xg, wg = _gauss(quad)
    vc = (np.arange(scan.nv) - 0.5 * (scan.nv - 1)) * scan.v_scl
    vq = vc[:, None] + xg[None, :] * scan.v_scl  # (nv, quad)
    out = np.zeros((len(scan.theta), scan.nv))
    for k, th in enumerate(scan.theta):
        p, d = _rays(th, vq, None, mode, scan.rsc, scan.rsd)
        out[k] = (chord_2d(p, d, ellipses) * wg[None, :]).sum(axis=1)
    return out * scan.v_scl


def projections_3d(ellipsoids, scan, quad=4, rsc=1000.0, rsd=1500.0):
    """(nviews, nv, nu): cell integrals of the line integrals of
    ``ellipsoids`` for a ``geometry.Scan3D`` of a circular orbit (parallel or
    cone beam, source-to-centre rsc and source-to-detector rsd in mm as
    passed to ``circular_scan_3d``)."""
    mode = scan.mode
    if mode not in (TRTT_PARALLEL_BEAM, TRTT_CONE_BEAM):
        raise ValueError("3D scans are parallel or cone beam")
    xg, wg = _gauss(quad)
    vc = (np.arange(scan.nv) - 0.5 * (scan.nv - 1)) * scan.v_scl
    uc = (np.arange(scan.nu) - 0.5 * (scan.nu - 1)) * scan.u_scl
    V = vc[:, None, None, None] + xg[None, None, :, None] * scan.v_scl
    U = uc[None, :, None, None] + xg[None, None, None, :] * scan.u_scl
    V, U = np.broadcast_arrays(V, U)  # (nv, nu, quad, quad)
    w2 = wg[:, None] * wg[None, :]
    out = np.zeros((len(scan.theta), scan.nv, scan.nu))
    for k, th in enumerate(scan.theta):
        p, d = _rays(th, V, U, mode, rsc, rsd)
        out[k] = (chord_3d(p, d, ellipsoids) * w2).sum(axis=(2, 3))
    return out * (scan.u_scl * scan.v_scl)


def ellipse_image(ellipses, nx, ny, s_scl, oversample=4):
    """Pixel averages of the ellipse phantom on an nx x ny grid of pitch
    s_scl (pixel (i, j) centred at ((i - (nx-1)/2) s, (j - (ny-1)/2) s)),
    each pixel sampled oversample^2 times; array [j][i]."""
    o = oversample
    f = (np.arange(o) + 0.5) / o - 0.5
    xs = ((np.arange(nx) - 0.5 * (nx - 1))[:, None] + f[None, :]).reshape(-1) * s_scl
    ys = ((np.arange(ny) - 0.5 * (ny - 1))[:, None] + f[None, :]).reshape(-1) * s_scl
    Y, X = np.meshgrid(ys, xs, indexing="ij")
    img = np.zeros_like(X)
    for cx, cy, a, b, ang, val in ellipses:
        ca, sa = math.cos(ang), math.sin(ang)
        xr = ((X - cx) * ca + (Y - cy) * sa) / a
        yr = (-(X - cx) * sa + (Y - cy) * ca) / b
        img += val * (xr * xr + yr * yr <= 1.0)
    return img.reshape(ny, o, nx, o).mean(axis=(1, 3))


def ellipsoid_volume(ellipsoids, nx, ny, nz, s_scl, oversample=2):
    """Voxel averages of the ellipsoid phantom, array [k][j][i]; with
    oversample=1 the voxel-centre samples of the simulator's ``make_image``
    (``Tomography_3D/Simul_Data/make_image.c:41-56``, inside when <= 1)."""
    o = oversample
    f = (np.arange(o) + 0.5) / o - 0.5

    def axis(n):
        return ((np.arange(n) - 0.5 * (n - 1))[:, None] + f[None, :]).reshape(-1) * s_scl

    Z, Y, X = np.meshgrid(axis(nz), axis(ny), axis(nx), indexing="ij")
    P = np.stack([X, Y, Z], axis=-1)
    vol = np.zeros_like(X)
    for e in ellipsoids:
        q = (P - np.asarray(e.center)) @ (e.rot / np.asarray(e.axes)[:, None]).T
        vol += e.value * ((q * q).sum(-1) <= 1.0)
    return vol.reshape(nz, o, ny, o, nx, o).mean(axis=(1, 3, 5))
