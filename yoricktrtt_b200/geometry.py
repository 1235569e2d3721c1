"""Host-side acquisition geometry: 3D affine "xforms", tomographic object and
data frames, and the per-view coefficient arrays the projectors consume.

This restates the Yorick glue of TRTT that builds the 12 ``xos`` and 12
``xsd`` coefficients handed to every projector call:

* ``Xform3D`` -- 3x4 row-major affine transform with move / rotate (unit
  quaternion) / scale / combine / invert, as ``plugin/trtt_xform3d.c:253-459``
  (storage ``plugin/trtt_xform3d.c:52-66``).  Every operation acts on the
  left: ``move`` adds a translation after the transform, ``rotate`` and
  ``scale`` pre-multiply it.
* object frame ``xi = S(s_scl) . T(-(n-1)/2)``  (``Ytrtt_tomobj.i:198-236``);
* detector frame ``xi = S(1, v_scl, u_scl) . T(0, -nv/2, -nu/2)``
  (``Ytrtt_tomdata.i:140-185``);
* circular orbits: per view ``xos = T(Rsc,0,0) . Rz(pi - theta)`` and
  ``xsd = T(-Rsd, -v_off, -u_off)`` (``Tomography_3D/Ytrtt3D_system.i:436-459``,
  2D ``Tomography_2D/Ytrtt2D_system.i:515-575``);
* the projector coefficients ``xos_coefs = (xos . (xotilt . obj_xi)).a`` and
  ``xsd_coefs = (data_xi^-1 . xsd).a`` (``Ytrtt_3D_projectors.i:104-110``,
  ``Ytrtt_2D_projectors.i:421-428``).

All arithmetic is FP64 on the host; a scan of 360 views costs microseconds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Geometry and projector-type constants (Ytrtt_common.i:60-77).
TRTT_SPLINE_DRIVEN = 1
TRTT_DISTANCE_DRIVEN = 2
TRTT_LONG_FESSLER = 3
TRTT_LONG_FESSLER_LINE_INTEG = 4
TRTT_PARALLEL_BEAM = 3
TRTT_CONE_BEAM = 4
TRTT_FAN_BEAM = 5


class Xform3D:
    """3x4 affine transform stored as 12 row-major coefficients
    (``plugin/trtt_xform3d.c:52-66``); the implicit 4th row is [0 0 0 1]."""

    __slots__ = ("a",)

    def __init__(self, a=None):
        if a is None:
            a = (1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0)
        self.a = np.array(a, dtype=np.float64).reshape(12).copy()

    def copy(self) -> "Xform3D":
        return Xform3D(self.a)

    # -- left-acting operations (plugin/trtt_xform3d.c:275-401) ------------
    def move(self, tx: float, ty: float, tz: float) -> "Xform3D":
        """Translate after the transform: a[3]+=tx, a[7]+=ty, a[11]+=tz."""
        b = self.a.copy()
        b[3] += tx
        b[7] += ty
        b[11] += tz
        return Xform3D(b)

    def rotate(self, qw: float, qx: float, qy: float, qz: float) -> "Xform3D":
        """Pre-multiply by the rotation of quaternion (qw,qx,qy,qz), normalised
        when its norm is not exactly one (plugin/trtt_xform3d.c:302-366)."""
        aww, axx, ayy, azz = qw * qw, qx * qx, qy * qy, qz * qz
        nrm2 = (aww + axx) + (ayy + azz)
        if nrm2 == 1.0:
            r00 = (aww + axx) - (ayy + azz)
            r11 = (aww + ayy) - (axx + azz)
            r22 = (aww + azz) - (axx + ayy)
            scl = 2.0
        elif nrm2 > 0.0:
            scl = 1.0 / nrm2
            r00 = scl * ((aww + axx) - (ayy + azz))
            r11 = scl * ((aww + ayy) - (axx + azz))
            r22 = scl * ((aww + azz) - (axx + ayy))
            scl += scl
        else:
            raise ValueError("quaternion cannot be normalised")
        awx, awy, awz = scl * qw * qx, scl * qw * qy, scl * qw * qz
        axy, axz, ayz = scl * qx * qy, scl * qx * qz, scl * qy * qz
        r = np.array([[r00, axy - awz, axz + awy],
                      [axy + awz, r11, ayz - awx],
                      [axz - awy, ayz + awx, r22]])
        return Xform3D(_rot_dot(r, self.a))

    def scale(self, sx: float, sy: float, sz: float) -> "Xform3D":
        """Pre-multiply by diag(sx, sy, sz) (scales whole rows)."""
        b = self.a.copy()
        b[0:4] *= sx
        b[4:8] *= sy
        b[8:12] *= sz
        return Xform3D(b)

    def combine(self, right: "Xform3D") -> "Xform3D":
        """Matrix product self . right (plugin/trtt_xform3d.c:253-273)."""
        return Xform3D(_xform_dot(self.a, right.a))

    def invert(self) -> "Xform3D":
        """Inverse affine transform.  The reference inverts the 4x4 matrix by
        LU (plugin/trtt_xform3d.c:438-459); a diagonal linear part is
        inverted in closed form so that its zero coefficients stay exactly
        zero, which the circular-orbit kernels rely on."""
        m = self.a.reshape(3, 4)
        lin, t = m[:, :3], m[:, 3]
        if np.count_nonzero(lin - np.diag(np.diag(lin))) == 0:
            d = np.diag(lin)
            if np.any(d == 0.0):
                raise ValueError("singular transform")
            inv = np.zeros((3, 4))
            for r in range(3):
                inv[r, r] = 1.0 / d[r]
                inv[r, 3] = -t[r] / d[r]
            return Xform3D(inv.reshape(12))
        full = np.eye(4)
        full[:3, :] = m
        inv = np.linalg.inv(full)
        return Xform3D(inv[:3, :].reshape(12))

    def __repr__(self) -> str:  # pragma: no cover - debugging aid
        return f"Xform3D({self.a.tolist()})"


def _xform_dot(a, b):
    c = np.empty(12)
    for r in range(3):
        ar = a[4 * r: 4 * r + 4]
        for col in range(4):
            c[4 * r + col] = ar[0] * b[col] + ar[1] * b[4 + col] + ar[2] * b[8 + col]
        c[4 * r + 3] += ar[3]
    return c


def _rot_dot(r, a):
    c = np.empty(12)
    for row in range(3):
        for col in range(4):
            c[4 * row + col] = (r[row, 0] * a[col] + r[row, 1] * a[4 + col]
                                + r[row, 2] * a[8 + col])
    return c


def object_xi(nx: int, ny: int, nz: int, s_scl: float) -> Xform3D:
    """Voxel -> metric frame centred on the object (Ytrtt_tomobj.i:198-236)."""
    return Xform3D().move(-0.5 * (nx - 1), -0.5 * (ny - 1), -0.5 * (nz - 1)) \
        .scale(s_scl, s_scl, s_scl)


def data_xi(nu: int, nv: int, u_scl: float, v_scl: float) -> Xform3D:
    """Detector pixel -> metric frame centred on the detector
    (Ytrtt_tomdata.i:140-185): x is the source axis, y the transaxial v axis,
    z the axial u axis."""
    return Xform3D().move(0.0, -0.5 * nv, -0.5 * nu).scale(1.0, v_scl, u_scl)


def view_xforms(theta: float, rsc: float | None, rsd: float | None,
                u_off: float = 0.0, v_off: float = 0.0,
                x_off: float = 0.0, y_off: float = 0.0, z_off: float = 0.0):
    """Per-view xos, xsd, xotilt of a circular orbit
    (Tomography_3D/Ytrtt3D_system.i:436-480).  ``rsc``/``rsd`` may be None
    for parallel beam (no translation along the source axis)."""
    th = 0.5 * (math.pi - theta)
    xos = Xform3D().rotate(math.cos(th), 0.0, 0.0, math.sin(th))
    if rsc is not None:
        xos = xos.move(rsc, 0.0, 0.0)
    xsd = Xform3D()
    if rsd is not None:
        xsd = xsd.move(-1.0 * rsd, 0.0, 0.0)
    if v_off:
        xsd = xsd.move(0.0, -1.0 * v_off, 0.0)
    if u_off:
        xsd = xsd.move(0.0, 0.0, -1.0 * u_off)
    xotilt = Xform3D()
    if x_off or y_off or z_off:
        xotilt = xotilt.move(x_off, y_off, z_off)
    return xos, xsd, xotilt


def projector_coefs(obj_xi: Xform3D, dat_xi: Xform3D, xos: Xform3D,
                    xsd: Xform3D, xotilt: Xform3D):
    """(xos . (xotilt . obj_xi)).a and (data_xi^-1 . xsd).a
    (Ytrtt_3D_projectors.i:104-110)."""
    xos_plus = xos.combine(xotilt.combine(obj_xi))
    xsd_plus = dat_xi.invert().combine(xsd)
    return xos_plus.a.copy(), xsd_plus.a.copy()


@dataclass
class Scan3D:
    """A tomographic object plus a list of views: the inputs of every 3D
    projector call.  ``xos``/``xsd`` are (nviews, 12) FP64 arrays."""

    nx: int
    ny: int
    nz: int
    s_scl: float
    s_deg: int
    nu: int
    nv: int
    u_scl: float
    v_scl: float
    mode: int
    xos: np.ndarray
    xsd: np.ndarray
    theta: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @property
    def nviews(self) -> int:
        return int(self.xos.shape[0])


def circular_scan_3d(nx, ny, nz, s_scl, s_deg, nu, nv, u_scl, v_scl, nviews,
                     mode=TRTT_CONE_BEAM, rsc=1000.0, rsd=1500.0,
                     theta=None, arc=2.0 * math.pi, u_off=0.0, v_off=0.0,
                     x_off=0.0, y_off=0.0, z_off=0.0) -> Scan3D:
    """Circular orbit of ``nviews`` views uniformly spaced over ``arc``
    (Tomography_3D/Ytrtt3D_system.i:368-511).  ``rsc`` is the source-to-
    isocentre distance (SID), ``rsd`` the source-to-detector distance (SDD);
    parallel beam ignores both."""
    if theta is None:
        theta = np.arange(nviews, dtype=np.float64) * (arc / nviews)
    theta = np.asarray(theta, dtype=np.float64)
    oxi = object_xi(nx, ny, nz, s_scl)
    dxi = data_xi(nu, nv, u_scl, v_scl)
    xos = np.empty((len(theta), 12))
    xsd = np.empty((len(theta), 12))
    par = mode == TRTT_PARALLEL_BEAM
    for k, th in enumerate(theta):
        a, b, c = view_xforms(th, None if par else rsc, None if par else rsd,
                              u_off, v_off, x_off, y_off, z_off)
        xos[k], xsd[k] = projector_coefs(oxi, dxi, a, b, c)
    return Scan3D(nx, ny, nz, s_scl, s_deg, nu, nv, u_scl, v_scl, mode,
                  xos, xsd, theta)


@dataclass
class Scan2D:
    """2D object (nx x ny) and a list of views onto an nv-cell detector."""

    nx: int
    ny: int
    s_scl: float
    s_deg: int
    nv: int
    v_scl: float
    mode: int
    xos: np.ndarray
    xsd: np.ndarray
    theta: np.ndarray = field(default_factory=lambda: np.zeros(0))
    rsc: float = 0.0
    rsd: float = 0.0

    @property
    def nviews(self) -> int:
        return int(self.xos.shape[0])


def circular_scan_2d(nx, ny, s_scl, s_deg, nv, v_scl, nviews,
                     mode=TRTT_FAN_BEAM, rsc=1000.0, rsd=1500.0, theta=None,
                     arc=None) -> Scan2D:
    """2D parallel (``arc`` defaults to pi) or fan beam (2 pi) scan
    (Tomography_2D/Ytrtt2D_system.i:454-575).  The 2D object is a single
    z-slice (nz=1) and the detector a single row (nu=1)."""
    par = mode == TRTT_PARALLEL_BEAM
    if arc is None:
        arc = math.pi if par else 2.0 * math.pi
    if theta is None:
        theta = np.arange(nviews, dtype=np.float64) * (arc / nviews)
    theta = np.asarray(theta, dtype=np.float64)
    oxi = object_xi(nx, ny, 1, s_scl)
    dxi = data_xi(1, nv, 1.0, v_scl)
    xos = np.empty((len(theta), 12))
    xsd = np.empty((len(theta), 12))
    for k, th in enumerate(theta):
        a, b, c = view_xforms(th, None if par else rsc, None if par else rsd)
        xos[k], xsd[k] = projector_coefs(oxi, dxi, a, b, c)
    return Scan2D(nx, ny, s_scl, s_deg, nv, v_scl, mode, xos, xsd, theta,
                  rsc, rsd)


def dd_coefs_2d(scan: "Scan2D"):
    """Per-view (xos . xotilt).a and xsd.a of a 2D circular scan: the
    coefficients of the distance-driven projector, which works in object and
    detector millimetres (Ytrtt_2D_projectors.i:868-880) where the
    spline-driven ones also carry the pixel and detector-cell transforms."""
    par = scan.mode == TRTT_PARALLEL_BEAM
    xos = np.empty((scan.nviews, 12))
    xsd = np.empty((scan.nviews, 12))
    for k, th in enumerate(scan.theta):
        a, b, c = view_xforms(th, None if par else scan.rsc, None if par else scan.rsd)
        xos[k] = a.combine(c).a
        xsd[k] = b.a
    return xos, xsd


def gate_weights(t_index: float, nt: int):
    """Linear temporal interpolation of one view between two gates
    (Ytrtt_3D_projectors.i:301-311): j = [floor(t), ceil(t)] mod nt and
    w = [1-pe, pe] with pe = t - floor(t)."""
    f = math.floor(t_index)
    c = math.ceil(t_index)
    pe = t_index - f
    return (int(f) % nt, int(c) % nt), (1.0 - pe, pe)


def gate_t_index(dates, tcycl: float, nt: int) -> np.ndarray:
    """Fractional gate index of each acquisition date
    (Tomography_4D/Ytrtt4D_system.i:439-452): (t mod tcycl) * nt / tcycl."""
    t = np.asarray(dates, dtype=np.float64)
    return np.mod(t, tcycl) * (nt / tcycl)


# ---------------------------------------------------------------------------
# Orbit symmetry of a scan's views
# ---------------------------------------------------------------------------
def quarter_turn_coefs(xos, m: int, nx: int, ny: int) -> np.ndarray:
    """xos coefficients of the view that sees voxel (i, j, k) where the view
    with coefficients ``xos`` sees voxel (R^m(i, j), k), R the quarter turn
    R(i, j) = (n-1-j, i) of a square nx = ny = n grid (m = 2, the half turn
    (nx-1-i, ny-1-j), needs no square grid).  Each row (a, b, c, d) of the
    3x4 matrix acts as a i + b j + c k + d."""
    x = np.asarray(xos, dtype=np.float64).reshape(3, 4)
    out = x.copy()
    a, b = x[:, 0], x[:, 1]
    if m == 1:
        out[:, 0], out[:, 1], out[:, 3] = b, -a, x[:, 3] + a * (nx - 1)
    elif m == 2:
        out[:, 0], out[:, 1], out[:, 3] = -a, -b, x[:, 3] + a * (nx - 1) + b * (ny - 1)
    elif m == 3:
        out[:, 0], out[:, 1], out[:, 3] = -b, a, x[:, 3] + b * (ny - 1)
    return out.reshape(12)


def _coefs_match(p, q, tol):
    p = np.asarray(p).reshape(3, 4)
    q = np.asarray(q).reshape(3, 4)
    scale = np.maximum(np.abs(p).max(axis=1), np.abs(q).max(axis=1))
    return bool(np.all(np.abs(p - q) <= tol * np.maximum(scale, 1e-300)[:, None]))


def view_groups(scan: "Scan3D", tol: float = 1e-10):
    """Groups of views related by turns of the volume grid about the z axis:
    [a, b1, b2, b3] when view b_m sees voxel (i, j, k) exactly where view a
    sees voxel (R^m(i, j), k) for m = 1, 2, 3 (square grid of even side),
    [a, b2] for the half turn alone (nx or ny even), [a] otherwise; xsd must
    be equal within the group.  Greedy in view order.  Projecting a group
    needs the footprints of view a only: view b_m's footprint of voxel
    column c is view a's footprint of column R^m(c)."""
    nx, ny, nv = scan.nx, scan.ny, scan.nviews
    used = np.zeros(nv, dtype=bool)
    groups = []
    quad_ok = nx == ny and nx % 2 == 0
    pair_ok = nx % 2 == 0 or ny % 2 == 0

    def find(coefs, xsd):
        for b in range(nv):
            if not used[b] and _coefs_match(scan.xos[b], coefs, tol) and \
                    _coefs_match(scan.xsd[b], xsd, tol):
                return b
        return -1

    for a in range(nv):
        if used[a]:
            continue
        used[a] = True
        mem = [a]
        if quad_ok:
            b = [find(quarter_turn_coefs(scan.xos[a], m, nx, ny), scan.xsd[a]) for m in (1, 2, 3)]
            if min(b) >= 0 and len(set(b)) == 3:
                mem += b
        if len(mem) == 1 and pair_ok:
            b2 = find(quarter_turn_coefs(scan.xos[a], 2, nx, ny), scan.xsd[a])
            if b2 >= 0:
                mem.append(b2)
        for b in mem[1:]:
            used[b] = True
        groups.append(mem)
    return groups


def turn_columns(i, j, m: int, nx: int, ny: int):
    """(i, j) -> R^m(i, j), R(i, j) = (n-1-j, i); the half turn
    R^2(i, j) = (nx-1-i, ny-1-j) also on a rectangular grid."""
    m %= 4
    if m == 2:
        return nx - 1 - i, ny - 1 - j
    for _ in range(m):
        i, j = nx - 1 - j, i
    return i, j
