"""numpy-level calls of the drop-in C ABI (the reference plugin signatures).

Each function takes the same arguments as the Yorick builtin it replaces
(``plugin/ywrap.c:231-403``, ``tomography-LongFessler-model/ywrap.c:6-77``),
with numpy float64 arrays in the reference layouts, accumulates into ``out``
as the reference does, and raises ``TrttError`` when the library returns
TRTT_FAILURE (-1).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import dptr, lptr


class LF2DParams(C.Structure):
    """lf2d_parameters (tomography-LongFessler-model/LongFessler2D.h:16-28)."""

    _fields_ = [("pixelSize", C.c_double), ("pixelStep", C.c_double),
                ("voxelSize", C.c_double), ("sourceDistance", C.c_double),
                ("detectorDistance", C.c_double),
                ("objectOffset1", C.c_double), ("objectOffset2", C.c_double),
                ("objectDimension1", C.c_long), ("objectDimension2", C.c_long),
                ("detectorDimension", C.c_long)]


def _c12(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(12)
    return a


def p3d(name: str, out, vol, nx, ny, nz, s_scl, s_deg, nu, nv, u_scl, v_scl,
        xos, xsd, job, table=None) -> None:
    """trtt_PB3D / trtt_CB3D (table given) or their _cubic twins."""
    lib = _lib.load()
    xos, xsd = _c12(xos), _c12(xsd)
    if table is None:
        fn = getattr(lib, f"trtt_{name}_cubic")
        rc = fn(dptr(out), dptr(vol), nx, ny, nz, s_scl, s_deg, nu, nv, u_scl, v_scl,
                dptr(xos), dptr(xsd), job)
    else:
        fn = getattr(lib, f"trtt_{name}")
        rc = fn(dptr(out), dptr(vol), nx, ny, nz, s_scl, s_deg, dptr(table.footprint),
                dptr(table.cum), table.size, table.step, dptr(table.coord), nu, nv,
                u_scl, v_scl, dptr(xos), dptr(xsd), job)
    _lib.check(rc, f"trtt_{name}")


def scan3d_call(name, out, vol, scan, view, job, table=None):
    """Convenience: one view of a Scan3D through the drop-in symbol."""
    p3d(name, out, vol, scan.nx, scan.ny, scan.nz, scan.s_scl, scan.s_deg,
        scan.nu, scan.nv, scan.u_scl, scan.v_scl, scan.xos[view], scan.xsd[view],
        job, table)


def dd2d(out, x, scan, job, view0: int = 0, nview: int | None = None, coefs=None):
    """Distance-driven 2D projector (``D_single_2D`` / ``D_whole_2D``,
    Ytrtt_2D_projectors.i:820-1245) for views [view0, view0 + nview) of a
    ``geometry.Scan2D``: job 0 adds H x (x image [ny][nx]) into out
    [nview][nv]; job 1 adds H^T x (x [nview][nv]) into out [ny][nx].
    ``coefs``: (xos, xsd) from ``geometry.dd_coefs_2d`` (computed if None)."""
    from .geometry import dd_coefs_2d
    nview = scan.nviews - view0 if nview is None else nview
    xos, xsd = dd_coefs_2d(scan) if coefs is None else coefs
    xos = np.ascontiguousarray(xos[view0:view0 + nview], dtype=np.float64)
    xsd = np.ascontiguousarray(xsd[view0:view0 + nview], dtype=np.float64)
    shape_in = (scan.ny, scan.nx) if job == 0 else (nview, scan.nv)
    shape_out = (nview, scan.nv) if job == 0 else (scan.ny, scan.nx)
    for a, shp, name in ((x, shape_in, "x"), (out, shape_out, "out")):
        if a.dtype != np.float64 or not a.flags.c_contiguous or a.size != int(np.prod(shp)):
            raise ValueError(f"{name} must be C-contiguous float64 of shape {shp}")
    rc = _lib.load().trtt_b200_dd2d(dptr(out), dptr(x), scan.nx, scan.ny, scan.s_scl, scan.nv,
                                    scan.v_scl, nview, dptr(xos), dptr(xsd), scan.mode, job)
    _lib.check(rc, "trtt_b200_dd2d")


class DistanceDriven2D:
    """The whole-scan distance-driven operator ``C(x, job)`` of a 2D scan
    (``D_whole_2D``): job 0 returns the sinogram [nviews][nv] of an image,
    job 1 the image of a sinogram; ``single_view(k)`` is ``D_single_2D``."""

    def __init__(self, scan):
        from .geometry import dd_coefs_2d
        self.scan = scan
        self.coefs = dd_coefs_2d(scan)

    def __call__(self, x, job: int = 0, view0: int = 0, nview: int | None = None):
        s = self.scan
        nview = s.nviews - view0 if nview is None else nview
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros((nview, s.nv) if job == 0 else (s.ny, s.nx))
        dd2d(out, x, s, job, view0, nview, self.coefs)
        return out

    def single_view(self, k: int):
        def op(x, job=0):
            r = self(np.asarray(x).reshape(-1, self.scan.nv) if job == 1 else x, job, k, 1)
            return r[0] if job == 0 else r
        return op


def dd_pb3d(out, vol, scan, view, job):
    lib = _lib.load()
    rc = lib.trtt_DD_PB3D(dptr(out), dptr(vol), scan.nx, scan.ny, scan.nz, scan.s_scl,
                          scan.nu, scan.nv, scan.u_scl, scan.v_scl,
                          dptr(_c12(scan.xos[view])), dptr(_c12(scan.xsd[view])), job)
    _lib.check(rc, "trtt_DD_PB3D")


def dd_cb3d(out, vol, scan, view, job):
    """trtt_DD_CB3D on one view (host FP64 arrays, accumulate into out)."""
    lib = _lib.load()
    rc = lib.trtt_DD_CB3D(dptr(out), dptr(vol), scan.nx, scan.ny, scan.nz, scan.s_scl,
                          scan.nu, scan.nv, scan.u_scl, scan.v_scl, dptr(_c12(scan.xos[view])),
                          dptr(_c12(scan.xsd[view])), job)
    _lib.check(rc, "trtt_DD_CB3D")


def dd_cb3d_batch(out, x, scan, job):
    """trtt_b200_dd_cb3d over all views of `scan`."""
    lib = _lib.load()
    rc = lib.trtt_b200_dd_cb3d(dptr(out), dptr(x), scan.nx, scan.ny, scan.nz, scan.s_scl,
                               scan.nu, scan.nv, scan.u_scl, scan.v_scl, scan.nviews,
                               dptr(np.ascontiguousarray(scan.xos)),
                               dptr(np.ascontiguousarray(scan.xsd)), job)
    _lib.check(rc, "trtt_b200_dd_cb3d")

def p2d(name: str, out, img, scan, view, job, table=None):
    """trtt_PB2D / trtt_FB2D (table) or _cubic, one view of a Scan2D."""
    lib = _lib.load()
    xos, xsd = _c12(scan.xos[view]), _c12(scan.xsd[view])
    if table is None:
        rc = getattr(lib, f"trtt_{name}_cubic")(
            dptr(out), dptr(img), scan.nx, scan.ny, scan.s_scl, scan.s_deg, scan.nv,
            scan.v_scl, dptr(xos), dptr(xsd), job)
    else:
        rc = getattr(lib, f"trtt_{name}")(
            dptr(out), dptr(img), scan.nx, scan.ny, scan.s_scl, scan.s_deg,
            dptr(table.footprint), dptr(table.cum), table.size, table.step,
            dptr(table.coord), scan.nv, scan.v_scl, dptr(xos), dptr(xsd), job)
    _lib.check(rc, f"trtt_{name}")


def sparser2d(name: str, out, i, j, scan, view, table):
    lib = _lib.load()
    rc = getattr(lib, f"trtt_{name}_sparser")(
        dptr(out), i, j, scan.nx, scan.ny, scan.s_scl, scan.s_deg,
        dptr(table.footprint), dptr(table.cum), table.size, table.step,
        dptr(table.coord), scan.nv, scan.v_scl, dptr(_c12(scan.xos[view])),
        dptr(_c12(scan.xsd[view])))
    _lib.check(rc, f"trtt_{name}_sparser")


def mvmult(out, vec, a, i, j):
    """out[i[k]-1] += a[k] * vec[j[k]-1] (1-based COO, plugin/trtt_common.c:62-69)."""
    lib = _lib.load()
    a = np.ascontiguousarray(a, dtype=np.float64)
    i = np.ascontiguousarray(i, dtype=np.int64)
    j = np.ascontiguousarray(j, dtype=np.int64)
    rc = lib.trtt_mvmult(dptr(out), dptr(vec), len(a), dptr(a), lptr(i), lptr(j))
    _lib.check(rc, "trtt_mvmult")


def lf2d(name: str, params: LF2DParams, beta, offset, src, dst, clr):
    """lf2d_direct / lf2d_adjoint / lf2d_line_integ_{direct,adjoint}."""
    lib = _lib.load()
    getattr(lib, f"lf2d_{name}")(C.addressof(params), beta, offset, dptr(src), dptr(dst), clr)
    err = _lib.last_error()
    if err:
        raise _lib.TrttError(f"lf2d_{name} failed: {err}")


def lf2d_sparser(name: str, params: LF2DParams, beta, offset, i1, i2, dst, clr):
    lib = _lib.load()
    getattr(lib, f"lf2d_{name}")(C.addressof(params), beta, offset, i1, i2, dptr(dst), clr)
    err = _lib.last_error()
    if err:
        raise _lib.TrttError(f"lf2d_{name} failed: {err}")
