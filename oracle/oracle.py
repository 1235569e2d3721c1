"""ctypes binding of the FP64 CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the cpu_baseline leg of bench.py, always as the checker or the timed CPU
baseline, never as part of the product path.

Two libraries expose the same routines:

* ``port`` -- ``oracle/liboracle.so``: the C restatement (trtt_oracle.c),
  built by ``make -C oracle`` (no reference sources needed);
* ``ref``  -- ``oracle/_ref/liboracle_ref.so``: the reference plugin C
  compiled from its own sources by ``make -C oracle ref`` (only where the
  reference tree is present; the built .so then travels with the repo).

Both are called with the reference signatures (``plugin/ywrap.c:231-403``,
``tomography-LongFessler-model/ywrap.c:6-77``): raw double* arrays,
accumulate-into-out semantics, 0/-1 return codes.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "liboracle_ref.so")
# reference checkout (read-only): $TRTT_REFERENCE_ROOT, else the mounted tree
REFROOT = os.environ.get("TRTT_REFERENCE_ROOT", "/root/reference")

_dp = C.POINTER(C.c_double)
_lp = C.POINTER(C.c_long)
_L, _D, _I = C.c_long, C.c_double, C.c_int

# argtypes in reference order (plugin/trtt_2D_projectors.h:72-82,
# plugin/trtt_3D_projectors.h:299-423, plugin/trtt_3D_projectors_cubic.h:299-363)
_SIGS = {
    "mvmult": [_dp, _dp, _L, _dp, _lp, _lp],
    "PB2D": [_dp, _dp, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp, _I],
    "FB2D": [_dp, _dp, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp, _I],
    "PB2D_cubic": [_dp, _dp, _L, _L, _D, _I, _L, _D, _dp, _dp, _I],
    "FB2D_cubic": [_dp, _dp, _L, _L, _D, _I, _L, _D, _dp, _dp, _I],
    "PB2D_sparser": [_dp, _L, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp],
    "FB2D_sparser": [_dp, _L, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _D, _dp, _dp],
    "PB3D": [_dp, _dp, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _L, _D, _D, _dp, _dp, _I],
    "CB3D": [_dp, _dp, _L, _L, _L, _D, _I, _dp, _dp, _L, _D, _dp, _L, _L, _D, _D, _dp, _dp, _I],
    "DD_PB3D": [_dp, _dp, _L, _L, _L, _D, _L, _L, _D, _D, _dp, _dp, _I],
    # port only: the reference carries trtt_DD_CB3D commented out
    "DD_CB3D": [_dp, _dp, _L, _L, _L, _D, _L, _L, _D, _D, _dp, _dp, _I],
    "PB3D_cubic": [_dp, _dp, _L, _L, _L, _D, _I, _L, _L, _D, _D, _dp, _dp, _I],
    "CB3D_cubic": [_dp, _dp, _L, _L, _L, _D, _I, _L, _L, _D, _D, _dp, _dp, _I],
}
_PORT_ONLY = {"DD_CB3D"}
_LF = ["direct", "line_integ_direct", "adjoint", "line_integ_adjoint"]
_LFS = ["sparser", "line_integ_sparser"]


class LF2DParams(C.Structure):
    """lf2d_parameters (tomography-LongFessler-model/LongFessler2D.h:16-28)."""

    _fields_ = [("pixelSize", C.c_double), ("pixelStep", C.c_double),
                ("voxelSize", C.c_double), ("sourceDistance", C.c_double),
                ("detectorDistance", C.c_double),
                ("objectOffset1", C.c_double), ("objectOffset2", C.c_double),
                ("objectDimension1", C.c_long), ("objectDimension2", C.c_long),
                ("detectorDimension", C.c_long)]


def build(ref: bool = False) -> None:
    """Build the oracle (and, if asked and the reference tree exists, the
    compiled reference) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(REFROOT):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REFROOT={REFROOT}"], check=True)


def _dptr(a):
    return a.ctypes.data_as(_dp)


def _lptr(a):
    return a.ctypes.data_as(_lp)


class Oracle:
    """FP64 reference routines bound from one of the two oracle libraries."""

    def __init__(self, kind: str = "port"):
        path = PORT_SO if kind == "port" else REF_SO
        if not os.path.exists(path):
            build(ref=(kind == "ref"))
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.kind = kind
        self.lib = C.CDLL(path)
        pre = "orc_" if kind == "port" else "trtt_"
        self._f = {}
        for name, sig in _SIGS.items():
            if kind != "port" and name in _PORT_ONLY:
                continue
            fn = getattr(self.lib, pre + name)
            fn.argtypes = sig
            fn.restype = C.c_int
            self._f[name] = fn
        lpre = "orc_lf2d_" if kind == "port" else "lf2d_"
        for name in _LF:
            fn = getattr(self.lib, lpre + name)
            fn.argtypes = [C.POINTER(LF2DParams), _D, _D, _dp, _dp, _I]
            fn.restype = None
            self._f["lf2d_" + name] = fn
        for name in _LFS:
            fn = getattr(self.lib, lpre + name)
            fn.argtypes = [C.POINTER(LF2DParams), _D, _D, _L, _L, _dp, _I]
            fn.restype = None
            self._f["lf2d_" + name] = fn
        if kind == "port":
            fn = self.lib.orc_footprint_table
            fn.argtypes = [_I, _L, _dp, _dp, _dp]
            fn.restype = C.c_double
            self._f["footprint_table"] = fn

    # -- raw access ---------------------------------------------------------
    def raw(self, name):
        return self._f[name]

    # -- numpy conveniences (out is accumulated in place, as the plugin does)
    def cb3d(self, out, vol, scan, view, job, table=None):
        return self._p3d("CB3D", out, vol, scan, view, job, table)

    def pb3d(self, out, vol, scan, view, job, table=None):
        return self._p3d("PB3D", out, vol, scan, view, job, table)

    def _p3d(self, base, out, vol, scan, view, job, table):
        xos = np.ascontiguousarray(scan.xos[view], dtype=np.float64)
        xsd = np.ascontiguousarray(scan.xsd[view], dtype=np.float64)
        _chk(out)
        _chk(vol)
        if table is None:
            return self._f[base + "_cubic"](
                _dptr(out), _dptr(vol), scan.nx, scan.ny, scan.nz, scan.s_scl,
                scan.s_deg, scan.nu, scan.nv, scan.u_scl, scan.v_scl,
                _dptr(xos), _dptr(xsd), job)
        return self._f[base](
            _dptr(out), _dptr(vol), scan.nx, scan.ny, scan.nz, scan.s_scl,
            scan.s_deg, _dptr(table.footprint), _dptr(table.cum), table.size,
            table.step, _dptr(table.coord), scan.nu, scan.nv, scan.u_scl,
            scan.v_scl, _dptr(xos), _dptr(xsd), job)

    def dd_pb3d(self, out, vol, scan, view, job):
        xos = np.ascontiguousarray(scan.xos[view], dtype=np.float64)
        xsd = np.ascontiguousarray(scan.xsd[view], dtype=np.float64)
        _chk(out)
        _chk(vol)
        return self._f["DD_PB3D"](
            _dptr(out), _dptr(vol), scan.nx, scan.ny, scan.nz, scan.s_scl,
            scan.nu, scan.nv, scan.u_scl, scan.v_scl, _dptr(xos), _dptr(xsd),
            job)

    def dd_cb3d(self, out, vol, scan, view, job):
        """Cone-beam distance-driven pair (the reference's unfinished
        trtt_DD_CB3D, completed; port only)."""
        xos = np.ascontiguousarray(scan.xos[view], dtype=np.float64)
        xsd = np.ascontiguousarray(scan.xsd[view], dtype=np.float64)
        _chk(out)
        _chk(vol)
        return self._f["DD_CB3D"](
            _dptr(out), _dptr(vol), scan.nx, scan.ny, scan.nz, scan.s_scl,
            scan.nu, scan.nv, scan.u_scl, scan.v_scl, _dptr(xos), _dptr(xsd),
            job)

    def p2d(self, base, out, img, scan, view, job, table=None):
        xos = np.ascontiguousarray(scan.xos[view], dtype=np.float64)
        xsd = np.ascontiguousarray(scan.xsd[view], dtype=np.float64)
        _chk(out)
        _chk(img)
        if table is None:
            return self._f[base + "_cubic"](
                _dptr(out), _dptr(img), scan.nx, scan.ny, scan.s_scl,
                scan.s_deg, scan.nv, scan.v_scl, _dptr(xos), _dptr(xsd), job)
        return self._f[base](
            _dptr(out), _dptr(img), scan.nx, scan.ny, scan.s_scl, scan.s_deg,
            _dptr(table.footprint), _dptr(table.cum), table.size, table.step,
            _dptr(table.coord), scan.nv, scan.v_scl, _dptr(xos), _dptr(xsd),
            job)

    def sparser2d(self, base, out, i, j, scan, view, table):
        xos = np.ascontiguousarray(scan.xos[view], dtype=np.float64)
        xsd = np.ascontiguousarray(scan.xsd[view], dtype=np.float64)
        _chk(out)
        return self._f[base + "_sparser"](
            _dptr(out), i, j, scan.nx, scan.ny, scan.s_scl, scan.s_deg,
            _dptr(table.footprint), _dptr(table.cum), table.size, table.step,
            _dptr(table.coord), scan.nv, scan.v_scl, _dptr(xos), _dptr(xsd))

    def mvmult(self, out, vec, a, i, j):
        _chk(out)
        _chk(vec)
        return self._f["mvmult"](_dptr(out), _dptr(vec), len(a), _dptr(a),
                                 _lptr(i), _lptr(j))

    def lf2d(self, name, params, beta, offset, src, dst, clr):
        _chk(src)
        _chk(dst)
        self._f["lf2d_" + name](C.byref(params), beta, offset, _dptr(src),
                                _dptr(dst), clr)

    def lf2d_sparser(self, name, params, beta, offset, i1, i2, dst, clr):
        _chk(dst)
        self._f["lf2d_" + name](C.byref(params), beta, offset, i1, i2,
                                _dptr(dst), clr)

    def footprint_table(self, deg, m):
        fp, cum, coord = np.zeros(m), np.zeros(m), np.zeros(m)
        step = self._f["footprint_table"](deg, m, _dptr(fp), _dptr(cum), _dptr(coord))
        return fp, cum, coord, step


def _chk(a):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise TypeError("oracle arrays must be C-contiguous float64")


_CACHE: dict[str, Oracle] = {}


def get(kind: str = "port") -> Oracle:
    if kind not in _CACHE:
        _CACHE[kind] = Oracle(kind)
    return _CACHE[kind]


def ref_available() -> bool:
    return os.path.exists(REF_SO) or os.path.isdir(REFROOT)
