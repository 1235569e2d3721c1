"""Pin the FP64 oracle restatement against the reference plugin compiled
from its own sources (oracle/_ref): every routine, bit-for-bit, on seeded
inputs and geometries that exercise clipping, offsets, anisotropic
sampling, non-circular xforms and the failure path."""
import ctypes as C
import math

import numpy as np
import pytest

from yoricktrtt_b200 import footprint as F, geometry as G, phantoms as P


def _tilt(sc, mode):
    oxi = G.object_xi(sc.nx, sc.ny, sc.nz, sc.s_scl)
    dxi = G.data_xi(sc.nu, sc.nv, sc.u_scl, sc.v_scl)
    for k, th in enumerate(sc.theta):
        par = mode == G.TRTT_PARALLEL_BEAM
        xos, xsd, xot = G.view_xforms(th, None if par else 60.0, None if par else 90.0)
        xos = xos.rotate(math.cos(0.1), math.sin(0.1), 0.0, 0.0)
        sc.xos[k], sc.xsd[k] = G.projector_coefs(oxi, dxi, xos, xsd, xot)
    return sc


SCANS3D = [
    dict(mode=G.TRTT_CONE_BEAM),
    dict(mode=G.TRTT_PARALLEL_BEAM),
    dict(mode=G.TRTT_CONE_BEAM, nu=20, nv=16),
    dict(mode=G.TRTT_CONE_BEAM, us=0.7, vs=1.3, s=0.8, u_off=2.5),
    dict(mode=G.TRTT_CONE_BEAM, tilt=True),
    dict(mode=G.TRTT_PARALLEL_BEAM, tilt=True),
]


def _scan3d(mode, nx=18, ny=16, nz=12, nu=30, nv=28, s=1.0, us=1.0, vs=1.0, tilt=False, **kw):
    sc = G.circular_scan_3d(nx, ny, nz, s, 3, nu, nv, us, vs, 3, mode=mode, rsc=60.0, rsd=90.0, **kw)
    return _tilt(sc, mode) if tilt else sc


@pytest.mark.parametrize("cfg", SCANS3D)
@pytest.mark.parametrize("table", [False, True])
def test_pin_3d(oracle_port, oracle_ref, cfg, table):
    sc = _scan3d(**cfg)
    tab = F.make_footprint(3, 5001) if table else None
    name = "CB3D" if cfg["mode"] == G.TRTT_CONE_BEAM else "PB3D"
    vol = np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=5, seed=1, dtype=np.float64))
    rng = np.random.default_rng(0)
    for v in range(sc.nviews):
        for job in (0, 1):
            x = vol if job == 0 else rng.random((sc.nv, sc.nu))
            shape = (sc.nv, sc.nu) if job == 0 else vol.shape
            pre = rng.random(shape)
            a, b = pre.copy(), pre.copy()
            assert oracle_port._p3d(name, a, x, sc, v, job, tab) == 0
            assert oracle_ref._p3d(name, b, x, sc, v, job, tab) == 0
            assert np.array_equal(a, b)


@pytest.mark.parametrize("vs", [1.0, 0.4])
def test_pin_dd(oracle_port, oracle_ref, vs):
    sc = G.circular_scan_3d(14, 12, 10, 1.0, 3, 30, 32, vs, vs, 3, mode=G.TRTT_PARALLEL_BEAM)
    vol = np.ascontiguousarray(P.ellipsoids_3d(14, 12, 10, n=5, seed=2, dtype=np.float64))
    rng = np.random.default_rng(1)
    for v in range(sc.nviews):
        for job in (0, 1):
            x = vol if job == 0 else rng.random((sc.nv, sc.nu))
            shape = (sc.nv, sc.nu) if job == 0 else vol.shape
            a, b = np.zeros(shape), np.zeros(shape)
            oracle_port.dd_pb3d(a, x, sc, v, job)
            oracle_ref.dd_pb3d(b, x, sc, v, job)
            assert np.array_equal(a, b)


@pytest.mark.parametrize("mode", [G.TRTT_FAN_BEAM, G.TRTT_PARALLEL_BEAM])
@pytest.mark.parametrize("table", [False, True])
@pytest.mark.parametrize("nv", [60, 24])
def test_pin_2d(oracle_port, oracle_ref, mode, table, nv):
    sc = G.circular_scan_2d(40, 36, 1.0, 3, nv, 1.0, 5, mode=mode, rsc=120.0, rsd=180.0)
    tab = F.make_footprint(3, 5001) if table else None
    name = "FB2D" if mode == G.TRTT_FAN_BEAM else "PB2D"
    img = np.ascontiguousarray(P.ellipses_2d(40, 36, n=5, seed=3))
    rng = np.random.default_rng(2)
    for v in range(sc.nviews):
        for job in (0, 1):
            x = img if job == 0 else rng.random(nv)
            shape = (nv,) if job == 0 else img.shape
            a, b = np.zeros(shape), np.zeros(shape)
            assert oracle_port.p2d(name, a, x, sc, v, job, tab) == 0
            assert oracle_ref.p2d(name, b, x, sc, v, job, tab) == 0
            assert np.array_equal(a, b)
        for (i, j) in [(0, 0), (7, 30), (39, 35), (-2, 40)]:
            a, b = np.zeros(nv), np.zeros(nv)
            tab3 = tab or F.make_footprint(3, 5001)
            oracle_port.sparser2d(name, a, i, j, sc, v, tab3)
            oracle_ref.sparser2d(name, b, i, j, sc, v, tab3)
            assert np.array_equal(a, b)


def test_pin_lf(oracle_port, oracle_ref):
    from oracle.oracle import LF2DParams
    p = LF2DParams(pixelSize=1.0, pixelStep=1.2, voxelSize=2.0, sourceDistance=300.0,
                   detectorDistance=150.0, objectOffset1=1.5, objectOffset2=-0.5,
                   objectDimension1=30, objectDimension2=26, detectorDimension=100)
    rng = np.random.default_rng(4)
    img = np.ascontiguousarray(P.ellipses_2d(30, 26, n=4, seed=5).T.copy())
    img = np.ascontiguousarray(P.ellipses_2d(26, 30, n=4, seed=5))
    for beta in (-1.2, 0.0, 2.4):
        for name in ("direct", "line_integ_direct", "adjoint", "line_integ_adjoint"):
            src = img if "direct" in name else rng.random(100)
            for clr in (0, 1):
                dst0 = rng.random(100) if "direct" in name else rng.random((26, 30))
                a, b = dst0.copy(), dst0.copy()
                oracle_port.lf2d(name, p, beta, 0.75, src, a, clr)
                oracle_ref.lf2d(name, p, beta, 0.75, src, b, clr)
                assert np.array_equal(a, b), name
        for name in ("sparser", "line_integ_sparser"):
            for (i1, i2) in [(0, 0), (11, 20), (29, 25)]:
                a, b = np.ones(100), np.ones(100)
                oracle_port.lf2d_sparser(name, p, beta, -1.0, i1, i2, a, 0)
                oracle_ref.lf2d_sparser(name, p, beta, -1.0, i1, i2, b, 0)
                assert np.array_equal(a, b)


def test_pin_mvmult(oracle_port, oracle_ref):
    rng = np.random.default_rng(5)
    nnz = 2000
    a = rng.standard_normal(nnz)
    i = rng.integers(1, 101, nnz).astype(np.int64)
    j = rng.integers(1, 151, nnz).astype(np.int64)
    vec = rng.standard_normal(150)
    x, y = np.zeros(100), np.zeros(100)
    oracle_port.mvmult(x, vec, a, i, j)
    oracle_ref.mvmult(y, vec, a, i, j)
    assert np.array_equal(x, y)


def test_pin_failure_paths(oracle_port, oracle_ref):
    xos = np.array([1.0, 0, 0, -5.0, 0, 1.0, 0, 0, 0, 0, 1.0, 0])
    xsd = np.array([1.0, 0, 0, -10.0, 0, 1.0, 0, 9.0, 0, 0, 1.0, 10.0])
    sc = G.Scan3D(12, 10, 8, 1.0, 3, 20, 18, 1.0, 1.0, G.TRTT_CONE_BEAM, xos[None], xsd[None])
    vol = np.ones((8, 10, 12))
    for orc in (oracle_port, oracle_ref):
        for tab in (None, F.make_footprint(3, 1001)):
            assert orc.cb3d(np.zeros((18, 20)), vol, sc, 0, 0, tab) == -1
