"""Cone-beam distance-driven 3D pair: the reference's trtt_DD_CB3D, which
it carries commented out and unfinished (plugin/trtt_3D_projectors.c:
1340-1434), completed with its intent (oracle/trtt_oracle.c orc_DD_CB3D).

CPU: the oracle pair is an exact adjoint (FP64), conserves each voxel's
cone-beam detector integral s^3 magn^2 delta_u delta_v when its footprint
lies inside the detector, and tends to the reference's compiled
trtt_DD_PB3D (oracle/_ref) as the source recedes, the error falling as
1/rsc: the parallel limit pins it to compiled reference code.
GPU: trtt_DD_CB3D / trtt_b200_dd_cb3d (FP64 kernels) against the oracle at
<= 1e-12 relative max error, accumulating onto a non-zero output; FP64
adjoint test of the GPU pair; the source-plane failure."""
import numpy as np
import pytest

from yoricktrtt_b200 import geometry as G, phantoms as P


def _scan(n=16, nz=12, nu=28, nv=26, views=4, rsc=60.0, rsd=90.0, us=1.0, vs=1.0, theta=None,
          **kw):
    th = np.deg2rad([0.0, 17.0, 45.0, 100.0, 200.0, 311.0])[:views] if theta is None else theta
    return G.circular_scan_3d(n, n, nz, 1.0, 3, nu, nv, us, vs, len(th), mode=G.TRTT_CONE_BEAM,
                              rsc=rsc, rsd=rsd, theta=th, **kw)


def _vol(sc, seed=1):
    return np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=5, seed=seed,
                                                dtype=np.float64))


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("kw", [{}, dict(us=0.7, vs=1.3), dict(u_off=2.5, v_off=-1.5),
                                dict(nu=12, nv=10)])
def test_oracle_adjoint(oracle_port, kw):
    sc = _scan(**kw)
    rng = np.random.default_rng(3)
    vol = rng.random((sc.nz, sc.ny, sc.nx))
    for v in range(sc.nviews):
        y = rng.random((sc.nv, sc.nu))
        hx = np.zeros((sc.nv, sc.nu))
        hty = np.zeros_like(vol)
        assert oracle_port.dd_cb3d(hx, vol, sc, v, 0) == 0
        assert oracle_port.dd_cb3d(hty, y, sc, v, 1) == 0
        lhs, rhs = float((hx * y).sum()), float((vol * hty).sum())
        assert abs(lhs - rhs) <= 1e-13 * abs(lhs)


def test_oracle_conserves_cone_beam_integral(oracle_port):
    """A voxel whose footprint is inside the detector puts s^3 magn^2
    delta_u delta_v (the integral trtt_CB3D's weight carries) on it."""
    sc = _scan(n=8, nz=6, nu=40, nv=40, views=3, us=0.5, vs=0.5)
    for v in range(sc.nviews):
        for (i, j, k) in [(0, 0, 0), (3, 4, 2), (7, 7, 5)]:
            vol = np.zeros((sc.nz, sc.ny, sc.nx))
            vol[k, j, i] = 1.0
            out = np.zeros((sc.nv, sc.nu))
            oracle_port.dd_cb3d(out, vol, sc, v, 0)
            # the B-spline cone-beam projector of the same voxel carries the
            # same total (its footprint weights sum to one)
            ref = np.zeros_like(out)
            oracle_port.cb3d(ref, vol, sc, v, 0)
            assert abs(out.sum() - ref.sum()) <= 1e-12 * ref.sum(), (v, i, j, k)


def test_parallel_limit_pinned_to_reference_dd_pb3d(oracle_port, oracle_ref):
    """Detector through the isocentre (rsd = rsc): as the source recedes the
    cone-beam footprints tend to the parallel-beam ones of the reference's
    compiled trtt_DD_PB3D, the difference falling as 1/rsc.  Transposes are
    compared where no v cell is fully covered by a footprint (v cells twice
    the voxel size), since the reference's parallel transpose writes fully
    covered v cells into one slot."""
    n, nz = 16, 12
    vol = np.ascontiguousarray(P.ellipsoids_3d(n, n, nz, n=5, seed=1, dtype=np.float64))
    th = np.deg2rad([0.0, 17.0, 45.0, 100.0])
    scp = G.circular_scan_3d(n, n, nz, 1.0, 3, 28, 26, 1.0, 1.0, 4, mode=G.TRTT_PARALLEL_BEAM,
                             theta=th)
    errs = []
    for rsc in (1e3, 1e4, 1e5):
        sc = G.circular_scan_3d(n, n, nz, 1.0, 3, 28, 26, 1.0, 1.0, 4, mode=G.TRTT_CONE_BEAM,
                                rsc=rsc, rsd=rsc, theta=th)
        e = 0.0
        for v in range(4):
            a, b = np.zeros((26, 28)), np.zeros((26, 28))
            assert oracle_port.dd_cb3d(a, vol, sc, v, 0) == 0
            assert oracle_ref.dd_pb3d(b, vol, scp, v, 0) == 0
            e = max(e, np.linalg.norm(a - b) / np.linalg.norm(b))
        errs.append(e)
    assert errs[2] < 2e-4
    assert errs[0] / errs[1] > 5 and errs[1] / errs[2] > 5, errs
    # transposes, 2 mm v cells
    scp2 = G.circular_scan_3d(n, n, nz, 1.0, 3, 28, 14, 1.0, 2.0, 4, mode=G.TRTT_PARALLEL_BEAM,
                              theta=th)
    sc2 = G.circular_scan_3d(n, n, nz, 1.0, 3, 28, 14, 1.0, 2.0, 4, mode=G.TRTT_CONE_BEAM,
                             rsc=1e6, rsd=1e6, theta=th)
    y = np.random.default_rng(2).random((14, 28))
    for v in range(4):
        a, b = np.zeros_like(vol), np.zeros_like(vol)
        oracle_port.dd_cb3d(a, y, sc2, v, 1)
        oracle_ref.dd_pb3d(b, y, scp2, v, 1)
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [{}, dict(us=0.7, vs=1.3), dict(u_off=2.5, v_off=-1.5),
                                dict(nu=12, nv=10), dict(rsc=40.0, rsd=55.0)])
@pytest.mark.parametrize("job", [0, 1])
def test_gpu_parity(oracle_port, kw, job):
    from yoricktrtt_b200 import dropin
    sc = _scan(views=6, **kw)
    vol = _vol(sc)
    rng = np.random.default_rng(9)
    det = rng.random((sc.nviews, sc.nv, sc.nu))
    # per view through the drop-in symbol, accumulating onto non-zero data
    for v in range(sc.nviews):
        x = vol if job == 0 else np.ascontiguousarray(det[v])
        shape = (sc.nv, sc.nu) if job == 0 else vol.shape
        pre = rng.random(shape)
        ref, got = pre.copy(), pre.copy()
        assert oracle_port.dd_cb3d(ref, x, sc, v, job) == 0
        dropin.dd_cb3d(got, x, sc, v, job)
        assert _relmax(got - pre, ref - pre) <= 1e-12
    # all views in one call
    if job == 0:
        ref = np.zeros((sc.nviews, sc.nv, sc.nu))
        for v in range(sc.nviews):
            oracle_port.dd_cb3d(ref[v], vol, sc, v, 0)
        got = np.zeros_like(ref)
        dropin.dd_cb3d_batch(got, vol, sc, 0)
    else:
        ref = np.zeros_like(vol)
        for v in range(sc.nviews):
            oracle_port.dd_cb3d(ref, np.ascontiguousarray(det[v]), sc, v, 1)
        got = np.zeros_like(vol)
        dropin.dd_cb3d_batch(got, det, sc, 1)
    assert _relmax(got, ref) <= 1e-12


@pytest.mark.gpu
def test_gpu_adjoint_and_failure():
    from yoricktrtt_b200 import _lib, dropin
    sc = _scan(n=20, nz=14, nu=36, nv=32, views=6)
    rng = np.random.default_rng(4)
    x = rng.random((sc.nz, sc.ny, sc.nx))
    y = rng.random((sc.nviews, sc.nv, sc.nu))
    hx = np.zeros_like(y)
    hty = np.zeros_like(x)
    dropin.dd_cb3d_batch(hx, x, sc, 0)
    dropin.dd_cb3d_batch(hty, y, sc, 1)
    lhs, rhs = float((hx * y).sum()), float((x * hty).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # a voxel centre in the source plane: -1, out unchanged
    nx, ny, nz, nu, nv = 12, 10, 8, 20, 18
    xos = np.array([1.0, 0, 0, -5.0, 0, 1.0, 0, 0, 0, 0, 1.0, 0])
    xsd = np.array([1.0, 0, 0, -10.0, 0, 1.0, 0, 9.0, 0, 0, 1.0, 10.0])
    vol = np.ones((nz, ny, nx))
    out = np.full((nv, nu), 3.0)
    rc = _lib.load().trtt_DD_CB3D(_lib.dptr(out), _lib.dptr(vol), nx, ny, nz, 1.0, nu, nv, 1.0,
                                  1.0, _lib.dptr(xos), _lib.dptr(xsd), 0)
    assert rc == -1 and "source plane" in _lib.last_error()
    assert np.all(out == 3.0)
