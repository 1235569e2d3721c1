"""2D distance-driven projector pair (the reference's Yorick evaluators
``_trtt_single_distance_driven_{PB,FB}2D_projector``,
Ytrtt_2D_projectors.i:943-1245).

CPU: the FP64 restatement of the reference's merged-boundary algorithm
(oracle/dd2d_oracle.py; Yorick cannot run here) agrees with an independent
overlap formulation, is an adjoint pair, conserves mass in parallel beam and
converges to analytic line integrals of ellipses (with the right
orientation: a mirrored phantom is far off).  In parallel beam it is pinned
to compiled reference code: the reference's C distance-driven 3D projector
(trtt_DD_PB3D) on a one-slice scan gives the same projection times the
slice thickness; the fan beam converges to it as the source recedes.
GPU: trtt_b200_dd2d (FP64 kernels) against the oracle at <= 1e-12 relative
max error, accumulating onto a non-zero output; the operator class; the
source-plane failure.
"""
import numpy as np
import pytest

from yoricktrtt_b200 import analytic as A, geometry as G

from oracle import dd2d_oracle as D

SHAPES = [(24, 20, 40, 1.0, 1.0), (30, 30, 25, 0.8, 1.7), (16, 22, 70, 1.3, 0.4), (21, 13, 17, 1.0, 1.3)]
MODES = [G.TRTT_PARALLEL_BEAM, G.TRTT_FAN_BEAM]


def _scan(mode, nx, ny, nv, s, v, views=9, rsc=60.0, rsd=90.0):
    return G.circular_scan_2d(nx, ny, s, 3, nv, v, views, mode=mode, rsc=rsc, rsd=rsd,
                              arc=2.0 * np.pi)


def _oracle(fn, sc, x, job):
    xo, xs = G.dd_coefs_2d(sc)
    if job == 0:
        out = np.zeros((sc.nviews, sc.nv))
        for k in range(sc.nviews):
            fn(out[k], x, sc.nx, sc.ny, sc.s_scl, sc.nv, sc.v_scl, xo[k], xs[k], sc.mode, 0)
    else:
        out = np.zeros((sc.ny, sc.nx))
        for k in range(sc.nviews):
            fn(out, x[k], sc.nx, sc.ny, sc.s_scl, sc.nv, sc.v_scl, xo[k], xs[k], sc.mode, 1)
    return out


def _relmax(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", SHAPES)
def test_oracle_forms_agree_and_adjoint(mode, shape):
    sc = _scan(mode, *shape)
    rng = np.random.default_rng(sum(shape[:3]))
    img = rng.random((sc.ny, sc.nx))
    det = rng.random((sc.nviews, sc.nv))
    f = _oracle(D.dd2d, sc, img, 0)
    b = _oracle(D.dd2d, sc, det, 1)
    assert _relmax(f, _oracle(D.dd2d_overlap, sc, img, 0)) <= 1e-13
    assert _relmax(b, _oracle(D.dd2d_overlap, sc, det, 1)) <= 1e-13
    lhs, rhs = (f * det).sum(), (img * b).sum()
    assert abs(lhs - rhs) <= 1e-13 * abs(lhs)


@pytest.mark.parametrize("shape", SHAPES)
def test_parallel_pinned_to_reference_dd_pb3d(oracle_ref, shape):
    """Parallel beam pinned to compiled reference code: on a one-slice scan
    (nz = 1, a 3-row detector whose rows are one voxel high) the centre row
    of the reference's trtt_DD_PB3D equals s times the 2D distance-driven
    projection (the slice is s thick), cell by cell.  The C
    projector leaves the last cell of each detector axis empty (its own edge
    handling: a one-row detector gets nothing), so that cell is excluded."""
    nx, ny, nv, s, v = shape
    th = np.linspace(0.0, np.pi, 7, endpoint=False) + 0.1
    s2 = G.circular_scan_2d(nx, ny, s, 3, nv, v, len(th), mode=G.TRTT_PARALLEL_BEAM, theta=th)
    s3 = G.circular_scan_3d(nx, ny, 1, s, 3, 3, nv, s, v, len(th), mode=G.TRTT_PARALLEL_BEAM, theta=th)
    xo, xs = G.dd_coefs_2d(s2)
    img = np.random.default_rng(nx * ny).random((ny, nx))
    for k in range(len(th)):
        a = np.zeros(nv)
        D.dd2d(a, img, nx, ny, s, nv, v, xo[k], xs[k], D.PARALLEL, 0)
        b = np.zeros((nv, 3))
        assert oracle_ref.dd_pb3d(b, np.ascontiguousarray(img[None]), s3, k, 0) == 0
        assert np.abs(b[:-1, 1] - s * a[:-1]).max() <= 1e-13 * np.abs(s * a).max()
        assert b[-1, 1] == 0.0 and not b[:, 0].any() and not b[:, 2].any()


def test_fan_tends_to_pinned_parallel():
    """Fan beam tied to the pinned parallel beam: with the detector through
    the isocentre (rsd = rsc) and the source receding, the fan projection
    (magnification and distortion -> 1) converges to the parallel one, the
    difference falling as 1/rsc."""
    nx, ny, nv = 24, 20, 40
    th = np.linspace(0.0, 2.0 * np.pi, 9, endpoint=False) + 0.2
    img = np.random.default_rng(0).random((ny, nx))
    par = G.circular_scan_2d(nx, ny, 1.0, 3, nv, 1.0, len(th), mode=G.TRTT_PARALLEL_BEAM, theta=th)
    ref = _oracle(D.dd2d, par, img, 0)
    errs = []
    for rsc in (1e3, 1e4, 1e5):
        fan = G.circular_scan_2d(nx, ny, 1.0, 3, nv, 1.0, len(th), mode=G.TRTT_FAN_BEAM, rsc=rsc,
                                 rsd=rsc, theta=th)
        errs.append(_relmax(_oracle(D.dd2d, fan, img, 0), ref))
    assert errs[2] <= 1e-3
    assert 5.0 < errs[0] / errs[1] < 20.0 and 5.0 < errs[1] / errs[2] < 20.0


def test_parallel_mass():
    """Parallel beam, detector wider than the object: every view's row sums
    to the image mass (the pixel intervals are partitioned among cells)."""
    sc = _scan(G.TRTT_PARALLEL_BEAM, 20, 16, 60, 1.0, 0.9)
    img = np.random.default_rng(3).random((sc.ny, sc.nx))
    f = _oracle(D.dd2d, sc, img, 0)
    assert np.allclose(f.sum(axis=1), img.sum() * sc.s_scl ** 2, rtol=1e-13)


@pytest.mark.parametrize("mode", MODES)
def test_oracle_matches_analytic(mode):
    ell = [(0.0, 0.0, 40.0, 30.0, 0.3, 1.0), (12.0, -8.0, 10.0, 6.0, 1.1, 0.5),
           (-15.0, 10.0, 7.0, 12.0, 0.2, -0.3)]
    errs = []
    for s in (1.0, 0.5):
        nx = int(110 / s)
        sc = G.circular_scan_2d(nx, nx, s, 3, 240, 0.75, 8, mode=mode, rsc=300.0, rsd=450.0)
        img = A.ellipse_image(ell, nx, nx, s, 4)
        ana = A.sinogram_2d(ell, sc)
        out = _oracle(D.dd2d_overlap, sc, img, 0)
        errs.append(np.linalg.norm(out - ana) / np.linalg.norm(ana))
        mir = _oracle(D.dd2d_overlap, sc, np.ascontiguousarray(img[::-1]), 0)
        assert np.linalg.norm(mir - ana) / np.linalg.norm(ana) > 0.1
    assert errs[1] <= 3e-3 and errs[1] < errs[0]


# -- GPU ---------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("job", [0, 1])
def test_dd2d_gpu_matches_oracle(mode, shape, job):
    from yoricktrtt_b200 import dropin
    sc = _scan(mode, *shape, views=13)
    rng = np.random.default_rng(7 + job)
    x = rng.random((sc.ny, sc.nx)) if job == 0 else rng.random((sc.nviews, sc.nv))
    ref = _oracle(D.dd2d, sc, x, job)
    pre = rng.random(ref.shape)
    out = pre.copy()
    dropin.dd2d(out, np.ascontiguousarray(x), sc, job)
    assert _relmax(out - pre, ref) <= 1e-12


@pytest.mark.gpu
def test_dd2d_gpu_operator_views_and_adjoint():
    from yoricktrtt_b200 import dropin
    sc = _scan(G.TRTT_FAN_BEAM, 64, 48, 96, 0.7, 0.6, views=40, rsc=120.0, rsd=200.0)
    op = dropin.DistanceDriven2D(sc)
    rng = np.random.default_rng(5)
    img = rng.random((sc.ny, sc.nx))
    det = rng.random((sc.nviews, sc.nv))
    f, b = op(img, 0), op(det, 1)
    assert abs((f * det).sum() - (img * b).sum()) <= 1e-12 * abs((f * det).sum())
    k = 17
    assert _relmax(op.single_view(k)(img, 0), f[k]) <= 1e-14
    assert _relmax(op(det[10:25], 1, view0=10, nview=15), _oracle(D.dd2d, _sub(sc, 10, 25), det[10:25], 1)) <= 1e-12


def _sub(sc, a, b):
    return G.Scan2D(sc.nx, sc.ny, sc.s_scl, sc.s_deg, sc.nv, sc.v_scl, sc.mode, sc.xos[a:b], sc.xsd[a:b],
                    sc.theta[a:b], sc.rsc, sc.rsd)


@pytest.mark.gpu
def test_dd2d_gpu_source_plane():
    """Fan beam with the source on a column of pixel centres (x_s == 0
    there): the call fails and leaves out unchanged, as the reference raises
    an error."""
    from yoricktrtt_b200 import _lib, dropin
    sc = G.circular_scan_2d(10, 10, 1.0, 3, 30, 1.0, 1, mode=G.TRTT_FAN_BEAM, rsc=4.5, rsd=20.0,
                            theta=[np.pi])
    xo, xs = G.dd_coefs_2d(sc)
    assert abs(xo[0, 4]) < abs(xo[0, 5]) and xo[0, 0] * -4.5 + xo[0, 3] == 0.0
    out = np.full((1, 30), 0.5)
    with pytest.raises(_lib.TrttError):
        dropin.dd2d(out, np.ones((10, 10)), sc, 0)
    assert np.all(out == 0.5)


# launch paths of the fan-beam direct kernel: a second grid row of cell
# blocks (more than 1024 detector cells), the shared-memory table above
# 48 KB (opt-in), and the per-cell kernel when the table would exceed 200 KB
FAN_PATHS = [
    ("cell_blocks", dict(nx=8, ny=6, nv=1500, s=1.0, v=0.05, views=3)),
    ("table_above_48k", dict(nx=3200, ny=4, nv=160, s=0.1, v=3.0, views=4)),
    ("per_cell_fallback", dict(nx=13000, ny=2, nv=120, s=0.02, v=3.0, views=4)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", FAN_PATHS)
def test_dd2d_gpu_fan_launch_paths(name, kw):
    from yoricktrtt_b200 import dropin
    k = dict(kw)
    views = k.pop("views")
    sc = _scan(G.TRTT_FAN_BEAM, k["nx"], k["ny"], k["nv"], k["s"], k["v"], views=views,
               rsc=600.0, rsd=900.0)
    rng = np.random.default_rng(21)
    img = rng.random((sc.ny, sc.nx))
    ref = _oracle(D.dd2d, sc, img, 0)
    assert np.abs(ref).max() > 0, name
    pre = rng.random(ref.shape)
    out = pre.copy()
    dropin.dd2d(out, np.ascontiguousarray(img), sc, 0)
    assert _relmax(out - pre, ref) <= 1e-12, name
