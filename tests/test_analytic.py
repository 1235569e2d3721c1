"""Model-level checks of the projectors and the data-file readers, on the CPU.

* Raw files: the simulator's float32 files with a 512-byte header and the
  16-bit detector frames with a 100-byte header are written and read back.
* The reference's analytic cone-beam ball (tests/golden/ball, made from
  ``Tomography_3D/Simul_Data`` by make_ball.py): the voxel image equals the
  phantom file sampled at voxel centres, the simulated projections equal the
  ray-ellipsoid line integrals at the simulator's sub-pixel sample points
  (its float32 arithmetic limits the agreement to a few 1e-3), and the
  oracle cone-beam projector of the voxel image conserves the ball's mass and
  converges to the analytic projections as the voxels shrink.
* Analytic ellipse / ellipsoid projections (cell integrals of line
  integrals) against the oracle projectors of finely voxelised phantoms, in
  parallel and fan beam 2D and parallel and cone beam 3D: relative L2 error
  of a few 1e-3 (2D) and 1e-2 (3D), shrinking with the voxel size, while the
  same comparison with a mirrored or axis-swapped phantom is off by >10%,
  which pins the orientation of the detector axes; the same for the
  reference's distance-driven parallel-beam projector (trtt_DD_PB3D).
"""
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import analytic as A, geometry as G, rawio as R

BALL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ball")
BALL_VIEWS = np.arange(0, 720, 45)
BALL_THETA = 2.0 * math.pi * BALL_VIEWS / 720.0
# simulator geometry (cm): source at 100, detector 153.6 from the source,
# 0.1 cm voxels and detector cells; here in mm
RSC, RSD = 1000.0, 1536.0
# simulator units -> mm: cell area cm^2 -> mm^2 (x100), chord cm -> mm (x10)
CM3_TO_MM3 = 1000.0


def _ball():
    ph = A.read_phantom(os.path.join(BALL, "boule.obj"), (7.5, 7.5, 7.5))
    vol = R.read_raw(os.path.join(BALL, "boule.data"), (16, 16, 16))
    proj = R.read_raw(os.path.join(BALL, "proj_boule_every45.data"), (32, 32, len(BALL_VIEWS)))
    return ph, vol, proj


def _to_scan_layout(sim_proj):
    """Simulator projection [v_sim][u_sim] (u_sim along (-sin, cos, 0), v_sim
    along z) -> projector layout [v][u] (v along (sin, -cos, 0), u along z)."""
    return np.stack([np.ascontiguousarray(p[:, ::-1].T) for p in sim_proj])


def _ball_scan(n=16, s=1.0):
    return G.circular_scan_3d(n, n, n, s, 3, 32, 32, 1.0, 1.0, len(BALL_THETA),
                              theta=BALL_THETA, rsc=RSC, rsd=RSD)


def _sim_sampling(ph, sub=10, centred=False):
    """Cell integrals of the ball's line integrals on the simulator's
    detector: sub x sub samples per cell, at the cell's lower corner offsets
    as ``sim_cone.c`` takes them (or centred)."""
    m = np.arange(32 * sub)
    pos = (m - 16 * sub + (0.5 if centred else 0.0)) / sub
    U, V = np.meshgrid(pos, pos, indexing="xy")
    out = np.zeros((len(BALL_THETA), 32, 32))
    for k, th in enumerate(BALL_THETA):
        c, s = math.cos(th), math.sin(th)
        src = np.array([RSC * c, RSC * s, 0.0])
        ctr = (RSC - RSD) * np.array([c, s, 0.0])
        B = ctr + U[..., None] * np.array([-s, c, 0.0]) + V[..., None] * np.array([0.0, 0.0, 1.0])
        D = B - src
        D /= np.linalg.norm(D, axis=-1, keepdims=True)
        L = A.chord_3d(np.broadcast_to(src, B.shape), D, ph) / (sub * sub)
        out[k] = L.reshape(32, sub, 32, sub).sum(axis=(1, 3))
    return out


# -- raw files ---------------------------------------------------------------

def test_raw_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    data = rng.random((5, 7, 3)).astype(np.float32)
    p = str(tmp_path / "x.data")
    R.write_raw(p, data, header={"cb_radius": 100.0, "x_pixels": 3})
    assert os.path.getsize(p) == 512 + data.nbytes
    h = R.read_header(p)
    assert h["records"] == 5 and h["record_rows"] == 7 and h["first_data_word"] == 513
    assert h["cb_radius"] == 100.0 and h["x_pixels"] == 3
    assert h["max_x1.01"] == pytest.approx(1.01 * data.max(), rel=1e-6)
    got = R.read_raw(p, (3, 7, 5))
    assert got.shape == (5, 7, 3) and np.array_equal(got, data)
    with pytest.raises(ValueError):
        R.read_raw(p, (3, 7, 6))
    with pytest.raises(ValueError):
        R.read_raw(p, (3, 0, 5))


def test_detector_frames(tmp_path):
    rng = np.random.default_rng(1)
    paths = []
    frames = rng.integers(-2 ** 15, 2 ** 15, size=(3, 6, 4), dtype=np.int16)
    for k in range(3):
        p = str(tmp_path / f"f{k}.raw")
        with open(p, "wb") as f:
            f.write(bytes(range(100)))
            f.write(frames[k].astype("<i2").tobytes())
        paths.append(p)
    got = R.read_detector_frames(paths, 4, 6)
    assert got.shape == (3, 6, 4)
    assert np.array_equal(got, frames.astype(np.float64) + 2 ** 15)
    assert got.min() >= 0
    got2 = R.read_detector_frames(paths, 4, 6, shift=2 ** 16 - 1)
    assert np.array_equal(got2, frames.astype(np.float64) + 2 ** 16 - 1)


# -- the reference's ball fixture --------------------------------------------

def test_ball_header_and_voxel_image():
    ph, vol, _ = _ball()
    h = R.read_header(os.path.join(BALL, "boule.data"))
    assert (h["x_pixels"], h["y_pixels"], h["z_pixels"]) == (16, 16, 16)
    assert h["x_size"] == pytest.approx(0.1) and h["x_off"] == 7.5
    assert h["cb_radius"] == 100.0 and h["cb_focal"] == pytest.approx(153.6)
    hp = R.read_header(os.path.join(BALL, "proj_boule_every45.data"))
    assert hp["records"] == len(BALL_VIEWS) and hp["record_rows"] == 32
    assert len(ph) == 1 and ph[0].axes == (4.6875,) * 3
    assert ph[0].value == pytest.approx(0.1928 * 0.025)
    img = A.ellipsoid_volume(ph, 16, 16, 16, 1.0, oversample=1)
    assert np.array_equal(img.astype(np.float32), vol)
    assert (vol > 0).sum() == 432


def test_ball_projections_are_line_integrals():
    ph, _, proj = _ball()
    emu = _sim_sampling(ph)  # [k][v_sim][u_sim] in mm^3
    ref = CM3_TO_MM3 * proj.astype(np.float64)
    assert rel_l2(emu, ref) <= 5e-3
    assert np.abs(emu - ref).max() <= 1.5e-2 * ref.max()
    # a ball 2% larger (as a 2% magnification error would make it) is off
    ph2 = [A.Ellipsoid(e.center, tuple(1.02 * a for a in e.axes), e.rot, e.value) for e in ph]
    assert rel_l2(_sim_sampling(ph2), ref) > 2e-2


def test_ball_analytic_projections():
    """The public cell-integral projections equal a fine centred midpoint
    sampling; against the fixture they differ by the simulator's half
    sub-pixel sampling offset (1.7%)."""
    ph, _, proj = _ball()
    an = A.projections_3d(ph, _ball_scan(), quad=8, rsc=RSC, rsd=RSD)
    emu = _to_scan_layout(_sim_sampling(ph, sub=20, centred=True))
    assert rel_l2(an, emu) <= 1e-3
    ref = _to_scan_layout(CM3_TO_MM3 * proj.astype(np.float64))
    assert rel_l2(an, ref) <= 2.5e-2


def test_ball_cone_projector(oracle_port):
    ph, vol, proj = _ball()
    sc = _ball_scan()
    ref = _to_scan_layout(CM3_TO_MM3 * proj.astype(np.float64))
    out = np.zeros((sc.nviews, 32, 32))
    v64 = vol.astype(np.float64)
    for k in range(sc.nviews):
        assert oracle_port.cb3d(out[k], v64, sc, k, 0) == 0
    # mass: detector sums equal the voxel image's mass x magnification^2
    mass_vox = v64.sum() * (RSD / RSC) ** 2
    assert out.sum(axis=(1, 2)) == pytest.approx(np.full(sc.nviews, mass_vox), rel=2e-3)
    assert ref.sum() / out.sum() == pytest.approx(1.0, abs=5e-3)
    assert rel_l2(out, ref) <= 0.12
    # finer voxels converge to the analytic projections
    an = A.projections_3d(ph, sc, quad=8, rsc=RSC, rsd=RSD)
    fine = _ball_scan(32, 0.5)
    v = A.ellipsoid_volume(ph, 32, 32, 32, 0.5, oversample=2)
    o2 = np.zeros_like(out)
    for k in range(sc.nviews):
        oracle_port.cb3d(o2[k], v, fine, k, 0)
    assert rel_l2(o2, an) <= 0.05 < rel_l2(out, an)


# -- analytic ellipses / ellipsoids vs the oracle projectors -----------------

ELL = [(0.0, 0.0, 40.0, 30.0, 0.3, 1.0), (12.0, -8.0, 10.0, 6.0, 1.1, 0.5),
       (-15.0, 10.0, 7.0, 12.0, 0.2, -0.3)]


@pytest.mark.parametrize("mode,name,tol", [(G.TRTT_PARALLEL_BEAM, "PB2D", 5e-3),
                                           (G.TRTT_FAN_BEAM, "FB2D", 6e-3)])
def test_2d_projectors_match_analytic(oracle_port, mode, name, tol):
    errs = []
    for s in (1.0, 0.5):
        nx = int(110 / s)
        sc = G.circular_scan_2d(nx, nx, s, 3, 240, 0.75, 12, mode=mode, rsc=300.0, rsd=450.0)
        img = A.ellipse_image(ELL, nx, nx, s, 4)
        ana = A.sinogram_2d(ELL, sc)
        out = np.zeros((sc.nviews, sc.nv))
        mir = np.zeros_like(out)
        for k in range(sc.nviews):
            assert oracle_port.p2d(name, out[k], img, sc, k, 0) == 0
            oracle_port.p2d(name, mir[k], np.ascontiguousarray(img[::-1]), sc, k, 0)
        errs.append(rel_l2(out, ana))
        assert rel_l2(mir, ana) > 0.1
        # each detector row integrates to the phantom's mass (times the
        # magnification Rsd / Rsc, up to its depth variation, in fan beam)
        mass = img.sum() * s * s
        if mode == G.TRTT_PARALLEL_BEAM:
            assert ana.sum(axis=1) == pytest.approx(np.full(sc.nviews, mass), rel=1e-3)
        else:
            assert ana.sum(axis=1) == pytest.approx(np.full(sc.nviews, 1.5 * mass), rel=2e-2)
    assert errs[1] <= tol and errs[1] < errs[0]


ELLIPSOIDS = [A.ellipsoid((0, 0, 0), (35, 25, 20), 1.0, phi=0.3),
              A.ellipsoid((10, -8, 5), (9, 6, 7), 0.5, phi=1.1, theta=0.6, psi=0.4),
              A.ellipsoid((-12, 9, -6), (6, 10, 5), -0.3, phi=0.2, theta=-0.4)]


@pytest.mark.parametrize("mode,name", [(G.TRTT_CONE_BEAM, "CB3D"), (G.TRTT_PARALLEL_BEAM, "PB3D")])
def test_3d_projectors_match_analytic(oracle_port, mode, name):
    errs = []
    for n, s in ((64, 1.5), (96, 1.0)):
        sc = G.circular_scan_3d(n, n, n, s, 3, 100, 100, 1.6, 1.6, 4, mode=mode,
                                rsc=300.0, rsd=450.0)
        vol = A.ellipsoid_volume(ELLIPSOIDS, n, n, n, s, 2)
        ana = A.projections_3d(ELLIPSOIDS, sc, rsc=300.0, rsd=450.0)
        out = np.zeros((sc.nviews, sc.nv, sc.nu))
        for k in range(sc.nviews):
            assert oracle_port._p3d(name, out[k], vol, sc, k, 0, None) == 0
        errs.append(rel_l2(out, ana))
    assert errs[1] <= 0.025 and errs[1] < errs[0]
    swapped = np.ascontiguousarray(np.swapaxes(vol, 1, 2))
    o = np.zeros((sc.nv, sc.nu))
    oracle_port._p3d(name, o, swapped, sc, 1, 0, None)
    assert rel_l2(o, ana[1]) > 0.1


def test_dd_pb3d_matches_analytic(oracle_port):
    """The reference's distance-driven parallel-beam projector (trtt_DD_PB3D,
    compiled restatement) converges to the analytic ellipsoid projections and
    conserves each view's mass; swapping x and y is far off."""
    errs = []
    for n, s in ((64, 1.5), (96, 1.0)):
        sc = G.circular_scan_3d(n, n, n, s, 3, 100, 100, 1.6, 1.6, 4, mode=G.TRTT_PARALLEL_BEAM)
        vol = A.ellipsoid_volume(ELLIPSOIDS[:2], n, n, n, s, 2)
        ana = A.projections_3d(ELLIPSOIDS[:2], sc)
        out = np.zeros((sc.nviews, sc.nv, sc.nu))
        for k in range(sc.nviews):
            assert oracle_port.dd_pb3d(out[k], vol, sc, k, 0) == 0
        errs.append(rel_l2(out, ana))
        assert out.sum(axis=(1, 2)) == pytest.approx(np.full(sc.nviews, vol.sum() * s ** 3), rel=1e-9)
    assert errs[1] <= 0.012 and errs[1] < errs[0]
    o = np.zeros((sc.nv, sc.nu))
    oracle_port.dd_pb3d(o, np.ascontiguousarray(np.swapaxes(vol, 1, 2)), sc, 1, 0)
    assert rel_l2(o, ana[1]) > 0.1


def test_euler_rotation_and_tilted_chords():
    R3 = A.euler_zxz(0.7, -0.4, 1.9)
    assert np.allclose(R3 @ R3.T, np.eye(3), atol=1e-14) and np.linalg.det(R3) == pytest.approx(1.0)
    # a chord through the centre along a body axis is twice that semi-axis
    e = A.ellipsoid((1.0, -2.0, 0.5), (3.0, 2.0, 1.0), 2.0, 0.7, -0.4, 1.9)
    for r, a in enumerate(e.axes):
        d = e.rot[r]
        assert A.chord_3d(np.array(e.center) - 10 * d, d, [e]) == pytest.approx(2 * a * 2.0)
    # phi alone is the in-plane rotation of the 2D ellipse
    e2 = A.ellipsoid((3.0, 1.0, 0.0), (5.0, 2.0, 1.0), 1.0, phi=0.8)
    p = np.array([[-20.0, y, 0.0] for y in np.linspace(-4, 6, 9)])
    u = np.tile([1.0, 0.0, 0.0], (9, 1))
    assert np.allclose(A.chord_3d(p, u, [e2]),
                       A.chord_2d(p[:, :2], u[:, :2], [(3.0, 1.0, 5.0, 2.0, 0.8, 1.0)]))


def test_read_phantom_rejects_other_shapes(tmp_path):
    p = tmp_path / "c.obj"
    p.write_text("phantom\nobject 1\ncylinder\nradius 1\nlength 2\ncenter 0 0 0\nangles 0 0\n1\nend\n")
    with pytest.raises(NotImplementedError):
        A.read_phantom(str(p), (1, 1, 1))
    p.write_text("object 1 ellipsoid\n")
    with pytest.raises(ValueError):
        A.read_phantom(str(p), (1, 1, 1))


@pytest.mark.gpu
def test_ball_cone_projector_gpu(oracle_port):
    """The B200 cone-beam projector (host-buffer batch entry point) on the
    ball's voxel image: oracle parity (1e-5) and the same model-level
    agreement with the simulated projections."""
    from yoricktrtt_b200 import _lib
    _, vol, proj = _ball()
    sc = _ball_scan()
    v64 = np.ascontiguousarray(vol, dtype=np.float64)
    out = np.zeros((sc.nviews, 32, 32))
    rc = _lib.load().trtt_b200_cb3d_batch(
        _lib.dptr(out), _lib.dptr(v64), sc.nx, sc.ny, sc.nz, sc.s_scl, sc.s_deg, None, 0,
        1.0, None, sc.nu, sc.nv, sc.u_scl, sc.v_scl, sc.nviews,
        _lib.dptr(np.ascontiguousarray(sc.xos)), _lib.dptr(np.ascontiguousarray(sc.xsd)), 4, 0)
    assert rc == 0, _lib.last_error()
    for k in range(sc.nviews):
        ref = np.zeros((32, 32))
        oracle_port.cb3d(ref, v64, sc, k, 0)
        assert rel_l2(out[k], ref) <= 1e-5
    sim = _to_scan_layout(CM3_TO_MM3 * proj.astype(np.float64))
    assert rel_l2(out, sim) <= 0.12
    assert sim.sum() / out.sum() == pytest.approx(1.0, abs=5e-3)
