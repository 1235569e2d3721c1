"""GPU parity of the group kernels (views related by turns of the volume
grid share their footprint evaluation) against the FP64 oracle and against
the per-view kernels (set_symmetry(False)).

Cases cover quarter-turn quads, half-turn pairs on rectangular grids of
even rows or even columns, mixed singles/pairs/quads, detector offsets,
parallel beam, detectors split into several u tiles, several detector-row
bands, transposes split over several launches, and an all-zero volume."""

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import geometry as G, phantoms as P

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _scan(nx=24, ny=24, nz=16, nu=40, nv=36, views=8, mode=G.TRTT_CONE_BEAM, us=1.0, vs=1.0,
          rsc=60.0, rsd=90.0, theta=None, **kw):
    return G.circular_scan_3d(nx, ny, nz, 1.0, 3, nu, nv, us, vs, views, mode=mode, rsc=rsc,
                              rsd=rsd, theta=theta, **kw)


CASES = {
    "quads": (dict(), (0, 0, 2)),
    "quads_offsets": (dict(views=12, u_off=2.3, v_off=-1.7), (0, 0, 3)),
    "quads_parallel": (dict(mode=G.TRTT_PARALLEL_BEAM, views=8), (0, 0, 2)),
    "pairs_even_rows": (dict(ny=20, views=8), (0, 4, 0)),
    "pairs_odd_rows": (dict(ny=19, views=6), (0, 3, 0)),
    "mixed": (dict(theta=np.deg2rad([0, 90, 180, 270, 45, 225, 10.0]), views=7), (1, 1, 1)),
    "u_tiles": (dict(nu=300, nv=70, us=0.15, vs=0.5, views=8), (0, 0, 2)),
    "u_tiles_3": (dict(nu=600, nv=40, us=0.08, vs=0.9, views=4), (0, 0, 1)),
    "bands": (dict(nu=48, nv=150, vs=0.2, views=8), (0, 0, 2)),
    "coarse_u": (dict(nu=20, nv=36, us=2.0, views=8), (0, 0, 2)),  # < 1 cell per voxel
    "odd_nu": (dict(nu=42, nv=37, views=8), (0, 0, 2)),  # scalar profile loads
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("mode", [1, 2])
def test_group_pair_matches_oracle(oracle_port, case, mode):
    """mode 1: group kernels; mode 2: the direct group kernel with member
    profiles interleaved per cell and plain updates on monotone columns."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    kw, expect = CASES[case]
    sc = _scan(**kw)
    name = "CB3D" if sc.mode == G.TRTT_CONE_BEAM else "PB3D"
    assert tuple(len([g for g in G.view_groups(sc) if len(g) == n]) for n in (1, 2, 4)) == expect
    pr = Projector3D(sc)
    pr.set_symmetry(mode)
    assert pr.groups() == expect
    vol = np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=7, seed=3, dtype=np.float64))
    xt = torch.tensor(vol, dtype=torch.float32, device="cuda")
    det = pr.forward(xt)
    rng = np.random.default_rng(5)
    y = torch.tensor(rng.random((sc.nviews, sc.nv, sc.nu)), dtype=torch.float32, device="cuda")
    back = pr.backward(y)
    pr.status()
    # the per-view kernels on the same plan
    pr.set_symmetry(False)
    det1 = pr.forward(xt)
    back1 = pr.backward(y)
    pr.status()
    d, d1 = det.double().cpu().numpy(), det1.double().cpu().numpy()
    b, b1 = back.double().cpu().numpy(), back1.double().cpu().numpy()
    assert rel_l2(d, d1) <= 1e-6 and rel_l2(b, b1) <= 1e-6
    volr = np.ascontiguousarray(xt.double().cpu().numpy())
    yh = y.double().cpu().numpy()
    ref_b = np.zeros_like(vol)
    for v in range(sc.nviews):
        ref = np.zeros((sc.nv, sc.nu))
        assert oracle_port._p3d(name, ref, volr, sc, v, 0, None) == 0
        assert rel_l2(d[v], ref) <= TOL, (case, v, rel_l2(d[v], ref))
        assert oracle_port._p3d(name, ref_b, np.ascontiguousarray(yh[v]), sc, v, 1, None) == 0
    assert rel_l2(b, ref_b) <= TOL, (case, rel_l2(b, ref_b))


def test_group_tiles_and_chunked_transpose(oracle_port):
    """Other band heights and a transpose split into one launch per group."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    sc = _scan(views=16, nu=44, nv=40)
    pr = Projector3D(sc)
    assert pr.groups() == (0, 0, 4)
    vol = torch.tensor(P.ellipsoids_3d(24, 24, 16, n=6, seed=8), device="cuda")
    y = torch.rand(sc.nviews, sc.nv, sc.nu, device="cuda")
    ref_f = pr.forward(vol).double().cpu().numpy()
    ref_b = pr.backward(y).double().cpu().numpy()
    for rows in (2, 7, 40):
        pr.set_group_tiles(band_rows4=rows, back_chunk_bytes=4 * sc.nu * sc.nv * 4)
        f = pr.forward(vol).double().cpu().numpy()
        b = pr.backward(y).double().cpu().numpy()
        pr.status()
        assert rel_l2(f, ref_f) <= 1e-6, rows
        assert rel_l2(b, ref_b) <= 1e-6, rows
    vol64 = np.ascontiguousarray(vol.double().cpu().numpy())
    for v in (0, 5, 15):
        r = np.zeros((sc.nv, sc.nu))
        oracle_port.cb3d(r, vol64, sc, v, 0)
        assert rel_l2(f[v], r) <= TOL


def test_group_zero_volume_and_accumulate():
    """An all-zero volume adds nothing; the projection accumulates into
    `out` like the per-view kernels."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    sc = _scan(views=8)
    pr = Projector3D(sc)
    out = torch.full((sc.nviews, sc.nv, sc.nu), 0.5, device="cuda")
    pr.forward(torch.zeros(16, 24, 24, device="cuda"), out=out)
    pr.status()
    assert torch.all(out == 0.5)
    vol = torch.tensor(P.ellipsoids_3d(24, 24, 16, n=5, seed=1), device="cuda")
    once = pr.forward(vol)
    pr.forward(vol, out=out)
    assert rel_l2((out - 0.5).double().cpu().numpy(), once.double().cpu().numpy()) <= 1e-6


def test_group_adjoint_fp64():
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    sc = _scan(nx=32, ny=32, nz=20, nu=52, nv=48, views=12)
    pr = Projector3D(sc)
    assert pr.groups() == (0, 0, 3)
    rng = np.random.default_rng(2)
    x = torch.tensor(rng.random((sc.nz, sc.ny, sc.nx)), dtype=torch.float32, device="cuda")
    y = torch.tensor(rng.random((sc.nviews, sc.nv, sc.nu)), dtype=torch.float32, device="cuda")
    hx = pr.forward(x).double().cpu().numpy()
    hty = pr.backward(y).double().cpu().numpy()
    lhs = float(np.sum(hx * y.double().cpu().numpy()))
    rhs = float(np.sum(x.double().cpu().numpy() * hty))
    assert abs(lhs - rhs) / (np.linalg.norm(hx) * np.linalg.norm(y.cpu().numpy())) <= 1e-6


@pytest.mark.parametrize("case", ["quads", "mixed", "u_tiles"])
@pytest.mark.parametrize("job", [0, 1])
def test_group_batch_entry_point(oracle_port, case, job):
    """The host-buffer batch call runs grouped scans through the group
    kernels in chunks of groups (reads back / uploads each chunk's views as
    runs of consecutive views); overwrite and accumulate modes."""
    from yoricktrtt_b200 import _lib
    kw, _ = CASES[case]
    if case == "quads":
        kw = dict(views=24)
    sc = _scan(**kw)
    rng = np.random.default_rng(13)
    vol = np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=6, seed=4, dtype=np.float64))
    det = rng.random((sc.nviews, sc.nv, sc.nu))
    inp = vol if job == 0 else det
    shape = (sc.nviews, sc.nv, sc.nu) if job == 0 else vol.shape
    ref = np.zeros(shape)
    for v in range(sc.nviews):
        if job == 0:
            oracle_port.cb3d(ref[v], vol, sc, v, 0)
        else:
            oracle_port.cb3d(ref, np.ascontiguousarray(det[v]), sc, v, 1)
    lib = _lib.load()
    xos, xsd = np.ascontiguousarray(sc.xos), np.ascontiguousarray(sc.xsd)

    def call(out, acc):
        rc = lib.trtt_b200_cb3d_batch_ex(
            _lib.dptr(out), _lib.dptr(inp), sc.nx, sc.ny, sc.nz, sc.s_scl, sc.s_deg, None, 0,
            1.0, None, sc.nu, sc.nv, sc.u_scl, sc.v_scl, sc.nviews, _lib.dptr(xos),
            _lib.dptr(xsd), 4, job, acc)
        assert rc == 0, _lib.last_error()

    out = np.full(shape, np.nan)
    call(out, 0)
    assert np.isfinite(out).all() and rel_l2(out, ref) <= TOL
    call(out, 1)
    assert rel_l2(out, 2 * ref) <= TOL


@pytest.mark.parametrize("job", [0, 1])
def test_group_batch_pageable_large(oracle_port, job):
    """The batch call on pageable (numpy) arrays of more than 4 MB: the
    input passes through the pinned staging ring, and the accumulated
    transpose is added into the host volume on the host (the FP32
    contribution comes back, not an FP64 round trip of out); overwrite and
    accumulate modes, grouped views."""
    from yoricktrtt_b200 import _lib
    sc = _scan(nx=96, ny=96, nz=96, nu=128, nv=128, views=8, rsc=300.0, rsd=450.0)
    rng = np.random.default_rng(17)
    vol = np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=6, seed=5, dtype=np.float64))
    det = rng.random((sc.nviews, sc.nv, sc.nu))
    inp = vol if job == 0 else det
    shape = (sc.nviews, sc.nv, sc.nu) if job == 0 else vol.shape
    assert 8 * vol.size >= 4 << 20  # the volume passes the 4 MB staging threshold
    ref = np.zeros(shape)
    for v in range(sc.nviews):
        if job == 0:
            oracle_port.cb3d(ref[v], vol, sc, v, 0)
        else:
            oracle_port.cb3d(ref, np.ascontiguousarray(det[v]), sc, v, 1)
    lib = _lib.load()
    xos, xsd = np.ascontiguousarray(sc.xos), np.ascontiguousarray(sc.xsd)

    def call(out, acc):
        rc = lib.trtt_b200_cb3d_batch_ex(
            _lib.dptr(out), _lib.dptr(inp), sc.nx, sc.ny, sc.nz, sc.s_scl, sc.s_deg, None, 0,
            1.0, None, sc.nu, sc.nv, sc.u_scl, sc.v_scl, sc.nviews, _lib.dptr(xos),
            _lib.dptr(xsd), 4, job, acc)
        assert rc == 0, _lib.last_error()

    out = np.full(shape, np.nan)
    call(out, 0)
    assert np.isfinite(out).all() and rel_l2(out, ref) <= TOL
    pre = rng.random(shape)
    out = pre.copy()
    call(out, 1)
    assert rel_l2(out - pre, ref) <= TOL


def test_group_quad_shapes(oracle_port):
    """Other shapes of the quad direct kernel (band rows, cells per u tile,
    CTAs per SM with their register budget) give the same projection."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    sc = _scan(views=8, nu=100, nv=60, us=0.6)
    pr = Projector3D(sc)
    vol = torch.tensor(P.ellipsoids_3d(24, 24, 16, n=6, seed=9), device="cuda")
    ref = pr.forward(vol).double().cpu().numpy()
    for shape in [(16, 32, 2), (32, 64, 1), (8, 0, 2), (60, 50, 1)]:
        pr.set_group_shape(*shape)
        got = pr.forward(vol).double().cpu().numpy()
        pr.status()
        assert rel_l2(got, ref) <= 1e-6, shape
    vol64 = np.ascontiguousarray(vol.double().cpu().numpy())
    for v in (0, 3, 7):
        r = np.zeros((sc.nv, sc.nu))
        oracle_port.cb3d(r, vol64, sc, v, 0)
        assert rel_l2(got[v], r) <= TOL
