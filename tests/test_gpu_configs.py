"""GPU parity at the benchmarked configurations, against the FP64 oracle.

The other GPU tests use small scans; these run the kernels at the sizes the
benchmarks time (so the launch shapes, band sizes, register spread and view
chunking are the benchmarked ones) and compare sampled views with the FP64
oracle, whose per-view calls run on all host threads (ctypes releases the
GIL):

* cone beam 256^3 -> 360 x 512^2, SID 1000 mm, SDD 1500 mm, 1 mm cells: the
  full 360-view forward and transpose launches, 8 sampled views checked;
  closed-form cubic footprint on the ellipsoid phantom and on a dense volume
  (every voxel non-zero, as a reconstruction iterate is); tabulated
  footprint with 10 001 samples; and a count of table-slot flips (a GPU
  table index whose floor differs from the reference's);
* fan beam 512^2 -> 720 views over 2 pi, 1024 cells, 0.5 mm: B-spline
  (closed form and table) and Long-Fessler, forward on sampled views and the
  transpose of all views;
* 4D: 10 gates of 128x128x64 with 20-60 views per gate (uneven), 256^2
  detector, tiles chosen by the autotuner, every view checked.

Bar: relative L2 <= 1e-5 per projection (the projectors compute in FP32).
"""
import concurrent.futures as cf
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import footprint as F, geometry as G, phantoms as P

pytestmark = pytest.mark.gpu

TOL = 1e-5
THREADS = max(1, min(32, os.cpu_count() or 1))
C3_SAMPLE = [0, 23, 67, 90, 149, 202, 271, 338]


def _pmap(fn, items):
    with cf.ThreadPoolExecutor(THREADS) as ex:
        return list(ex.map(fn, items))


def _c3_scan():
    return G.circular_scan_3d(256, 256, 256, 1.0, 3, 512, 512, 1.0, 1.0, 360,
                              mode=G.TRTT_CONE_BEAM, rsc=1000.0, rsd=1500.0)


@pytest.fixture(scope="module")
def c3():
    sc = _c3_scan()
    vol = P.ellipsoids_3d(256, 256, 256, n=20, seed=0, dtype=np.float32)
    return sc, vol


def _forward_views(pr, vol32, views):
    import torch
    det = pr.forward(torch.tensor(vol32, device="cuda"))
    pr.status()
    return {v: det[v].double().cpu().numpy() for v in views}


def _check_forward(orc, sc, vol32, got, table=None):
    vol64 = np.ascontiguousarray(vol32, dtype=np.float64)

    def ref(v):
        out = np.zeros((sc.nv, sc.nu))
        assert orc._p3d("CB3D", out, vol64, sc, v, 0, table) == 0
        return out

    refs = _pmap(ref, list(got))
    errs = [rel_l2(got[v], r) for v, r in zip(got, refs)]
    return max(errs), errs


def _check_transpose(orc, sc, pr, views, table=None, seed=3):
    """Transpose of the full 360-view launch with a detector stack that is
    random on `views` and zero elsewhere, against the oracle's sum over
    `views`."""
    import torch
    y = torch.zeros(sc.nviews, sc.nv, sc.nu, device="cuda")
    rng = np.random.default_rng(seed)
    yv = {v: rng.random((sc.nv, sc.nu)) for v in views}
    for v in views:
        y[v] = torch.tensor(yv[v], dtype=torch.float32)
    back = pr.backward(y)
    pr.status()
    got = back.double().cpu().numpy()

    def ref(v):
        out = np.zeros((sc.nz, sc.ny, sc.nx))
        yr = np.ascontiguousarray(y[v].double().cpu().numpy())
        assert orc._p3d("CB3D", out, yr, sc, v, 1, table) == 0
        return out

    total = np.zeros_like(got)
    for r in _pmap(ref, views):
        total += r
    return rel_l2(got, total)


def test_c3_cubic_phantom(oracle_port, c3):
    from yoricktrtt_b200.projectors import Projector3D
    sc, vol = c3
    pr = Projector3D(sc)
    assert pr.factorized
    worst, errs = _check_forward(oracle_port, sc, vol, _forward_views(pr, vol, C3_SAMPLE))
    print(f"C3 cubic phantom forward rel-L2 per view: {['%.2e' % e for e in errs]}")
    assert worst <= TOL
    err_b = _check_transpose(oracle_port, sc, pr, C3_SAMPLE)
    print(f"C3 cubic transpose rel-L2: {err_b:.2e}")
    assert err_b <= TOL


def test_c3_cubic_dense(oracle_port, c3):
    """Every voxel non-zero: no zero-voxel shortcut applies."""
    from yoricktrtt_b200.projectors import Projector3D
    sc, vol = c3
    rng = np.random.default_rng(1)
    dense = (vol + 0.05 + 0.1 * rng.random(vol.shape)).astype(np.float32)
    pr = Projector3D(sc)
    worst, errs = _check_forward(oracle_port, sc, dense, _forward_views(pr, dense, C3_SAMPLE[::2]))
    print(f"C3 cubic dense forward rel-L2 per view: {['%.2e' % e for e in errs]}")
    assert worst <= TOL


def test_c3_cubic_per_view_kernels(oracle_port, c3):
    """The per-view band and column kernels (view groups off) at the same
    size: long voxel columns select the row-locked spread."""
    from yoricktrtt_b200.projectors import Projector3D
    sc, vol = c3
    pr = Projector3D(sc)
    pr.set_symmetry(0)
    worst, errs = _check_forward(oracle_port, sc, vol, _forward_views(pr, vol, C3_SAMPLE[1::2]))
    print(f"C3 per-view kernels forward rel-L2 per view: {['%.2e' % e for e in errs]}")
    assert worst <= TOL
    err_b = _check_transpose(oracle_port, sc, pr, C3_SAMPLE[1::2])
    print(f"C3 per-view kernels transpose rel-L2: {err_b:.2e}")
    assert err_b <= TOL


def test_c3_table(oracle_port, c3):
    from yoricktrtt_b200.projectors import Projector3D
    sc, vol = c3
    tab = F.make_footprint(3, 10001)
    pr = Projector3D(sc, tab)
    worst, errs = _check_forward(oracle_port, sc, vol, _forward_views(pr, vol, C3_SAMPLE), tab)
    print(f"C3 table forward rel-L2 per view: {['%.2e' % e for e in errs]}")
    assert worst <= TOL
    err_b = _check_transpose(oracle_port, sc, pr, C3_SAMPLE[::2], tab)
    print(f"C3 table transpose rel-L2: {err_b:.2e}")
    assert err_b <= TOL


def test_c3_table_slot_flips(oracle_port, c3):
    """Table-slot agreement at the full configuration.  With the cumulative
    table replaced by the ramp cum[i] = i, every footprint weight is the
    integer number of table slots between two edges (about 830 per detector
    cell here), so a GPU slot that differs by one from the reference's
    changes the weight by 1/830 of itself.  The volume holds one voxel in 8
    along y and z and one in 16 along x: a detector cell then sums at most
    ~32 positive terms (16 columns, at most two voxels of each), whose FP32
    rounding stays below 2e-6 relative, while one flipped slot moves its cell
    by more than 3.7e-5.  Cells that differ by more than 5e-6
    relative are counted as flips; the count must be zero."""
    from yoricktrtt_b200.projectors import Projector3D
    sc, _ = c3
    tab = F.make_footprint(3, 10001)
    ramp = F.FootprintTable(3, tab.footprint, np.arange(tab.size, dtype=np.float64),
                            tab.coord, tab.step)
    rng = np.random.default_rng(5)
    vol = np.zeros((256, 256, 256), dtype=np.float32)
    vol[1::8, 5::8, 3::16] = (1.0 + rng.random((32, 32, 16))).astype(np.float32)
    pr = Projector3D(sc, ramp)
    got = _forward_views(pr, vol, C3_SAMPLE)
    vol64 = np.ascontiguousarray(vol, dtype=np.float64)

    def ref(v):
        out = np.zeros((sc.nv, sc.nu))
        assert oracle_port._p3d("CB3D", out, vol64, sc, v, 0, ramp) == 0
        return out

    flips = 0
    cells = 0
    for v, r in zip(C3_SAMPLE, _pmap(ref, C3_SAMPLE)):
        m = r > 1e-6 * r.max()
        cells += int(m.sum())
        flips += int((np.abs(got[v] - r)[m] > 5e-6 * r[m]).sum())
    edges = 32 * 32 * 16 * len(C3_SAMPLE) * 2 * 8
    print(f"C3 table-slot flips: {flips} cells of {cells} checked "
          f"(~{edges:.2e} footprint edges, 10 001-sample table)")
    assert flips == 0


def test_c3_batch_call_host_buffers(oracle_port, c3):
    """The end-to-end path at the benchmarked size: trtt_b200_cb3d_batch_ex
    on pinned host FP64 arrays in the reference layouts, as the bench's e2e
    leg calls it (view groups; direct view chunks alternating over two
    streams with each chunk's read-back overlapping later chunks; the
    transpose's upload chunks growing by half).  Overwrite mode (out = H in)
    on sampled views of the forward and on the transpose of a stack that is
    random on the sampled views, against the FP64 oracle; then the plugin's
    accumulate mode (out += H in) on top of the forward result."""
    import torch
    from yoricktrtt_b200 import _lib
    lib = _lib.load()
    sc, vol = c3
    vol64 = torch.from_numpy(np.ascontiguousarray(vol, dtype=np.float64)).pin_memory().numpy()
    det = torch.full((sc.nviews, sc.nv, sc.nu), 7.0, dtype=torch.float64).pin_memory().numpy()
    xos, xsd = np.ascontiguousarray(sc.xos), np.ascontiguousarray(sc.xsd)

    def call(out, inp, job, accumulate):
        rc = lib.trtt_b200_cb3d_batch_ex(_lib.dptr(out), _lib.dptr(inp), sc.nx, sc.ny, sc.nz, sc.s_scl,
                                         sc.s_deg, None, 0, 1.0, None, sc.nu, sc.nv, sc.u_scl, sc.v_scl,
                                         sc.nviews, _lib.dptr(xos), _lib.dptr(xsd), G.TRTT_CONE_BEAM, job,
                                         accumulate)
        _lib.check(rc, "trtt_b200_cb3d_batch_ex")

    call(det, vol64, 0, 0)
    got = {v: det[v].copy() for v in C3_SAMPLE}
    worst, errs = _check_forward(oracle_port, sc, vol, got)
    print(f"C3 batch call forward rel-L2 per view: {['%.2e' % e for e in errs]}")
    assert worst <= TOL
    call(det, vol64, 0, 1)  # accumulate: twice the projection
    assert max(rel_l2(det[v], 2.0 * got[v]) for v in C3_SAMPLE[:3]) <= 1e-6
    rng = np.random.default_rng(4)
    y = torch.zeros((sc.nviews, sc.nv, sc.nu), dtype=torch.float64).pin_memory().numpy()
    for v in C3_SAMPLE:
        y[v] = rng.random((sc.nv, sc.nu))
    back = torch.full((sc.nz, sc.ny, sc.nx), 3.0, dtype=torch.float64).pin_memory().numpy()
    call(back, y, 1, 0)

    def ref(v):
        out = np.zeros((sc.nz, sc.ny, sc.nx))
        assert oracle_port._p3d("CB3D", out, np.ascontiguousarray(y[v]), sc, v, 1, None) == 0
        return out

    total = np.zeros_like(back)
    for r in _pmap(ref, C3_SAMPLE):
        total += r
    err_b = rel_l2(back, total)
    print(f"C3 batch call transpose rel-L2: {err_b:.2e}")
    assert err_b <= TOL


def test_c3_dropin_per_view_pageable(oracle_port, c3):
    """The symbol an unchanged Yorick closure calls, trtt_CB3D_cubic, one
    view per call on pageable FP64 arrays at the benchmarked size: the
    volume upload passes through the pinned staging ring in several slots,
    and the transpose adds its FP32 result into the host volume on the host
    (two slots).  out += H in (and H^T) on pre-filled outputs, against the
    FP64 oracle."""
    from yoricktrtt_b200 import dropin
    sc, vol = c3
    vol64 = np.ascontiguousarray(vol, dtype=np.float64)
    rng = np.random.default_rng(6)
    for v in (0, 137):
        pre = rng.random((sc.nv, sc.nu))
        got = pre.copy()
        ref = pre.copy()
        dropin.scan3d_call("CB3D", got, vol64, sc, v, 0, None)
        assert oracle_port._p3d("CB3D", ref, vol64, sc, v, 0, None) == 0
        assert rel_l2(got - pre, ref - pre) <= TOL
        y = rng.random((sc.nv, sc.nu))
        pre_b = rng.random((sc.nz, sc.ny, sc.nx))
        got_b = pre_b.copy()
        ref_b = pre_b.copy()
        dropin.scan3d_call("CB3D", got_b, y, sc, v, 1, None)
        assert oracle_port._p3d("CB3D", ref_b, y, sc, v, 1, None) == 0
        err = rel_l2(got_b - pre_b, ref_b - pre_b)
        print(f"C3 per-view drop-in view {v}: forward {rel_l2(got - pre, ref - pre):.2e}, transpose {err:.2e}")
        assert err <= TOL


# ---------------------------------------------------------------------------
# 2D fan beam 512^2 -> 720 x 1024
# ---------------------------------------------------------------------------
def _c2_scan():
    return G.circular_scan_2d(512, 512, 0.5, 3, 1024, 0.5, 720, mode=G.TRTT_FAN_BEAM,
                              rsc=1000.0, rsd=1500.0)


@pytest.mark.parametrize("model", ["cubic", "table"])
def test_c2_fan_bspline(oracle_port, model):
    import torch
    from yoricktrtt_b200.recon import Projector2D
    sc = _c2_scan()
    tab = F.make_footprint(3, 10001) if model == "table" else None
    img = P.ellipses_2d(512, 512, n=10, seed=0).astype(np.float32)
    img64 = np.ascontiguousarray(img, dtype=np.float64)
    pr = Projector2D(sc, tab)
    det = pr.forward(torch.tensor(img, device="cuda")).double().cpu().numpy()
    views = list(range(0, 720, 45)) + [1, 359, 719]

    def ref(v):
        out = np.zeros(sc.nv)
        assert oracle_port.p2d("FB2D", out, img64, sc, v, 0, tab) == 0
        return out

    errs = [rel_l2(det[v], r) for v, r in zip(views, _pmap(ref, views))]
    print(f"C2 FB2D {model} forward max rel-L2 {max(errs):.2e}")
    assert max(errs) <= TOL
    rng = np.random.default_rng(2)
    y = rng.random((sc.nviews, sc.nv)).astype(np.float32)
    back = pr.backward(torch.tensor(y, device="cuda")).double().cpu().numpy()
    y64 = y.astype(np.float64)

    def refb(vs):
        out = np.zeros((sc.ny, sc.nx))
        for v in vs:
            assert oracle_port.p2d("FB2D", out, np.ascontiguousarray(y64[v]), sc, v, 1, tab) == 0
        return out

    total = sum(_pmap(refb, [list(range(t, 720, THREADS)) for t in range(THREADS)]))
    err_b = rel_l2(back, total)
    print(f"C2 FB2D {model} transpose rel-L2 {err_b:.2e}")
    assert err_b <= TOL


def test_c2_fan_long_fessler(oracle_port):
    import torch
    from oracle.oracle import LF2DParams as OP
    from yoricktrtt_b200 import dropin
    from yoricktrtt_b200.recon import Projector2D
    sc = _c2_scan()
    lf = dict(pixelSize=0.5, pixelStep=0.5, voxelSize=0.5, sourceDistance=1000.0,
              detectorDistance=500.0, objectOffset1=0.0, objectOffset2=0.0,
              objectDimension1=512, objectDimension2=512, detectorDimension=1024)
    beta = sc.theta - math.pi / 2
    pr = Projector2D(lf_params=dropin.LF2DParams(**lf), beta=beta, offset=np.zeros(sc.nviews))
    img = P.ellipses_2d(512, 512, n=10, seed=0).astype(np.float32)
    img64 = np.ascontiguousarray(img, dtype=np.float64)
    det = pr.forward(torch.tensor(img, device="cuda")).double().cpu().numpy()
    op = OP(**lf)
    views = list(range(0, 720, 45)) + [1, 359, 719]

    def ref(v):
        out = np.zeros(1024)
        oracle_port.lf2d("direct", op, float(beta[v]), 0.0, img64, out, 1)
        return out

    errs = [rel_l2(det[v], r) for v, r in zip(views, _pmap(ref, views))]
    print(f"C2 Long-Fessler forward max rel-L2 {max(errs):.2e}")
    assert max(errs) <= TOL
    rng = np.random.default_rng(4)
    y = rng.random((sc.nviews, 1024)).astype(np.float32)
    back = pr.backward(torch.tensor(y, device="cuda")).double().cpu().numpy()
    y64 = y.astype(np.float64)

    def refb(vs):
        out = np.zeros((512, 512))
        for v in vs:
            part = np.zeros((512, 512))
            oracle_port.lf2d("adjoint", op, float(beta[v]), 0.0, np.ascontiguousarray(y64[v]),
                             part, 1)
            out += part
        return out

    total = sum(_pmap(refb, [list(range(t, 720, THREADS)) for t in range(THREADS)]))
    err_b = rel_l2(back, total)
    print(f"C2 Long-Fessler adjoint rel-L2 {err_b:.2e}")
    assert err_b <= TOL


# ---------------------------------------------------------------------------
# 4D: 10 gates of 128 x 128 x 64, 20-60 views per gate, 256^2 detector
# ---------------------------------------------------------------------------
def test_c4_gates_autotuned(oracle_port):
    import torch
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz, xyz_from_columns
    nt = 10
    rng = np.random.default_rng(0)
    counts = rng.integers(20, 61, nt)
    t_index = np.concatenate([g + rng.uniform(0.0, 1.0, c) for g, c in enumerate(counts)])
    nviews = int(counts.sum())
    theta = np.sort(rng.uniform(0, 2 * math.pi, nviews))
    sc = G.circular_scan_3d(128, 128, 64, 1.0, 3, 256, 256, 1.0, 1.0, nviews, theta=theta)
    gates = P.breathing_gates(128, 128, 64, nt, 1.0, amplitude_mm=10.0, seed=0)
    pr = Projector3D(sc)
    pr.set_gates(nt, t_index)
    xc = columns_from_xyz(torch.tensor(gates, device="cuda"))
    _, choice = pr.autotune(xc, layout="columns", nview=nviews, reps=1)
    det = pr.forward(xc, layout="columns").double().cpu().numpy()
    y = torch.rand(nviews, 256, 256, device="cuda")
    back = xyz_from_columns(pr.backward(y, layout="columns")).double().cpu().numpy()
    pr.status()
    g64 = gates.astype(np.float64)
    y64 = y.double().cpu().numpy()

    def fwd(k):
        (g0, g1), (w0, w1) = G.gate_weights(float(t_index[k]), nt)
        bx = np.ascontiguousarray(w0 * g64[g0] + w1 * g64[g1])
        ref = np.zeros((256, 256))
        assert oracle_port.cb3d(ref, bx, sc, k, 0) == 0
        return rel_l2(det[k], ref)

    def back_chunk(ks):
        acc = np.zeros_like(g64)
        bt = np.zeros((64, 128, 128))
        for k in ks:
            (g0, g1), (w0, w1) = G.gate_weights(float(t_index[k]), nt)
            bt.fill(0.0)
            assert oracle_port.cb3d(bt, np.ascontiguousarray(y64[k]), sc, k, 1) == 0
            if g0 != g1:
                acc[g0] += w0 * bt
                acc[g1] += w1 * bt
            else:
                acc[g0] += w1 * bt  # repeated index: the second write wins
        return acc

    worst = max(_pmap(fwd, range(nviews)))
    nw = min(THREADS, 16)
    ref_back = sum(_pmap(back_chunk, [list(range(t, nviews, nw)) for t in range(nw)]))
    err_b = rel_l2(back, ref_back)
    print(f"C4 gates {counts.tolist()} tiles {choice}: forward max rel-L2 {worst:.2e}, "
          f"transpose {err_b:.2e}")
    assert worst <= TOL and err_b <= TOL
