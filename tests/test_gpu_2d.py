"""GPU parity of the 2D projectors, sparse column generators, Long-Fessler
model, distance-driven 3D projector and COO product against the FP64
oracle, through the drop-in C ABI and the native 2D plan."""
import ctypes as C
import math

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import _lib, dropin, footprint as F, geometry as G, phantoms as P

pytestmark = pytest.mark.gpu

TOL = 1e-5
TABLE = F.make_footprint(3, 10001)


def _scan2d(mode, nx=48, ny=40, nv=80, views=5, s=1.0, vs=1.0, rsc=120.0, rsd=180.0, deg=3):
    return G.circular_scan_2d(nx, ny, s, deg, nv, vs, views, mode=mode, rsc=rsc, rsd=rsd)


def _img(sc, seed=1):
    return np.ascontiguousarray(P.ellipses_2d(sc.nx, sc.ny, n=6, seed=seed))


CASES2D = [
    ("FB2D", G.TRTT_FAN_BEAM, {}),
    ("PB2D", G.TRTT_PARALLEL_BEAM, {}),
    ("FB2D", G.TRTT_FAN_BEAM, dict(nv=40)),                 # clipped detector
    ("PB2D", G.TRTT_PARALLEL_BEAM, dict(nv=36, vs=0.7)),
    ("FB2D", G.TRTT_FAN_BEAM, dict(s=0.5, vs=0.5, deg=2)),
]


@pytest.mark.parametrize("name,mode,kw", CASES2D)
@pytest.mark.parametrize("model", ["cubic", "table"])
@pytest.mark.parametrize("job", [0, 1])
def test_2d_parity(oracle_port, name, mode, kw, model, job):
    sc = _scan2d(mode, **kw)
    table = (F.make_footprint(sc.s_deg, 10001) if model == "table" else None)
    img = _img(sc)
    rng = np.random.default_rng(3)
    for v in range(sc.nviews):
        if job == 0:
            x, shape = img, (sc.nv,)
        else:
            x, shape = rng.random(sc.nv), img.shape
        pre = rng.random(shape)
        ref, got = pre.copy(), pre.copy()
        assert oracle_port.p2d(name, ref, x, sc, v, job, table) == 0
        dropin.p2d(name, got, x, sc, v, job, table)
        assert rel_l2(got - pre, ref - pre) <= TOL


@pytest.mark.parametrize("name,mode", [("FB2D", G.TRTT_FAN_BEAM), ("PB2D", G.TRTT_PARALLEL_BEAM)])
def test_sparsers(oracle_port, name, mode):
    sc = _scan2d(mode)
    for (i, j) in [(0, 0), (5, 7), (47, 39), (20, 13), (-3, 50)]:
        for v in range(2):
            pre = np.random.default_rng(i + 17 * j).random(sc.nv)
            ref, got = pre.copy(), pre.copy()
            assert oracle_port.sparser2d(name, ref, i, j, sc, v, TABLE) == 0
            dropin.sparser2d(name, got, i, j, sc, v, TABLE)
            assert np.allclose(got, ref, rtol=1e-13, atol=1e-15)


def test_assembly_matches_sparser(oracle_port):
    import torch
    sc = _scan2d(G.TRTT_FAN_BEAM, nx=12, ny=10, nv=30, views=2)
    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.trtt_b200_plan2d_create(C.byref(h), 5, sc.nx, sc.ny, sc.s_scl, sc.s_deg,
                                     _lib.dptr(TABLE.cum), TABLE.size, TABLE.step,
                                     _lib.dptr(TABLE.coord), sc.nv, sc.v_scl, sc.nviews,
                                     _lib.dptr(np.ascontiguousarray(sc.xos)),
                                     _lib.dptr(np.ascontiguousarray(sc.xsd)))
    _lib.check(rc, "plan2d_create")
    mc = 16
    n = sc.nviews * sc.nx * sc.ny * mc
    a = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = torch.zeros(n, dtype=torch.int64, device="cuda")
    c = torch.zeros(n, dtype=torch.int64, device="cuda")
    _lib.check(lib.trtt_b200_plan2d_assemble(h, mc, C.c_void_p(a.data_ptr()),
                                             C.c_void_p(r.data_ptr()), C.c_void_p(c.data_ptr()),
                                             None), "assemble")
    torch.cuda.synchronize()
    _lib.check(lib.trtt_b200_plan2d_status(h, None), "status")
    a, r, c = a.cpu().numpy(), r.cpu().numpy(), c.cpu().numpy()
    per = sc.nx * sc.ny * mc
    for v in range(sc.nviews):
        dense = np.zeros((sc.nv, sc.nx * sc.ny))
        av, rv, cv = a[v * per:(v + 1) * per], r[v * per:(v + 1) * per], c[v * per:(v + 1) * per]
        m = rv > 0
        np.add.at(dense, (rv[m] - 1, cv[m] - 1), av[m])
        for p in range(sc.nx * sc.ny):
            col = np.zeros(sc.nv)
            oracle_port.sparser2d("FB2D", col, p % sc.nx, p // sc.nx, sc, v, TABLE)
            assert np.allclose(dense[:, p], col, rtol=1e-13, atol=1e-15)
    lib.trtt_b200_plan2d_destroy(h)


@pytest.mark.parametrize("mode,name", [(G.TRTT_PARALLEL_BEAM, "PB2D"), (G.TRTT_FAN_BEAM, "FB2D")])
@pytest.mark.parametrize("model", ["cubic", "table"])
def test_sparse_system_products(oracle_port, mode, name, model):
    """Precomputed-matrix mode: H assembled on the GPU, sorted into
    compressed rows, H x and H^T y by trtt_b200_csr_spmv in FP64 against the
    FP64 oracle projector; accumulate adds onto the output."""
    import torch
    from yoricktrtt_b200.recon import Projector2D
    sc = _scan2d(mode, nx=20, ny=16, nv=40, views=5)
    table = TABLE if model == "table" else None
    S = Projector2D(sc, table).sparse_system(max_cells=32)
    rng = np.random.default_rng(9)
    img = _img(sc, seed=4)
    y = rng.random((sc.nviews, sc.nv))
    f = S.forward(torch.tensor(img, dtype=torch.float64, device="cuda"))
    b = S.backward(torch.tensor(y, dtype=torch.float64, device="cuda"))
    S.status()
    f, b = f.cpu().numpy(), b.cpu().numpy()
    ref_b = np.zeros((sc.ny, sc.nx))
    for v in range(sc.nviews):
        ref = np.zeros(sc.nv)
        assert oracle_port.p2d(name, ref, img, sc, v, 0, table) == 0
        assert np.abs(f[v] - ref).max() <= 1e-12 * np.abs(ref).max()
        oracle_port.p2d(name, ref_b, np.ascontiguousarray(y[v]), sc, v, 1, table)
    assert np.abs(b - ref_b).max() <= 1e-12 * np.abs(ref_b).max()
    pre = torch.full((sc.nviews, sc.nv), 0.25, dtype=torch.float64, device="cuda")
    S.forward(torch.tensor(img, dtype=torch.float64, device="cuda"), out=pre, accumulate=True)
    assert np.abs(pre.cpu().numpy() - 0.25 - f).max() <= 1e-14 * np.abs(f).max()


def test_sparse_product_bad_index_flag():
    """A column index outside the matrix is skipped and reported by
    trtt_b200_csr_status (no out-of-range read)."""
    import torch
    from yoricktrtt_b200.recon import _ptr, _stream
    lib = _lib.load()
    rp = torch.tensor([0, 2, 3], dtype=torch.int64, device="cuda")
    col = torch.tensor([0, 5, 1], dtype=torch.int64, device="cuda")   # 5 >= ncols = 2
    val = torch.tensor([1.0, 7.0, 2.0], dtype=torch.float64, device="cuda")
    x = torch.tensor([3.0, 4.0], dtype=torch.float64, device="cuda")
    y = torch.zeros(2, dtype=torch.float64, device="cuda")
    _lib.check(lib.trtt_b200_csr_spmv(_ptr(rp), _ptr(col), _ptr(val), 2, 2, _ptr(x), _ptr(y), 0,
                                      _stream()), "csr_spmv")
    assert lib.trtt_b200_csr_status(_stream()) == -1
    assert y.tolist() == [3.0, 8.0]
    assert lib.trtt_b200_csr_status(_stream()) == 0


def _lf_params(nx=40, ny=36, nd=120, vs=2.0, ps=1.0, sd=300.0, dd=150.0, off=(0.0, 0.0)):
    from oracle.oracle import LF2DParams as OP
    kw = dict(pixelSize=ps, pixelStep=ps, voxelSize=vs, sourceDistance=sd,
              detectorDistance=dd, objectOffset1=off[0], objectOffset2=off[1],
              objectDimension1=nx, objectDimension2=ny, detectorDimension=nd)
    return OP(**kw), dropin.LF2DParams(**kw)


@pytest.mark.parametrize("name", ["direct", "line_integ_direct", "adjoint", "line_integ_adjoint"])
@pytest.mark.parametrize("clr", [0, 1])
@pytest.mark.parametrize("off", [(0.0, 0.0), (3.5, -2.0)])
def test_lf2d(oracle_port, name, clr, off):
    op, dp = _lf_params(off=off)
    rng = np.random.default_rng(5)
    direct = "direct" in name
    for beta in (-math.pi / 2, 0.3, 2.0):
        for doff in (0.0, 4.25):
            if direct:
                src = np.ascontiguousarray(P.ellipses_2d(36, 40, n=5, seed=2))  # [i2][i1]
                dst0 = rng.random(120)
            else:
                src = rng.random(120)
                dst0 = rng.random((36, 40))
            ref, got = dst0.copy(), dst0.copy()
            oracle_port.lf2d(name, op, beta, doff, src, ref, clr)
            dropin.lf2d(name, dp, beta, doff, src, got, clr)
            base = 0.0 if clr else dst0
            assert rel_l2(got - base, ref - base) <= TOL, (name, beta, doff)


@pytest.mark.parametrize("name", ["sparser", "line_integ_sparser"])
def test_lf2d_sparsers(oracle_port, name):
    op, dp = _lf_params()
    for (i1, i2) in [(0, 0), (13, 7), (39, 35)]:
        for clr in (0, 1):
            pre = np.random.default_rng(i1 + i2).random(120)
            ref, got = pre.copy(), pre.copy()
            oracle_port.lf2d_sparser(name, op, 0.7, 1.5, i1, i2, ref, clr)
            dropin.lf2d_sparser(name, dp, 0.7, 1.5, i1, i2, got, clr)
            assert np.allclose(got, ref, rtol=1e-12, atol=1e-14)


def test_lf_plan_and_adjoint(oracle_port):
    import torch
    op, dp = _lf_params()
    nviews = 6
    beta = np.linspace(0, 2 * math.pi, nviews, endpoint=False) - math.pi / 2
    offs = np.full(nviews, 0.5)
    lib = _lib.load()
    h = C.c_void_p()
    _lib.check(lib.trtt_b200_plan2d_create_lf(C.byref(h), C.addressof(dp), 0, nviews,
                                              _lib.dptr(beta), _lib.dptr(offs)), "create_lf")
    img = np.ascontiguousarray(P.ellipses_2d(36, 40, n=5, seed=4))
    x = torch.tensor(img, dtype=torch.float32, device="cuda")
    y = torch.zeros(nviews, 120, dtype=torch.float32, device="cuda")
    _lib.check(lib.trtt_b200_plan2d_forward(h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None), "fwd")
    r = torch.rand(nviews, 120, dtype=torch.float32, device="cuda")
    b = torch.zeros_like(x)
    _lib.check(lib.trtt_b200_plan2d_backward(h, C.c_void_p(r.data_ptr()), C.c_void_p(b.data_ptr()), None), "back")
    torch.cuda.synchronize()
    yh = y.double().cpu().numpy()
    for v in range(nviews):
        ref = np.zeros(120)
        oracle_port.lf2d("direct", op, beta[v], offs[v], img, ref, 1)
        assert rel_l2(yh[v], ref) <= TOL
    lhs = float((y.double() * r.double()).sum())
    rhs = float((x.double() * b.double()).sum())
    assert abs(lhs - rhs) / (float(y.double().norm()) * float(r.double().norm())) <= 1e-6
    lib.trtt_b200_plan2d_destroy(h)


@pytest.mark.parametrize("mode,model", [(G.TRTT_FAN_BEAM, "cubic"), (G.TRTT_FAN_BEAM, "table"),
                                        (G.TRTT_PARALLEL_BEAM, "cubic")])
def test_plan2d_matches_oracle_and_adjoint(oracle_port, mode, model):
    import torch
    sc = _scan2d(mode, views=9)
    table = TABLE if model == "table" else None
    lib = _lib.load()
    h = C.c_void_p()
    geom = 5 if mode == G.TRTT_FAN_BEAM else 3
    cum = _lib.dptr(table.cum) if table else None
    coord = _lib.dptr(table.coord) if table else None
    _lib.check(lib.trtt_b200_plan2d_create(C.byref(h), geom, sc.nx, sc.ny, sc.s_scl, sc.s_deg, cum,
                                           table.size if table else 0, table.step if table else 1.0,
                                           coord, sc.nv, sc.v_scl, sc.nviews,
                                           _lib.dptr(np.ascontiguousarray(sc.xos)),
                                           _lib.dptr(np.ascontiguousarray(sc.xsd))), "create")
    img = _img(sc, seed=6)
    x = torch.tensor(img, dtype=torch.float32, device="cuda")
    y = torch.zeros(sc.nviews, sc.nv, dtype=torch.float32, device="cuda")
    _lib.check(lib.trtt_b200_plan2d_forward(h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), None), "fwd")
    r = torch.rand(sc.nviews, sc.nv, dtype=torch.float32, device="cuda")
    b = torch.zeros_like(x)
    _lib.check(lib.trtt_b200_plan2d_backward(h, C.c_void_p(r.data_ptr()), C.c_void_p(b.data_ptr()), None), "back")
    _lib.check(lib.trtt_b200_plan2d_status(h, None), "status")
    name = "FB2D" if mode == G.TRTT_FAN_BEAM else "PB2D"
    yh = y.double().cpu().numpy()
    rb = np.zeros_like(img)
    rh = r.double().cpu().numpy()
    for v in range(sc.nviews):
        ref = np.zeros(sc.nv)
        oracle_port.p2d(name, ref, img, sc, v, 0, table)
        assert rel_l2(yh[v], ref) <= TOL
        oracle_port.p2d(name, rb, np.ascontiguousarray(rh[v]), sc, v, 1, table)
    assert rel_l2(b.double().cpu().numpy(), rb) <= TOL
    lhs = float((y.double() * r.double()).sum())
    rhs = float((x.double() * b.double()).sum())
    assert abs(lhs - rhs) / (float(y.double().norm()) * float(r.double().norm())) <= 1e-6
    lib.trtt_b200_plan2d_destroy(h)


@pytest.mark.parametrize("vs", [1.0, 0.4])   # 0.4 < voxel size: full cells in v
@pytest.mark.parametrize("job", [0, 1])
def test_dd_pb3d(oracle_port, vs, job):
    sc = G.circular_scan_3d(20, 18, 12, 1.0, 3, 40, 44, vs, vs, 4, mode=G.TRTT_PARALLEL_BEAM)
    vol = np.ascontiguousarray(P.ellipsoids_3d(20, 18, 12, n=6, seed=2, dtype=np.float64))
    rng = np.random.default_rng(1)
    for v in range(sc.nviews):
        if job == 0:
            x, shape = vol, (sc.nv, sc.nu)
        else:
            x, shape = rng.random((sc.nv, sc.nu)), vol.shape
        pre = rng.random(shape)
        ref, got = pre.copy(), pre.copy()
        assert oracle_port.dd_pb3d(ref, x, sc, v, job) == 0
        dropin.dd_pb3d(got, x, sc, v, job)
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_mvmult(oracle_port):
    rng = np.random.default_rng(0)
    nnz, nout, nin = 5000, 300, 400
    a = rng.standard_normal(nnz)
    i = rng.integers(1, nout + 1, nnz).astype(np.int64)
    j = rng.integers(1, nin + 1, nnz).astype(np.int64)
    vec = rng.standard_normal(nin)
    pre = rng.standard_normal(nout)
    ref, got = pre.copy(), pre.copy()
    oracle_port.mvmult(ref, vec, a, i, j)
    # extents of the call are max(i), max(j): pass arrays of exactly that size
    dropin.mvmult(got, vec, a, i, j)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)
    # transpose = swapped index arrays (Tomography_2D/Ytrtt2D_optim.i:48-60)
    pre_t = rng.standard_normal(nin)
    ref, got = pre_t.copy(), pre_t.copy()
    oracle_port.mvmult(ref, pre, a, j, i)
    dropin.mvmult(got, pre, a, j, i)
    assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)
    bad = i.copy()
    bad[7] = 0
    with pytest.raises(_lib.TrttError, match="below 1"):
        dropin.mvmult(np.zeros(nout), vec, a, bad, j)


def test_source_line_failure_2d(oracle_port):
    # pixel (5, *) on the source line: wk = i - 5
    xos = np.array([1.0, 0, 0, -5.0, 0, 1.0, 0, 0, 0, 0, 1.0, 0])
    xsd = np.array([1.0, 0, 0, -10.0, 0, 1.0, 0, 20.0, 0, 0, 1.0, 0.5])
    sc = G.Scan2D(12, 10, 1.0, 3, 40, 1.0, G.TRTT_FAN_BEAM, xos[None], xsd[None])
    img = np.ones((10, 12))
    ref = np.zeros(40)
    assert oracle_port.p2d("FB2D", ref, img, sc, 0, 0, None) == -1
    out = np.full(40, 2.0)
    with pytest.raises(_lib.TrttError, match="source line"):
        dropin.p2d("FB2D", out, img, sc, 0, 0, None)
    assert np.all(out == 2.0)
