"""GPU parity of the 3D projector pair against the FP64 oracle.

The B200 kernels are called through the C ABI (the drop-in trtt_PB3D /
trtt_CB3D / *_cubic symbols and the native plan API) on seeded phantoms at
sizes the oracle finishes in well under a second, and compared with the
oracle's FP64 result: relative L2 error <= 1e-5 per projection (the
projectors compute in FP32).  Also checked: accumulate-into-out semantics,
the FP64 adjoint identity <Hx,y> = <x,H^T y>, clipped and empty
footprints, non-circular (per-voxel kernel) geometry, anisotropic
sampling, the failure path (a voxel in the source plane) and the 4D
per-gate projection.
"""
import math

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import dropin, footprint as F, geometry as G, phantoms as P

pytestmark = pytest.mark.gpu

TOL = 1e-5          # relative L2, FP32 kernels vs FP64 oracle
ADJ_TOL = 1e-6      # relative adjoint mismatch of the FP32 pair

TABLE = F.make_footprint(3, 10001)


def _scan(mode, nx=24, ny=20, nz=16, nu=40, nv=36, views=4, s=1.0, us=1.0, vs=1.0,
          rsc=60.0, rsd=90.0, deg=3, **kw):
    return G.circular_scan_3d(nx, ny, nz, s, deg, nu, nv, us, vs, views, mode=mode,
                              rsc=rsc, rsd=rsd, **kw)


def _vol(sc, seed=1):
    return np.ascontiguousarray(
        P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=8, seed=seed, dtype=np.float64))


CASES = [
    ("CB3D", G.TRTT_CONE_BEAM, {}),
    ("PB3D", G.TRTT_PARALLEL_BEAM, {}),
    ("CB3D", G.TRTT_CONE_BEAM, dict(nu=22, nv=18)),             # clipped at edges
    ("CB3D", G.TRTT_CONE_BEAM, dict(us=0.7, vs=1.3, s=0.8)),     # anisotropic
    ("CB3D", G.TRTT_CONE_BEAM, dict(u_off=3.3, v_off=-2.1)),     # detector offsets
    ("PB3D", G.TRTT_PARALLEL_BEAM, dict(nu=22, nv=18, us=0.6, vs=0.6)),
    ("CB3D", G.TRTT_CONE_BEAM, dict(nu=20, nv=18, us=1.8, vs=1.8)),  # coarse cells: non-monotone columns
]


@pytest.mark.parametrize("name,mode,kw", CASES)
@pytest.mark.parametrize("model", ["cubic", "table"])
@pytest.mark.parametrize("job", [0, 1])
def test_dropin_parity(oracle_port, name, mode, kw, model, job):
    sc = _scan(mode, **kw)
    table = TABLE if model == "table" else None
    rng = np.random.default_rng(7)
    vol = _vol(sc)
    for v in range(sc.nviews):
        if job == 0:
            x = vol
            shape = (sc.nv, sc.nu)
        else:
            x = rng.random((sc.nv, sc.nu))
            shape = vol.shape
        pre = rng.random(shape)
        ref = pre.copy()
        got = pre.copy()
        assert oracle_port._p3d(name, ref, x, sc, v, job, table) == 0
        dropin.scan3d_call(name, got, x, sc, v, job, table)
        assert rel_l2(got - pre, ref - pre) <= TOL, (v, rel_l2(got - pre, ref - pre))


@pytest.mark.parametrize("deg", [0, 1, 2, 4])
def test_table_degrees(oracle_port, deg):
    tab = F.make_footprint(deg, 4001)
    sc = _scan(G.TRTT_CONE_BEAM, deg=deg, views=2)
    vol = _vol(sc, seed=3)
    for v in range(2):
        ref = np.zeros((sc.nv, sc.nu))
        got = np.zeros_like(ref)
        oracle_port.cb3d(ref, vol, sc, v, 0, tab)
        dropin.scan3d_call("CB3D", got, vol, sc, v, 0, tab)
        assert rel_l2(got, ref) <= TOL


def _tilted_scan(mode, views=3):
    """Non-circular geometry: each view's source frame is also tilted about
    the x axis, so the transaxial footprint depends on k (per-voxel
    kernels)."""
    sc = _scan(mode, views=views)
    oxi = G.object_xi(sc.nx, sc.ny, sc.nz, sc.s_scl)
    dxi = G.data_xi(sc.nu, sc.nv, sc.u_scl, sc.v_scl)
    for k, th in enumerate(sc.theta):
        par = mode == G.TRTT_PARALLEL_BEAM
        xos, xsd, xot = G.view_xforms(th, None if par else 60.0, None if par else 90.0)
        a = 0.15 + 0.05 * k
        xos = xos.rotate(math.cos(a / 2), math.sin(a / 2), 0.0, 0.0)
        sc.xos[k], sc.xsd[k] = G.projector_coefs(oxi, dxi, xos, xsd, xot)
    return sc


@pytest.mark.parametrize("name,mode", [("CB3D", G.TRTT_CONE_BEAM), ("PB3D", G.TRTT_PARALLEL_BEAM)])
@pytest.mark.parametrize("model", ["cubic", "table"])
def test_general_geometry(oracle_port, name, mode, model):
    sc = _tilted_scan(mode)
    table = TABLE if model == "table" else None
    vol = _vol(sc, seed=5)
    rng = np.random.default_rng(11)
    for v in range(sc.nviews):
        ref = np.zeros((sc.nv, sc.nu))
        got = np.zeros_like(ref)
        oracle_port._p3d(name, ref, vol, sc, v, 0, table)
        dropin.scan3d_call(name, got, vol, sc, v, 0, table)
        assert rel_l2(got, ref) <= TOL
        y = rng.random((sc.nv, sc.nu))
        ref = np.zeros_like(vol)
        got = np.zeros_like(vol)
        oracle_port._p3d(name, ref, y, sc, v, 1, table)
        dropin.scan3d_call(name, got, y, sc, v, 1, table)
        assert rel_l2(got, ref) <= TOL


@pytest.mark.parametrize("mode", [G.TRTT_CONE_BEAM, G.TRTT_PARALLEL_BEAM])
@pytest.mark.parametrize("model", ["cubic", "table"])
def test_adjoint_fp64(mode, model):
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    sc = _scan(mode, nx=40, ny=36, nz=32, nu=64, nv=60, views=6)
    table = TABLE if model == "table" else None
    pr = Projector3D(sc, table)
    rng = np.random.default_rng(2)
    x = torch.tensor(rng.random((sc.nz, sc.ny, sc.nx)), dtype=torch.float32, device="cuda")
    y = torch.tensor(rng.random((sc.nviews, sc.nv, sc.nu)), dtype=torch.float32, device="cuda")
    hx = pr.forward(x).double().cpu().numpy()
    hty = pr.backward(y).double().cpu().numpy()
    lhs = float(np.sum(hx * y.double().cpu().numpy()))
    rhs = float(np.sum(x.double().cpu().numpy() * hty))
    assert abs(lhs - rhs) / (np.linalg.norm(hx) * np.linalg.norm(y.cpu().numpy())) <= ADJ_TOL


@pytest.mark.parametrize("model", ["cubic", "table"])
@pytest.mark.parametrize("layout", ["xyz", "columns"])
def test_plan_matches_oracle(oracle_port, model, layout):
    import torch
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz, xyz_from_columns
    sc = _scan(G.TRTT_CONE_BEAM, views=5)
    table = TABLE if model == "table" else None
    vol = _vol(sc, seed=9)
    pr = Projector3D(sc, table)
    assert pr.factorized
    xt = torch.tensor(vol, dtype=torch.float32, device="cuda")
    if layout == "columns":
        xt = columns_from_xyz(xt)
    det = pr.forward(xt, layout=layout).double().cpu().numpy()
    rng = np.random.default_rng(4)
    y = rng.random((sc.nviews, sc.nv, sc.nu))
    back = pr.backward(torch.tensor(y, dtype=torch.float32, device="cuda"), layout=layout)
    if layout == "columns":
        back = xyz_from_columns(back)
    back = back.double().cpu().numpy()
    ref_back = np.zeros_like(vol)
    for v in range(sc.nviews):
        ref = np.zeros((sc.nv, sc.nu))
        oracle_port._p3d("CB3D", ref, vol, sc, v, 0, table)
        assert rel_l2(det[v], ref) <= TOL
        oracle_port._p3d("CB3D", ref_back, np.ascontiguousarray(y[v]), sc, v, 1, table)
    assert rel_l2(back, ref_back) <= TOL


def test_view_subrange_and_tiles(oracle_port):
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    sc = _scan(G.TRTT_CONE_BEAM, views=7)
    vol = _vol(sc, seed=12)
    pr = Projector3D(sc)
    xt = torch.tensor(vol, dtype=torch.float32, device="cuda")
    full = pr.forward(xt).cpu().numpy()
    for tiles in [(4, 2), (7, 4), (36, 16), (-1, 0), (-2, 0), (0, 0), (4, 2, 2), (7, 4, 2), (36, 16, 2),
                  (0, 0, 2)]:
        pr.set_tiles(*tiles)
        part = pr.forward(xt, view0=2, nview=3).cpu().numpy()
        assert rel_l2(part, full[2:5]) <= 1e-6, tiles
    pr.set_tiles(0, 0, 2)
    ref_f = np.zeros((sc.nviews, sc.nv, sc.nu))
    for v in range(sc.nviews):
        oracle_port.cb3d(ref_f[v], vol, sc, v, 0)
    assert rel_l2(pr.forward(xt).double().cpu().numpy(), ref_f) <= TOL
    pr.set_tiles(0, 0)
    y = torch.rand(sc.nviews, sc.nv, sc.nu, device="cuda")
    a = pr.backward(y[2:5], view0=2, nview=3).double().cpu().numpy()
    ref = np.zeros_like(vol)
    for v in range(2, 5):
        oracle_port.cb3d(ref, np.ascontiguousarray(y[v].double().cpu().numpy()), sc, v, 1)
    assert rel_l2(a, ref) <= TOL


@pytest.mark.parametrize("model", ["cubic", "table"])
@pytest.mark.parametrize("off", [(400.0, -300.0), (-30.0, 12.0)])
def test_empty_and_offdetector(oracle_port, model, off):
    # detector shifted far away: every footprint is clipped to nothing or
    # to the last cells, exactly as the reference clamps; shifted by part of
    # its width: many footprints start left of the first cell (clamped)
    sc = _scan(G.TRTT_CONE_BEAM, views=2, u_off=off[0], v_off=off[1])
    table = TABLE if model == "table" else None
    vol = _vol(sc)
    for v in range(2):
        ref = np.zeros((sc.nv, sc.nu))
        got = np.zeros_like(ref)
        assert oracle_port._p3d("CB3D", ref, vol, sc, v, 0, table) == 0
        dropin.scan3d_call("CB3D", got, vol, sc, v, 0, table)
        assert np.allclose(got, ref, rtol=1e-5, atol=1e-9 * max(1.0, np.abs(ref).max()))


def test_source_plane_failure(oracle_port):
    from yoricktrtt_b200 import _lib
    nx, ny, nz, nu, nv = 12, 10, 8, 20, 18
    xos = np.array([1.0, 0, 0, -5.0, 0, 1.0, 0, 0, 0, 0, 1.0, 0])
    xsd = np.array([1.0, 0, 0, -10.0, 0, 1.0, 0, 9.0, 0, 0, 1.0, 10.0])
    vol = np.ones((nz, ny, nx))
    ref = np.zeros((nv, nu))
    rc = oracle_port.raw("CB3D_cubic")(
        ref.ctypes.data_as(_lib._dp), vol.ctypes.data_as(_lib._dp), nx, ny, nz, 1.0, 3,
        nu, nv, 1.0, 1.0, xos.ctypes.data_as(_lib._dp), xsd.ctypes.data_as(_lib._dp), 0)
    assert rc == -1
    out = np.full((nv, nu), 3.0)
    with pytest.raises(_lib.TrttError, match="source plane"):
        dropin.p3d("CB3D", out, vol, nx, ny, nz, 1.0, 3, nu, nv, 1.0, 1.0, xos, xsd, 0)
    assert np.all(out == 3.0)  # left unchanged


def test_batch_entry_point(oracle_port):
    from yoricktrtt_b200 import _lib
    sc = _scan(G.TRTT_CONE_BEAM, views=5)
    vol = _vol(sc, seed=21)
    lib = _lib.load()
    out = np.zeros((sc.nviews, sc.nv, sc.nu))
    rc = lib.trtt_b200_cb3d_batch(
        _lib.dptr(out), _lib.dptr(vol), sc.nx, sc.ny, sc.nz, sc.s_scl, sc.s_deg, None, 0,
        1.0, None, sc.nu, sc.nv, sc.u_scl, sc.v_scl, sc.nviews,
        _lib.dptr(np.ascontiguousarray(sc.xos)), _lib.dptr(np.ascontiguousarray(sc.xsd)), 4, 0)
    assert rc == 0, _lib.last_error()
    for v in range(sc.nviews):
        ref = np.zeros((sc.nv, sc.nu))
        oracle_port.cb3d(ref, vol, sc, v, 0)
        assert rel_l2(out[v], ref) <= TOL


def test_batch_entry_point_transpose_chunks(oracle_port):
    """Transpose through the host-buffer batch call: the detector stack is
    uploaded and projected back in view chunks; accumulate onto a non-zero
    output, twice in a row."""
    from yoricktrtt_b200 import _lib
    sc = _scan(G.TRTT_CONE_BEAM, views=13)
    rng = np.random.default_rng(5)
    det = rng.random((sc.nviews, sc.nv, sc.nu))
    lib = _lib.load()
    ref = np.zeros((sc.nz, sc.ny, sc.nx))
    for v in range(sc.nviews):
        oracle_port.cb3d(ref, np.ascontiguousarray(det[v]), sc, v, 1)
    out = np.full((sc.nz, sc.ny, sc.nx), 0.5)
    for call in range(2):
        rc = lib.trtt_b200_cb3d_batch(
            _lib.dptr(out), _lib.dptr(det), sc.nx, sc.ny, sc.nz, sc.s_scl, sc.s_deg, None, 0,
            1.0, None, sc.nu, sc.nv, sc.u_scl, sc.v_scl, sc.nviews,
            _lib.dptr(np.ascontiguousarray(sc.xos)), _lib.dptr(np.ascontiguousarray(sc.xsd)), 4, 1)
        assert rc == 0, _lib.last_error()
        assert rel_l2(out - 0.5, (call + 1) * ref) <= TOL


@pytest.mark.parametrize("tilted", [False, True])
@pytest.mark.parametrize("job", [0, 1])
def test_batch_entry_point_overwrite(oracle_port, tilted, job):
    """trtt_b200_cb3d_batch_ex with accumulate == 0: `out` (filled with NaN
    here) is replaced by the projection, for column-factorised (circular)
    and per-voxel (tilted) views; accumulate == 1 equals the plain call."""
    from yoricktrtt_b200 import _lib
    sc = _tilted_scan(G.TRTT_CONE_BEAM, views=7) if tilted else _scan(G.TRTT_CONE_BEAM, views=7)
    rng = np.random.default_rng(11)
    vol = _vol(sc, seed=3)
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
    call(out, 0)  # again: still replaced, not doubled
    assert rel_l2(out, ref) <= TOL
    call(out, 1)
    assert rel_l2(out, 2 * ref) <= TOL


@pytest.mark.parametrize("model", ["cubic", "table"])
def test_4d_gates(oracle_port, model):
    """Per-gate projection of the 4D path: view k sees
    w0*x[g0] + w1*x[g1] (Ytrtt_3D_projectors.i:301-311, 366-368); the
    transpose adds w_j * H_k^T r into gate j (Tomography_4D/Ytrtt4D_optim.i:196-211)."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    nt = 4
    sc = _scan(G.TRTT_CONE_BEAM, views=7)
    table = TABLE if model == "table" else None
    gates = np.stack([_vol(sc, seed=30 + g) for g in range(nt)])
    t_index = np.array([0.0, 0.4, 1.0, 1.75, 2.5, 3.2, 3.9])
    pr = Projector3D(sc, table)
    pr.set_gates(nt, t_index)
    xt = torch.tensor(gates, dtype=torch.float32, device="cuda")
    det = pr.forward(xt).double().cpu().numpy()
    rng = np.random.default_rng(8)
    y = rng.random((sc.nviews, sc.nv, sc.nu))
    back = pr.backward(torch.tensor(y, dtype=torch.float32, device="cuda")).double().cpu().numpy()
    ref_back = np.zeros_like(gates)
    for k, t in enumerate(t_index):
        (g0, g1), (w0, w1) = G.gate_weights(t, nt)
        bx = np.ascontiguousarray(w0 * gates[g0] + w1 * gates[g1])
        ref = np.zeros((sc.nv, sc.nu))
        oracle_port._p3d("CB3D", ref, bx, sc, k, 0, table)
        assert rel_l2(det[k], ref) <= TOL
        bt = np.zeros_like(gates[0])
        oracle_port._p3d("CB3D", bt, np.ascontiguousarray(y[k]), sc, k, 1, table)
        if g0 != g1:
            ref_back[g0] += w0 * bt
            ref_back[g1] += w1 * bt
        else:
            ref_back[g0] += w1 * bt  # repeated index: the second write wins
    assert rel_l2(back, ref_back) <= TOL


TC_CASES = [
    (G.TRTT_CONE_BEAM, {}),                                    # nu 40: one u chunk, band > nv
    (G.TRTT_PARALLEL_BEAM, {}),
    (G.TRTT_CONE_BEAM, dict(nu=22, nv=18)),                    # clipped footprints
    (G.TRTT_CONE_BEAM, dict(us=0.7, vs=1.3, s=0.8)),           # anisotropic
    (G.TRTT_CONE_BEAM, dict(u_off=3.3, v_off=-2.1)),           # detector offsets
    (G.TRTT_CONE_BEAM, dict(nu=300, nv=140, us=0.15, vs=0.2)), # 3 u chunks, several bands
    (G.TRTT_CONE_BEAM, dict(nu=640, nv=70, us=0.08, vs=0.5)),  # 5 chunks, one-group ring
]


@pytest.mark.parametrize("mode,kw", TC_CASES)
def test_tensor_band_kernel(oracle_port, mode, kw):
    """Direct projector with the band accumulated on the tensor cores
    (set_tiles(-3, 0), TF32 split in three products) against the FP64
    oracle, accumulating onto a non-zero detector; the status flag stays
    clear."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    name = "CB3D" if mode == G.TRTT_CONE_BEAM else "PB3D"
    sc = _scan(mode, views=6, **kw)
    vol = _vol(sc, seed=17)
    pr = Projector3D(sc)
    assert pr.factorized
    pr.set_tiles(-3, 0)
    xt = torch.tensor(vol, dtype=torch.float32, device="cuda")
    pre = torch.rand(sc.nviews, sc.nv, sc.nu, device="cuda")
    det = pr.forward(xt, out=pre.clone())
    pr.status()
    det = (det - pre).double().cpu().numpy()
    for v in range(sc.nviews):
        ref = np.zeros((sc.nv, sc.nu))
        assert oracle_port._p3d(name, ref, vol, sc, v, 0, None) == 0
        assert rel_l2(det[v], ref) <= TOL, (v, rel_l2(det[v], ref))


def test_tensor_band_kernel_gates_and_empty(oracle_port):
    """4D per-gate direct projection and an all-zero volume (no column
    reaches the tensor cores) through the tensor-core band kernel."""
    import torch
    from yoricktrtt_b200.projectors import Projector3D
    nt = 3
    sc = _scan(G.TRTT_CONE_BEAM, views=5)
    gates = np.stack([_vol(sc, seed=40 + g) for g in range(nt)])
    t_index = np.array([0.0, 0.6, 1.5, 2.2, 2.9])
    pr = Projector3D(sc)
    pr.set_gates(nt, t_index)
    pr.set_tiles(-3, 0)
    det = pr.forward(torch.tensor(gates, dtype=torch.float32, device="cuda")).double().cpu().numpy()
    for k, t in enumerate(t_index):
        (g0, g1), (w0, w1) = G.gate_weights(t, nt)
        ref = np.zeros((sc.nv, sc.nu))
        oracle_port.cb3d(ref, np.ascontiguousarray(w0 * gates[g0] + w1 * gates[g1]), sc, k, 0)
        assert rel_l2(det[k], ref) <= TOL
    pr2 = Projector3D(sc)
    pr2.set_tiles(-3, 0)
    zero = torch.zeros(pr2.volume_shape(), device="cuda")
    out = torch.full((sc.nviews, sc.nv, sc.nu), 0.25, device="cuda")
    pr2.forward(zero, out=out)
    pr2.status()
    assert torch.all(out == 0.25)
