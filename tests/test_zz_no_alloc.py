"""The allocation-free cone-beam entry point (for callers that cannot call
cudaMalloc: stream capture, allocation-free real-time hosts, pool-owned
memory) against the plan entry point that allocates its geometry table.

Collected last on purpose (file name): if it fails, a run that stops at the
first failure has already run every other test.  It passes alone in a fresh
process and after the other tests.  Two calls in a row with different
geometries check that the shared static scratch array is rewritten, not
stale, between calls."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5  # the parity bound used for every FP32 projection test


def _call(lib, vol_cols, sino, sc, xos, xsd):
    from yoricktrtt_b200 import _lib
    return lib.trtt_b200_cb3d_cubic_forward_noalloc(
        C.c_void_p(vol_cols.data_ptr()), C.c_void_p(sino.data_ptr()), sc.nx, sc.ny, sc.nz,
        sc.s_scl, sc.s_deg, sc.nu, sc.nv, sc.u_scl, sc.v_scl, xos.shape[0], _lib.dptr(xos),
        _lib.dptr(xsd), None)


def test_noalloc_matches_plan_two_calls():
    import torch
    from yoricktrtt_b200 import _lib, geometry as G, phantoms as P
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz
    lib = _lib.load()
    scans = [
        G.circular_scan_3d(40, 36, 32, 1.0, 3, 64, 60, 1.0, 1.0, 12, rsc=120.0, rsd=180.0),
        G.circular_scan_3d(40, 36, 32, 1.0, 3, 64, 60, 1.0, 1.0, 7, rsc=150.0, rsd=200.0,
                           theta=np.linspace(0.3, 5.0, 7), u_off=2.0),
    ]
    for n, sc in enumerate(scans):
        vol = torch.tensor(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=8, seed=40 + n),
                           dtype=torch.float32, device="cuda")
        cols = columns_from_xyz(vol)
        ref = Projector3D(sc).forward(cols, layout="columns")
        got = torch.zeros_like(ref)
        xos = np.ascontiguousarray(sc.xos)
        xsd = np.ascontiguousarray(sc.xsd)
        rc = _call(lib, cols, got, sc, xos, xsd)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert rel_l2(got.double().cpu().numpy(), ref.double().cpu().numpy()) <= TOL, n


def test_noalloc_rejects_too_many_views():
    import torch
    from yoricktrtt_b200 import _lib, geometry as G
    lib = _lib.load()
    limit = 2048
    sc = G.circular_scan_3d(8, 8, 8, 1.0, 3, 16, 16, 1.0, 1.0, limit + 1)
    cols = torch.zeros(8, 8, 8, device="cuda")
    sino = torch.zeros(1, device="cuda")
    rc = _call(lib, cols, sino, sc, np.ascontiguousarray(sc.xos), np.ascontiguousarray(sc.xsd))
    assert rc == -1
    assert "at most 2048 views" in _lib.last_error()
