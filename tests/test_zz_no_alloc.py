"""The allocation-free cone-beam entry point, for callers that cannot call
cudaMalloc (real-time hosts that forbid device allocation after start-up,
frameworks whose device memory belongs to their own pool allocator).

Its output is checked against the FP64 oracle and against the plan entry
point (which allocates its geometry table), within the FP32 parity bound,
on three calls in a row with different geometries: two circular orbits
(column-factorised views, detector-row band kernel) and a tilted orbit
(per-voxel kernel).  Successive calls with different geometries check that
the shared static scratch array is rewritten, not stale, between calls.

Collected last on purpose (file name): if it fails, a run that stops at the
first failure has already run every other test.  It passes alone in a fresh
process and after the other tests."""
import ctypes as C
import math

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


def _tilted(sc, rsc, rsd):
    """Each view's source frame is also tilted about the x axis: the
    transaxial footprint then depends on k, so no view is factorised."""
    from yoricktrtt_b200 import geometry as G
    oxi = G.object_xi(sc.nx, sc.ny, sc.nz, sc.s_scl)
    dxi = G.data_xi(sc.nu, sc.nv, sc.u_scl, sc.v_scl)
    for k, th in enumerate(sc.theta):
        xos, xsd, xot = G.view_xforms(th, rsc, rsd)
        a = 0.12 + 0.04 * k
        xos = xos.rotate(math.cos(a / 2), math.sin(a / 2), 0.0, 0.0)
        sc.xos[k], sc.xsd[k] = G.projector_coefs(oxi, dxi, xos, xsd, xot)
    return sc


def test_noalloc_matches_oracle_and_plan_three_calls(oracle_port):
    import torch
    from yoricktrtt_b200 import _lib, geometry as G, phantoms as P
    from yoricktrtt_b200.projectors import Projector3D, columns_from_xyz
    lib = _lib.load()
    scans = [
        G.circular_scan_3d(40, 36, 32, 1.0, 3, 64, 60, 1.0, 1.0, 12, rsc=120.0, rsd=180.0),
        G.circular_scan_3d(40, 36, 32, 1.0, 3, 64, 60, 1.0, 1.0, 7, rsc=150.0, rsd=200.0,
                           theta=np.linspace(0.3, 5.0, 7), u_off=2.0),
        _tilted(G.circular_scan_3d(40, 36, 32, 1.0, 3, 64, 60, 1.0, 1.0, 5, rsc=130.0,
                                   rsd=190.0), 130.0, 190.0),
    ]
    for n, sc in enumerate(scans):
        vol64 = np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=8, seed=40 + n,
                                                     dtype=np.float64))
        vol = torch.tensor(vol64, dtype=torch.float32, device="cuda")
        cols = columns_from_xyz(vol)
        pr = Projector3D(sc)
        assert pr.factorized == (n < 2)
        plan = pr.forward(cols, layout="columns")
        got = torch.zeros_like(plan)
        xos = np.ascontiguousarray(sc.xos)
        xsd = np.ascontiguousarray(sc.xsd)
        rc = _call(lib, cols, got, sc, xos, xsd)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = got.double().cpu().numpy()
        assert rel_l2(got, plan.double().cpu().numpy()) <= TOL, n
        # FP64 oracle on the FP32-rounded volume the GPU saw
        volr = np.ascontiguousarray(vol.double().cpu().numpy())
        for v in range(sc.nviews):
            ref = np.zeros((sc.nv, sc.nu))
            assert oracle_port.cb3d(ref, volr, sc, v, 0) == 0
            assert rel_l2(got[v], ref) <= TOL, (n, v, rel_l2(got[v], ref))


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
