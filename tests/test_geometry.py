"""Host-side geometry and footprint tables against the reference C
(plugin/trtt_xform3d.c compiled into oracle/_ref) and the oracle."""
import ctypes as C
import math

import numpy as np
import pytest

from yoricktrtt_b200 import footprint as F, geometry as G

_dp = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


def test_xform_ops_match_reference(oracle_ref):
    lib = oracle_ref.lib
    for fn in ("trtt_xform3d_move", "trtt_xform3d_scale"):
        getattr(lib, fn).argtypes = [_dp, C.c_double, C.c_double, C.c_double, _dp]
    lib.trtt_xform3d_rotate.argtypes = [_dp, C.c_double, C.c_double, C.c_double, C.c_double, _dp]
    lib.trtt_xform3d_combine.argtypes = [_dp, _dp, _dp]
    lib.trtt_xform3d_invert.argtypes = [_dp, _dp]
    rng = np.random.default_rng(0)
    for _ in range(20):
        a = rng.standard_normal(12)
        x = G.Xform3D(a)
        r = a.copy()
        t = rng.standard_normal(3)
        lib.trtt_xform3d_move(_p(r), *t, _p(r))
        assert np.array_equal(x.move(*t).a, r)
        s = rng.uniform(0.5, 2, 3)
        r = a.copy()
        lib.trtt_xform3d_scale(_p(r), *s, _p(r))
        assert np.array_equal(x.scale(*s).a, r)
        q = rng.standard_normal(4)
        r = a.copy()
        lib.trtt_xform3d_rotate(_p(r), *q, _p(r))
        assert np.allclose(x.rotate(*q).a, r, rtol=1e-15, atol=1e-15)
        b = rng.standard_normal(12)
        r = np.zeros(12)
        lib.trtt_xform3d_combine(_p(r), _p(a), _p(b))
        assert np.allclose(x.combine(G.Xform3D(b)).a, r, rtol=1e-14, atol=1e-14)
        r = np.zeros(12)
        assert lib.trtt_xform3d_invert(_p(r), _p(a)) == 0
        assert np.allclose(x.invert().a, r, rtol=1e-9, atol=1e-9)


def test_circular_orbit_is_factorised():
    """Circular orbits give exact zeros in the z-mixing coefficients that the
    column-factorised kernels test for (o3, o7, den_z, num_v_z)."""
    sc = G.circular_scan_3d(64, 64, 32, 1.0, 3, 128, 128, 1.0, 1.0, 37)
    for xos, xsd in zip(sc.xos, sc.xsd):
        assert xos[2] == 0.0 and xos[6] == 0.0
        assert xsd[1] == 0.0 and xsd[2] == 0.0 and xsd[4] == 0.0 and xsd[6] == 0.0
        a1inv = -1.0 * (1.0 / xsd[0])
        b2 = xsd[6] + a1inv * xsd[4] * xsd[2]
        b1 = xsd[5] + a1inv * xsd[4] * xsd[1]
        assert b1 * xos[6] + b2 * xos[10] == 0.0
        assert xsd[0] * xos[2] + xsd[1] * xos[6] + xsd[2] * xos[10] == 0.0


def test_projection_of_centre():
    """The volume centre projects to the detector centre for every view, and
    the magnification is SDD/SID there."""
    sc = G.circular_scan_3d(33, 33, 17, 1.0, 3, 64, 64, 1.0, 1.0, 8, rsc=1000.0, rsd=1500.0)
    i = j = 16
    k = 8
    for xos, xsd in zip(sc.xos, sc.xsd):
        # object (i,j,k) -> source frame -> detector pixel coordinates
        o = np.array(xos).reshape(3, 4) @ np.array([i, j, k, 1.0])
        m = np.array(xsd).reshape(3, 4)
        # solve m @ [x_d, v, u, 1]' along the ray: detector plane is x = -Rsd
        assert abs(o[1]) < 1e-9 and abs(o[2]) < 1e-9
        assert abs(o[0] - 1000.0) < 1e-9


def test_gate_weights():
    assert G.gate_weights(2.25, 10) == ((2, 3), (0.75, 0.25))
    assert G.gate_weights(9.5, 10) == ((9, 0), (0.5, 0.5))
    assert G.gate_weights(4.0, 10) == ((4, 4), (1.0, 0.0))
    t = G.gate_t_index([0.0, 1.0, 2.5, 4.0], tcycl=4.0, nt=8)
    assert np.allclose(t, [0.0, 2.0, 5.0, 0.0])


@pytest.mark.parametrize("deg", [0, 1, 2, 3, 4, 7])
def test_footprint_table_matches_oracle(oracle_port, deg):
    fp, cum, coord, step = oracle_port.footprint_table(deg, 2001)
    t = F.make_footprint(deg, 2001)
    assert step == t.step
    assert np.array_equal(coord, t.coord)
    assert np.allclose(fp, t.footprint, rtol=1e-13, atol=1e-15)
    assert np.allclose(cum, t.cum, rtol=1e-12, atol=1e-15)
    # unit integral, centred support
    assert abs(t.cum[-1] - 1.0) < 1e-5
    assert t.coord[0] == -(deg + 1)


def test_cubic_table_close_to_closed_form():
    """Table and closed-form cubic primitives agree to the table's own
    resolution (the reference's two footprint models of the same B-spline)."""
    t = F.make_footprint(3, 10001)
    x = t.coord
    prim = np.where(x <= -2, 0.0, np.where(x >= 2, 1.0, 0.0))
    inner = np.abs(x) < 2
    from yoricktrtt_b200.footprint import bspline
    xs = np.linspace(-4, 4, 200001)
    cdf = np.cumsum(bspline(3, xs)) * (xs[1] - xs[0])
    assert np.max(np.abs(np.interp(x, xs, cdf) - t.cum)) < 2e-4
    assert prim is not None and inner.any()
