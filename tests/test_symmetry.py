"""Orbit symmetry of circular scans (CPU, FP64 oracle).

A view at angle theta + 90 degrees of a circular orbit about the z axis
sees the volume grid turned by a quarter turn: its footprint of voxel
column c is the theta view's footprint of column R(c), R(i, j) =
(n-1-j, i).  The symmetric projector kernels evaluate the footprints of one
view of each group and apply them to all members; these tests pin the
grouping and the column mapping on the reference projector itself."""
import math

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import geometry as G, phantoms as P


def _scan(n=12, nz=6, views=8, mode=G.TRTT_CONE_BEAM, ny=None, **kw):
    return G.circular_scan_3d(n, ny or n, nz, 1.0, 3, 20, 18, 1.0, 1.0, views, mode=mode,
                              rsc=40.0, rsd=60.0, **kw)


def _turned(vol, m):
    """Y with Y[k, R^m(i, j)] = X[k, i, j] in (i, j) column terms, i.e.
    Y[k, j', i'] = X[k, j, i] where (i', j') = R^m(i, j)."""
    nz, ny, nx = vol.shape
    out = np.zeros_like(vol)
    for j in range(ny):
        for i in range(nx):
            i2, j2 = G.turn_columns(i, j, m, nx, ny)
            out[:, j2, i2] = vol[:, j, i]
    return out


def test_groups_of_uniform_orbit():
    sc = _scan(views=8)
    g = G.view_groups(sc)
    assert sorted(len(x) for x in g) == [4, 4]
    assert sorted(sum(g, [])) == list(range(8))
    # 6 views (60 degree steps): half turns only
    g = G.view_groups(_scan(views=6))
    assert sorted(len(x) for x in g) == [2, 2, 2]
    # odd number of views over 2 pi: no symmetric partner
    assert all(len(x) == 1 for x in G.view_groups(_scan(views=5)))
    # odd square grid: no quarter or half turn maps columns onto columns
    assert all(len(x) == 1 for x in G.view_groups(_scan(n=11, views=8)))
    # rectangular even grid: half turns
    g = G.view_groups(_scan(n=12, ny=10, views=8))
    assert sorted(len(x) for x in g) == [2, 2, 2, 2]
    # detector offsets and parallel beam keep the symmetry
    assert sorted(len(x) for x in G.view_groups(_scan(views=8, u_off=1.5, v_off=-2.0))) == [4, 4]
    assert sorted(len(x) for x in G.view_groups(_scan(views=8, mode=G.TRTT_PARALLEL_BEAM))) == [4, 4]


@pytest.mark.parametrize("mode", [G.TRTT_CONE_BEAM, G.TRTT_PARALLEL_BEAM])
@pytest.mark.parametrize("kw", [{}, dict(v_off=-1.3, u_off=0.7), dict(ny=10)])
def test_member_footprints_are_turned_base_footprints(oracle_port, mode, kw):
    """proj_{b_m}(X) equals proj_a(Y) with Y the volume turned so that
    column R^m(c) of Y holds column c of X (the reference's own projector,
    FP64): the relation the symmetric kernels rely on."""
    sc = _scan(views=8, mode=mode, **kw)
    name = "CB3D" if mode == G.TRTT_CONE_BEAM else "PB3D"
    vol = np.ascontiguousarray(P.ellipsoids_3d(sc.nx, sc.ny, sc.nz, n=5, seed=2, dtype=np.float64))
    checked = 0
    for grp in G.view_groups(sc):
        a = grp[0]
        ms = [1, 2, 3] if len(grp) == 4 else [2]
        for b, m in zip(grp[1:], ms):
            ref = np.zeros((sc.nv, sc.nu))
            oracle_port._p3d(name, ref, vol, sc, b, 0, None)
            got = np.zeros_like(ref)
            oracle_port._p3d(name, got, np.ascontiguousarray(_turned(vol, m)), sc, a, 0, None)
            assert rel_l2(got, ref) <= 1e-12, (a, b, m)
            checked += 1
    assert checked >= 4
