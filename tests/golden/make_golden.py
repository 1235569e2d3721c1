"""Generate tests/golden/trtt_golden.npz from the reference plugin C.

The reference routines are compiled from their own sources into
oracle/_ref/liboracle_ref.so (``make -C oracle ref``) and evaluated on
small seeded inputs; the inputs, geometries and FP64 outputs are stored so
that the oracle restatement and the B200 kernels can be checked where the
reference tree is absent.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from yoricktrtt_b200 import footprint as F, geometry as G, phantoms as P  # noqa: E402


def main(out=os.path.join(HERE, "trtt_golden.npz")):
    oracle.build(ref=True)
    ref = oracle.get("ref")
    g = {}
    tab = F.make_footprint(3, 2001)
    g["table_cum"], g["table_coord"], g["table_step"] = tab.cum, tab.coord, np.array(tab.step)
    rng = np.random.default_rng(20261203)

    # 3D cone and parallel beam, cubic and table, direct and transpose
    for mode, name in ((G.TRTT_CONE_BEAM, "CB3D"), (G.TRTT_PARALLEL_BEAM, "PB3D")):
        sc = G.circular_scan_3d(16, 14, 12, 1.0, 3, 26, 22, 1.0, 1.0, 3, mode=mode,
                                rsc=50.0, rsd=80.0, u_off=1.5)
        vol = np.ascontiguousarray(P.ellipsoids_3d(16, 14, 12, n=5, seed=11, dtype=np.float64))
        det = rng.random((22, 26))
        g[f"{name}_xos"], g[f"{name}_xsd"] = sc.xos, sc.xsd
        g[f"{name}_vol"], g[f"{name}_det"] = vol, det
        for model, t in (("cubic", None), ("table", tab)):
            fwd = np.zeros((sc.nviews, 22, 26))
            back = np.zeros((sc.nviews,) + vol.shape)
            for v in range(sc.nviews):
                assert ref._p3d(name, fwd[v], vol, sc, v, 0, t) == 0
                assert ref._p3d(name, back[v], det, sc, v, 1, t) == 0
            g[f"{name}_{model}_fwd"], g[f"{name}_{model}_back"] = fwd, back

    # DD parallel beam with full cells in v (exercises the transpose fill)
    sc = G.circular_scan_3d(12, 10, 8, 1.0, 3, 24, 26, 0.4, 0.4, 2, mode=G.TRTT_PARALLEL_BEAM)
    vol = np.ascontiguousarray(P.ellipsoids_3d(12, 10, 8, n=4, seed=12, dtype=np.float64))
    det = rng.random((26, 24))
    g["DD_xos"], g["DD_xsd"], g["DD_vol"], g["DD_det"] = sc.xos, sc.xsd, vol, det
    fwd = np.zeros((2, 26, 24))
    back = np.zeros((2,) + vol.shape)
    for v in range(2):
        ref.dd_pb3d(fwd[v], vol, sc, v, 0)
        ref.dd_pb3d(back[v], det, sc, v, 1)
    g["DD_fwd"], g["DD_back"] = fwd, back

    # 2D fan and parallel beam
    for mode, name in ((G.TRTT_FAN_BEAM, "FB2D"), (G.TRTT_PARALLEL_BEAM, "PB2D")):
        sc = G.circular_scan_2d(24, 20, 1.0, 3, 40, 1.0, 4, mode=mode, rsc=80.0, rsd=120.0)
        img = np.ascontiguousarray(P.ellipses_2d(24, 20, n=4, seed=13))
        det = rng.random(40)
        g[f"{name}_xos"], g[f"{name}_xsd"], g[f"{name}_img"], g[f"{name}_det"] = sc.xos, sc.xsd, img, det
        for model, t in (("cubic", None), ("table", tab)):
            fwd = np.zeros((sc.nviews, 40))
            back = np.zeros((sc.nviews,) + img.shape)
            for v in range(sc.nviews):
                assert ref.p2d(name, fwd[v], img, sc, v, 0, t) == 0
                assert ref.p2d(name, back[v], det, sc, v, 1, t) == 0
            g[f"{name}_{model}_fwd"], g[f"{name}_{model}_back"] = fwd, back
        sp = np.zeros((sc.nviews, 3, 40))
        for v in range(sc.nviews):
            for s, (i, j) in enumerate([(0, 0), (11, 9), (23, 19)]):
                ref.sparser2d(name, sp[v, s], i, j, sc, v, tab)
        g[f"{name}_sparser"] = sp

    # Long-Fessler
    lfp = dict(pixelSize=1.0, pixelStep=1.0, voxelSize=2.0, sourceDistance=200.0,
               detectorDistance=100.0, objectOffset1=0.5, objectOffset2=-1.0,
               objectDimension1=20, objectDimension2=18, detectorDimension=60)
    g["LF_params"] = np.array([lfp[k] for k in ("pixelSize", "pixelStep", "voxelSize", "sourceDistance",
                                                "detectorDistance", "objectOffset1", "objectOffset2",
                                                "objectDimension1", "objectDimension2", "detectorDimension")])
    p = oracle.LF2DParams(**lfp)
    img = np.ascontiguousarray(P.ellipses_2d(18, 20, n=4, seed=14))
    det = rng.random(60)
    betas = np.array([-math.pi / 2, 0.4, 2.5])
    g["LF_img"], g["LF_det"], g["LF_beta"] = img, det, betas
    for name in ("direct", "line_integ_direct", "adjoint", "line_integ_adjoint"):
        src = img if "direct" in name else det
        res = []
        for b in betas:
            dst = np.zeros(60) if "direct" in name else np.zeros((18, 20))
            ref.lf2d(name, p, b, 0.5, src, dst, 1)
            res.append(dst)
        g[f"LF_{name}"] = np.array(res)
    for name in ("sparser", "line_integ_sparser"):
        res = []
        for b in betas:
            dst = np.zeros(60)
            ref.lf2d_sparser(name, p, b, 0.5, 7, 9, dst, 1)
            res.append(dst)
        g[f"LF_{name}"] = np.array(res)

    # COO product
    nnz = 300
    a = rng.standard_normal(nnz)
    i = rng.integers(1, 41, nnz).astype(np.int64)
    j = rng.integers(1, 51, nnz).astype(np.int64)
    vec = rng.standard_normal(50)
    o = np.zeros(40)
    ref.mvmult(o, vec, a, i, j)
    g["MV_a"], g["MV_i"], g["MV_j"], g["MV_vec"], g["MV_out"] = a, i, j, vec, o

    np.savez_compressed(out, **g)
    print(f"wrote {out} ({os.path.getsize(out)} bytes, {len(g)} arrays)")


if __name__ == "__main__":
    main()
