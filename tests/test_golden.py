"""Golden vectors produced by the reference plugin C (tests/golden/
make_golden.py, compiled from the reference sources): the oracle
restatement must reproduce them bit-for-bit (CPU), the B200 kernels within
the FP32 parity bound (GPU).  Travels with the repository, so the reference
tree is not needed at test time."""
import math
import os

import numpy as np
import pytest

from conftest import rel_l2

from yoricktrtt_b200 import footprint as F, geometry as G

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "trtt_golden.npz"))
TOL = 1e-5


class _Tab:
    def __init__(self):
        self.cum = GOLD["table_cum"]
        self.coord = GOLD["table_coord"]
        self.step = float(GOLD["table_step"])
        self.footprint = np.zeros_like(self.cum)

    @property
    def size(self):
        return len(self.cum)


TAB = _Tab()


def _scan3d(name):
    mode = G.TRTT_CONE_BEAM if name == "CB3D" else G.TRTT_PARALLEL_BEAM
    return G.Scan3D(16, 14, 12, 1.0, 3, 26, 22, 1.0, 1.0, mode, GOLD[f"{name}_xos"], GOLD[f"{name}_xsd"])


def _scan2d(name):
    mode = G.TRTT_FAN_BEAM if name == "FB2D" else G.TRTT_PARALLEL_BEAM
    return G.Scan2D(24, 20, 1.0, 3, 40, 1.0, mode, GOLD[f"{name}_xos"], GOLD[f"{name}_xsd"])


def _lf(mod):
    p = GOLD["LF_params"]
    return mod.LF2DParams(pixelSize=p[0], pixelStep=p[1], voxelSize=p[2], sourceDistance=p[3],
                          detectorDistance=p[4], objectOffset1=p[5], objectOffset2=p[6],
                          objectDimension1=int(p[7]), objectDimension2=int(p[8]),
                          detectorDimension=int(p[9]))


def _run_all(kind, orc=None):
    """Yield (label, result, expected) for every fixture."""
    from yoricktrtt_b200 import dropin
    from oracle import oracle
    for name in ("CB3D", "PB3D"):
        sc = _scan3d(name)
        vol, det = GOLD[f"{name}_vol"], GOLD[f"{name}_det"]
        for model, t in (("cubic", None), ("table", TAB)):
            for v in range(sc.nviews):
                f = np.zeros((22, 26))
                b = np.zeros_like(vol)
                if kind == "port":
                    orc._p3d(name, f, vol, sc, v, 0, t)
                    orc._p3d(name, b, det, sc, v, 1, t)
                else:
                    dropin.scan3d_call(name, f, vol, sc, v, 0, t)
                    dropin.scan3d_call(name, b, det, sc, v, 1, t)
                yield f"{name}-{model}-fwd{v}", f, GOLD[f"{name}_{model}_fwd"][v]
                yield f"{name}-{model}-back{v}", b, GOLD[f"{name}_{model}_back"][v]
    sc = G.Scan3D(12, 10, 8, 1.0, 3, 24, 26, 0.4, 0.4, G.TRTT_PARALLEL_BEAM, GOLD["DD_xos"], GOLD["DD_xsd"])
    for v in range(2):
        f = np.zeros((26, 24))
        b = np.zeros_like(GOLD["DD_vol"])
        if kind == "port":
            orc.dd_pb3d(f, GOLD["DD_vol"], sc, v, 0)
            orc.dd_pb3d(b, GOLD["DD_det"], sc, v, 1)
        else:
            dropin.dd_pb3d(f, GOLD["DD_vol"], sc, v, 0)
            dropin.dd_pb3d(b, GOLD["DD_det"], sc, v, 1)
        yield f"DD-fwd{v}", f, GOLD["DD_fwd"][v]
        yield f"DD-back{v}", b, GOLD["DD_back"][v]
    for name in ("FB2D", "PB2D"):
        sc = _scan2d(name)
        img, det = GOLD[f"{name}_img"], GOLD[f"{name}_det"]
        for model, t in (("cubic", None), ("table", TAB)):
            for v in range(sc.nviews):
                f = np.zeros(40)
                b = np.zeros_like(img)
                if kind == "port":
                    orc.p2d(name, f, img, sc, v, 0, t)
                    orc.p2d(name, b, det, sc, v, 1, t)
                else:
                    dropin.p2d(name, f, img, sc, v, 0, t)
                    dropin.p2d(name, b, det, sc, v, 1, t)
                yield f"{name}-{model}-fwd{v}", f, GOLD[f"{name}_{model}_fwd"][v]
                yield f"{name}-{model}-back{v}", b, GOLD[f"{name}_{model}_back"][v]
        for v in range(sc.nviews):
            for s, (i, j) in enumerate([(0, 0), (11, 9), (23, 19)]):
                o = np.zeros(40)
                if kind == "port":
                    orc.sparser2d(name, o, i, j, sc, v, TAB)
                else:
                    dropin.sparser2d(name, o, i, j, sc, v, TAB)
                yield f"{name}-sparser{v}-{s}", o, GOLD[f"{name}_sparser"][v, s]
    for name in ("direct", "line_integ_direct", "adjoint", "line_integ_adjoint"):
        src = GOLD["LF_img"] if "direct" in name else GOLD["LF_det"]
        for n, b in enumerate(GOLD["LF_beta"]):
            dst = np.zeros(60) if "direct" in name else np.zeros((18, 20))
            if kind == "port":
                orc.lf2d(name, _lf(oracle), b, 0.5, src, dst, 1)
            else:
                dropin.lf2d(name, _lf(dropin), b, 0.5, src, dst, 1)
            yield f"LF-{name}{n}", dst, GOLD[f"LF_{name}"][n]
    for name in ("sparser", "line_integ_sparser"):
        for n, b in enumerate(GOLD["LF_beta"]):
            dst = np.zeros(60)
            if kind == "port":
                orc.lf2d_sparser(name, _lf(oracle), b, 0.5, 7, 9, dst, 1)
            else:
                dropin.lf2d_sparser(name, _lf(dropin), b, 0.5, 7, 9, dst, 1)
            yield f"LF-{name}{n}", dst, GOLD[f"LF_{name}"][n]
    o = np.zeros(40)
    if kind == "port":
        orc.mvmult(o, GOLD["MV_vec"], GOLD["MV_a"], GOLD["MV_i"], GOLD["MV_j"])
    else:
        dropin.mvmult(o, GOLD["MV_vec"], GOLD["MV_a"], GOLD["MV_i"], GOLD["MV_j"])
    yield "mvmult", o, GOLD["MV_out"]


def test_oracle_reproduces_golden(oracle_port):
    n = 0
    for label, got, exp in _run_all("port", oracle_port):
        assert np.array_equal(got, exp), label
        n += 1
    assert n > 100


@pytest.mark.gpu
def test_b200_matches_golden():
    n = 0
    for label, got, exp in _run_all("b200"):
        if label.startswith(("DD", "mvmult")) or "sparser" in label:
            assert np.allclose(got, exp, rtol=1e-12, atol=1e-13), label  # FP64 paths
        else:
            assert rel_l2(got, exp) <= TOL, (label, rel_l2(got, exp))
        n += 1
    assert n > 100
