"""C-ABI library checks that need no GPU: it loads, exports every symbol
that include/trtt_b200.h declares, and fails loudly (no CPU fallback) when
no CUDA device is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    """Function names declared in include/*.h (declarations end with ';')."""
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = "\n".join(l for l in src.splitlines() if not l.lstrip().startswith("#"))
        src = src.replace('extern "C" {', "").replace("}", ";")
        for stmt in src.split(";"):
            m = re.search(r"([A-Za-z_][A-Za-z0-9_]*)\s*\(", stmt)
            if m and not stmt.strip().startswith("typedef"):
                names.append(m.group(1))
    return sorted(set(names))


def test_header_symbols_exported(lib):
    names = _declared()
    assert len(names) >= 30, names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_reference_symbols_present(lib):
    # every builtin of the reference plugins that the projector path binds
    # (plugin/ywrap.c:231-403, tomography-LongFessler-model/ywrap.c:6-77)
    for n in ["trtt_mvmult", "trtt_PB2D_cubic", "trtt_FB2D_cubic", "trtt_PB2D", "trtt_FB2D",
              "trtt_PB2D_sparser", "trtt_FB2D_sparser", "trtt_PB3D", "trtt_DD_PB3D",
              "trtt_CB3D", "trtt_PB3D_cubic", "trtt_CB3D_cubic", "lf2d_direct",
              "lf2d_line_integ_direct", "lf2d_adjoint", "lf2d_line_integ_adjoint",
              "lf2d_sparser", "lf2d_line_integ_sparser"]:
        assert hasattr(lib, n), n


def test_no_cpu_fallback(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    from yoricktrtt_b200 import _lib, dropin, geometry as G
    sc = G.circular_scan_3d(8, 8, 8, 1.0, 3, 12, 12, 1.0, 1.0, 1)
    out = np.zeros((12, 12))
    with pytest.raises(_lib.TrttError):
        dropin.scan3d_call("CB3D", out, np.ones((8, 8, 8)), sc, 0, 0)
    assert np.all(out == 0.0)
    assert _lib.last_error()


def test_version(lib):
    from yoricktrtt_b200 import _lib
    assert b"sm_100a" in _lib.load().trtt_b200_version()
