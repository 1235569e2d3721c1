"""Operand layout and arithmetic of the tensor-core band kernel of the direct
3D projector, checked on the CPU (no GPU) with the library's own plans
(trtt_b200_fwd3d_tc_plan_info).

Layout (K-major, no swizzle): the 16-byte K chunk of row m (a detector cell
of the A operand, a band row of B) and column c of a group sits at
(m/8) SBO + c 128 + (m%8) 16, LBO = 128, SBO = columns per group x 128; the
MMA of K-step t (columns 2t, 2t+1) reads element (m, k) at
start + 2t 128 + (m/8) SBO + (m%8) 16 + (k/4) LBO + (k%4) 4.

* Every producer store and every byte an MMA descriptor reads lies inside
  the group's operand, the groups and the profiles fit the dynamic shared
  memory, two CTAs fit on an SM when the ring has two groups, and the TMEM
  accumulator (chunks x rows FP32 columns) fits the allocation.
* A warp's store of one column (32 consecutive rows, 16 bytes each) covers
  whole 128-byte lines (no bank conflicts).
* An emulation of the stores and of the MMA reads with the TF32 split
  (x_hi = TF32(x), x_lo = TF32(x - x_hi); A chunk (P_hi, P_lo, P_hi, P_lo),
  B chunk (w_hi, w_hi, w_lo, w_lo)) reproduces sum_c P_c(u) w_c(r) to ~1e-7
  of FP64, where a single TF32 product would be off by ~1e-4.
"""
import ctypes as C

import numpy as np
import pytest

SMEM_SM = 233472
LBO = 128
WIDTHS = [40, 128, 256, 300, 512, 640, 1000, 1024, 1536]


def _plan(nu):
    from yoricktrtt_b200 import _lib
    info = np.zeros(10, dtype=np.int64)
    rc = _lib.load().trtt_b200_fwd3d_tc_plan_info(nu, info.ctypes.data_as(C.POINTER(C.c_long)))
    return rc, dict(zip(["rows", "nuc", "ng", "tmem", "a", "b", "prof", "smem", "prod", "G"],
                        info.tolist()))


def _chunk(m, c, sbo):
    return (m // 8) * sbo + c * 128 + (m % 8) * 16


def _read(start, m, k, sbo):
    return start + (m // 8) * sbo + (m % 8) * 16 + (k // 4) * LBO + (k % 4) * 4


def tf32(x):
    """Round-to-nearest (ties away) to 10 explicit mantissa bits."""
    b = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x1000) & 0xFFFFE000).astype(np.uint32)
    return r.view(np.float32)


@pytest.mark.parametrize("nu", WIDTHS)
def test_plan_bounds(nu):
    rc, t = _plan(nu)
    assert rc == 0
    rows, nuc, ng, G = t["rows"], t["nuc"], t["ng"], t["G"]
    sbo = G * 128
    assert G % 2 == 0 and nuc * 128 >= nu and rows % 16 == 0 and 16 <= rows <= 64
    assert t["tmem"] >= nuc * rows and t["tmem"] <= 256 and t["tmem"] & (t["tmem"] - 1) == 0
    assert t["a"] == nuc * 128 * G * 16 and t["b"] == rows * G * 16
    # producer stores (16 bytes) stay inside the operand, without overlaps
    u = np.arange(nuc * 128)[:, None]
    c = np.arange(G)[None, :]
    st = _chunk(u, c, sbo)
    assert st.min() >= 0 and st.max() + 16 <= t["a"] and len(np.unique(st)) == st.size
    r = np.arange(rows)[:, None]
    stb = _chunk(r, c, sbo)
    assert stb.max() + 16 <= t["b"] and len(np.unique(stb)) == stb.size
    # one warp-wide store of a column covers 4 whole 128-byte lines
    for cc in range(G):
        lines = _chunk(np.arange(32), cc, sbo) // 128
        assert len(set(lines.tolist())) == 4
        assert sorted((_chunk(np.arange(32), cc, sbo) % 128).tolist()) == sorted(list(range(0, 128, 16)) * 4)
    # descriptor reads: M = 128 rows of chunk uc (N = rows for B), K = 8 per step
    m = np.arange(128)[:, None]
    k = np.arange(8)[None, :]
    for t_ in range(G // 2):
        for uc in range(nuc):
            start = uc * 16 * sbo + t_ * 2 * LBO
            rd = _read(start, m, k, sbo)
            assert rd.min() >= 0 and rd.max() + 4 <= t["a"]
        rdb = _read(t_ * 2 * LBO, r, k, sbo)
        assert rdb.max() + 4 <= t["b"]
    need = ng * (t["a"] + t["b"]) + 4 * t["prod"] * t["prof"]
    assert t["smem"] == need and t["prof"] >= nu and t["prof"] % 4 == 0
    assert t["smem"] + 2048 <= SMEM_SM
    if ng == 2:
        assert 2 * (t["smem"] + 2048) <= SMEM_SM


def test_too_wide():
    assert _plan(2048)[0] == -1 and _plan(4096)[0] == -1


@pytest.mark.parametrize("nu", [40, 300, 512])
def test_emulated_band_product(nu):
    """Stores, descriptor reads and the split TF32 products reproduce the
    band sum_c w_c(r) P_c(u) of one group of columns."""
    rc, t = _plan(nu)
    rows, nuc, G = t["rows"], t["nuc"], t["G"]
    sbo = G * 128
    rng = np.random.default_rng(nu)
    P = np.zeros((G, nuc * 128), np.float32)
    P[:, :nu] = (rng.random((G, nu)) * rng.choice([1e-3, 1.0, 30.0], size=(G, 1))).astype(np.float32)
    W = rng.random((G, rows)).astype(np.float32)
    W[:, rows // 2:] = 0.0
    A = np.full(t["a"] // 4, np.nan, np.float32)
    B = np.full(t["b"] // 4, np.nan, np.float32)
    for c in range(G):
        h = tf32(P[c])
        l_ = tf32(P[c] - h)
        o = _chunk(np.arange(nuc * 128), c, sbo) // 4
        A[o], A[o + 1], A[o + 2], A[o + 3] = h, l_, h, l_
        h = tf32(W[c])
        l_ = tf32(W[c] - h)
        o = _chunk(np.arange(rows), c, sbo) // 4
        B[o], B[o + 1], B[o + 2], B[o + 3] = h, h, l_, l_
    k = np.arange(8)[None, :]
    D = np.zeros((nuc * 128, rows))
    for uc in range(nuc):
        for t_ in range(G // 2):
            a = A[_read(uc * 16 * sbo + t_ * 2 * LBO, np.arange(128)[:, None], k, sbo) // 4].astype(np.float64)
            b = B[_read(t_ * 2 * LBO, np.arange(rows)[:, None], k, sbo) // 4].astype(np.float64)
            assert not np.isnan(a).any() and not np.isnan(b).any()
            D[uc * 128:(uc + 1) * 128] += a @ b.T
    ref = P.astype(np.float64).T @ W.astype(np.float64)
    assert np.abs(D - ref).max() <= 2e-7 * np.abs(ref).max()
    one = tf32(P).astype(np.float64).T @ tf32(W).astype(np.float64)
    assert np.abs(one - ref).max() > 1e-4 * np.abs(ref).max()
