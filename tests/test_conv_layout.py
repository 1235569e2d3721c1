"""Staging and descriptor arithmetic of the tensor-core convolutions, checked
on the CPU (no GPU): with the shared-memory plans the library itself uses
(trtt_b200_conv3_plan_info), every cp.async destination and every byte a
tcgen05.mma descriptor reads must lie inside the CTA's allocation, and an
emulation of the staged slabs and of the MMAs (the canonical no-swizzle
layouts: K-major element (r, k) at start + (r/8) SBO + (r%8) 16 + (k/8) LBO +
(k%8) 2; MN-major element (r, k) at start + (r/8) SBO + (r%8) 2 + (k/8) LBO +
(k%8) 16) must reproduce the convolution and its weight gradient."""
import ctypes as C

import numpy as np
import pytest

# (cin, cout) of the U-Net layers (forward), and of their input gradients
NET_FWD = [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (96, 32), (48, 16), (32, 96), (16, 48), (64, 32)]
# (cout, cin) of the weight gradients
NET_WGRAD = [(16, 16), (32, 16), (32, 32), (64, 32), (64, 64), (32, 96), (16, 48)]
SMEM_MAX = 227 * 1024


def _plan(which, cin, cout, nb, d, h, w):
    from yoricktrtt_b200 import _lib
    info = np.zeros(10, dtype=np.int64)
    rc = _lib.load().trtt_b200_conv3_plan_info(which, cin, cout, nb, d, h, w,
                                               info.ctypes.data_as(C.POINTER(C.c_long)))
    assert rc == 0, _lib.last_error()
    return info


def _grid(nb, d, h, w):
    hp, wp = h + 2, w + 2
    plane = hp * wp
    vol = (d + 2) * plane
    return dict(hp=hp, wp=wp, plane=plane, vol=vol, rows=nb * vol)


def _kmajor(start, lbo, sbo, rows):
    r = np.arange(rows)[:, None]
    k = np.arange(16)[None, :]
    return start + (r // 8) * sbo + (r % 8) * 16 + (k // 8) * lbo + (k % 8) * 2


def _mnmajor(start, lbo, sbo, rows):
    r = np.arange(rows)[:, None]
    k = np.arange(16)[None, :]
    return start + (r // 8) * sbo + (r % 8) * 2 + (k // 8) * lbo + (k % 8) * 16


class Smem:
    """Shared memory of one CTA: one value per 2-byte slot, NaN = never written."""

    def __init__(self, nbytes):
        self.nbytes = nbytes
        self.v = np.full(nbytes // 2, np.nan)

    def cp16(self, dst, vals):
        assert dst % 16 == 0 and 0 <= dst and dst + 16 <= self.nbytes, dst
        self.v[dst // 2:dst // 2 + 8] = vals

    def read(self, addr):
        assert addr.min() >= 0 and addr.max() + 2 <= self.nbytes, (addr.min(), addr.max(), self.nbytes)
        return self.v[addr // 2]


def _padded(rng, nb, d, h, w, c):
    g = _grid(nb, d, h, w)
    x = np.zeros((nb, d + 2, h + 2, w + 2, c))
    x[:, 1:-1, 1:-1, 1:-1] = rng.standard_normal((nb, d, h, w, c))
    return x.reshape(g["rows"], c)


def _conv_ref(X, W, nb, d, h, w):
    """out[p][n] = sum_tap X[p + off(tap)] W[n][tap] on the interior."""
    g = _grid(nb, d, h, w)
    Xv = X.reshape(nb, d + 2, h + 2, w + 2, -1)
    out = np.zeros((nb, d + 2, h + 2, w + 2, W.shape[0]))
    for tap in range(27):
        dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        out[:, 1:-1, 1:-1, 1:-1] += Xv[:, 1 + dz:1 + dz + d, 1 + dy:1 + dy + h, 1 + dx:1 + dx + w] @ W[:, tap].T
    return out.reshape(g["rows"], -1)


@pytest.mark.parametrize("cin,cout", NET_FWD)
def test_forward_plan_bounds_at_128(cin, cout):
    """Full-size layers (128^3 and the coarser levels): the slab of every
    stage holds the reads of all 9 taps and both sub-tiles."""
    for n in (128, 64, 32):
        S, rh, cs, stage, nstg, smem, tmem_cols, tiles = _plan(0, cin, cout, 1, n, n, n)[:8]
        g = _grid(1, n, n, n)
        assert smem <= SMEM_MAX and nstg * stage <= smem and tmem_cols >= S * cout
        assert rh == 128 * S + 2 * g["wp"] + 2 and cs >= rh * 16
        # last byte read by the A operand of tap (dy, dx) = (2, 2), sub-tile S-1
        a_end = _kmajor((2 * g["wp"] + 2 + 128 * (S - 1)) * 16, cs, 128, 128).max() + 2
        assert a_end <= 2 * cs
        b_end = _kmajor(2 * cs + 8 * cout * 32, cout * 16, 128, cout).max() + 2
        assert b_end <= 2 * cs + 9 * cout * 32 <= stage
        assert tiles * 128 * S >= g["rows"] - 2 * g["plane"]


@pytest.mark.parametrize("cout,cin", NET_WGRAD)
def test_wgrad_plan_bounds_at_128(cout, cin):
    for n in (128, 64, 32):
        kt, csa, csb, ab, bb, nstg, smem, tmem_cols, chunks, steps = _plan(1, cin, cout, 1, n, n, n)
        g = _grid(1, n, n, n)
        nca, ncb = cout // 8, cin // 8
        assert smem <= SMEM_MAX and tmem_cols >= 3 * cin
        assert (nca - 1) * csa + kt * 16 <= ab and (ncb - 1) * csb + (kt + 2) * 16 <= bb
        for buf in range(nstg):
            a0, b0 = buf * ab, nstg * ab + buf * bb
            ks = kt // 16 - 1
            assert _mnmajor(a0 + ks * 256, 128, csa, 64).max() + 2 <= smem  # M = 64, rows >= cout included
            assert _mnmajor(b0 + (ks * 16 + 2) * 16, 128, csb, cin).max() + 2 <= smem
        total = -(-(g["rows"] - 2 * g["plane"]) // kt)
        assert chunks * steps >= total and (chunks - 1) * steps < total


def test_forward_emulation_reproduces_convolution():
    rng = np.random.default_rng(0)
    nb, d, h, w, c1, c2, n = 2, 2, 3, 6, 16, 16, 32
    cin, G = c1 + c2, (c1 + c2) // 16
    S, rh, cs, stage, nstg, smem, tmem_cols, tiles = _plan(0, cin, n, nb, d, h, w)[:8]
    g = _grid(nb, d, h, w)
    X = np.concatenate([_padded(rng, nb, d, h, w, c1), _padded(rng, nb, d, h, w, c2)], 1)
    W = rng.standard_normal((n, 27, cin))
    # packed weights: [stage = dz*G + gi][t9][c][n][k8] (trtt_b200_conv3_pack, transpose = 0)
    pack = np.zeros((3 * G, 9, 2, n, 8))
    for st in range(3 * G):
        dzi, gi = divmod(st, G)
        for t9 in range(9):
            for c in range(2):
                pack[st, t9, c] = W[:, dzi * 9 + t9, gi * 16 + c * 8:gi * 16 + c * 8 + 8]
    pack = pack.reshape(-1)
    out = np.zeros((g["rows"], n))
    for tile in range(tiles):
        m0 = g["plane"] + tile * 128 * S
        D = np.zeros((S, 128, n))
        for it in range(3 * G):
            sm = Smem(smem)
            buf = it % nstg
            hs = buf * stage
            dz, ch = it // G - 1, (it % G) * 16
            hb = m0 + dz * g["plane"] - g["wp"] - 1
            for e in range(2 * rh):
                r, c = e >> 1, e & 1
                row = hb + r
                ok = 0 <= row < g["rows"]
                sm.cp16(hs + c * cs + r * 16, X[row, ch + c * 8:ch + c * 8 + 8] if ok else np.zeros(8))
            ws = hs + 2 * cs
            for e in range(9 * n * 2):
                src = it * 9 * n * 16 + e * 8
                assert src + 8 <= pack.size
                sm.cp16(ws + e * 16, pack[src:src + 8])
            for t9 in range(9):
                dy, dx = divmod(t9, 3)
                B = sm.read(_kmajor(ws + t9 * n * 32, n * 16, 128, n))
                for s in range(S):
                    A = sm.read(_kmajor(hs + (dy * g["wp"] + dx + 128 * s) * 16, cs, 128, 128))
                    assert not np.isnan(A).any() and not np.isnan(B).any()
                    D[s] += A @ B.T
        for s in range(S):
            for r in range(128):
                p = m0 + 128 * s + r
                if p < g["rows"]:
                    out[p] = D[s, r]
    ref = _conv_ref(X, W, nb, d, h, w)
    inner = np.zeros((nb, d + 2, h + 2, w + 2), bool)
    inner[:, 1:-1, 1:-1, 1:-1] = True
    inner = inner.reshape(-1)
    assert np.abs(out[inner] - ref[inner]).max() <= 1e-12 * np.abs(ref).max()


def test_wgrad_emulation_reproduces_weight_gradient():
    rng = np.random.default_rng(1)
    nb, d, h, w, cout, c1, c2 = 2, 3, 4, 5, 16, 16, 16
    cin = c1 + c2
    kt, csa, csb, ab, bb, nstg, smem, tmem_cols, chunks, steps = _plan(1, cin, cout, nb, d, h, w)
    g = _grid(nb, d, h, w)
    dY = _padded(rng, nb, d, h, w, cout)
    X = np.concatenate([_padded(rng, nb, d, h, w, c1), _padded(rng, nb, d, h, w, c2)], 1)
    nca, ncb = cout // 8, cin // 8
    r0, r1 = g["plane"], g["rows"] - g["plane"]
    dW = np.zeros((cout, 27, cin))
    for gidx in range(9):
        dzi, dyi = divmod(gidx, 3)
        off = (dzi - 1) * g["plane"] + (dyi - 1) * g["wp"]
        for cy in range(chunks):
            qbeg = r0 + cy * steps * kt
            T = 0 if r1 - qbeg <= 0 else min(steps, -(-(r1 - qbeg) // kt))
            acc = np.zeros((3, 64, cin))
            sm = Smem(smem)
            sm.v[:] = 0.0  # rows above cout read whatever lies there; not read back
            for it in range(T):
                buf = it % nstg
                a0, b0 = buf * ab, nstg * ab + buf * bb
                q0 = qbeg + it * kt
                for e in range(kt * nca):
                    r, c = divmod(e, nca)
                    row = q0 + r
                    sm.cp16(a0 + c * csa + r * 16, dY[row, c * 8:c * 8 + 8] if row < r1 else np.zeros(8))
                hb = q0 + off - 1
                for e in range((kt + 2) * ncb):
                    r, c = divmod(e, ncb)
                    row = hb + r
                    ok = 0 <= row < g["rows"]
                    sm.cp16(b0 + c * csb + r * 16, X[row, c * 8:c * 8 + 8] if ok else np.zeros(8))
                for ks in range(kt // 16):
                    A = sm.read(_mnmajor(a0 + ks * 256, 128, csa, 64))
                    for j in range(3):
                        B = sm.read(_mnmajor(b0 + (ks * 16 + j) * 16, 128, csb, cin))
                        acc[j] += A @ B.T
            for j in range(3):
                dW[:, gidx * 3 + j] += acc[j, :cout]
    ref = np.zeros((cout, 27, cin))
    for tap in range(27):
        dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        o = dz * g["plane"] + dy * g["wp"] + dx
        p = np.arange(r0, r1)
        ok = (p + o >= 0) & (p + o < g["rows"])
        ref[:, tap] = dY[p[ok]].T @ X[p[ok] + o]
    assert np.abs(dW - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("cin,cout", NET_FWD)
def test_forward_persistent_plan_bounds_at_128(cin, cout):
    """The persistent TMA forward kernel's plan (tiles of 4 x 128 rows where
    two CTAs still fit on an SM, else 2 x 128): every TMA box (8 channels x
    256 rows, and the tail box) lands 128-byte aligned inside its chunk, the
    stage's transaction bytes fit the stage, the taps' A reads stay in the
    slab, and the two tensor-memory accumulators fit the CTAs per SM."""
    for n in (128, 64, 32):
        S, rh, cs, stage, nstg, smem, tmem_cols, tiles = _plan(2, cin, cout, 1, n, n, n)[:8]
        g = _grid(1, n, n, n)
        assert S in (2, 4) and (S == 2 or cout <= 32)
        if n == 128 and cout <= 32:
            assert S == 4  # the 16- and 32-channel layers at full size
        assert smem <= SMEM_MAX and nstg * stage <= smem
        assert 2 * S * cout <= tmem_cols <= 512
        if S == 4:
            assert 2 * (smem + 2048) <= SMEM_MAX and 2 * tmem_cols <= 512
        assert rh == 128 * S + 2 * g["wp"] + 2 and cs % 128 == 0 and stage % 1024 == 0
        boxes = [(r0, min(256, rh - r0)) for r0 in range(0, rh, 256)]
        assert sum(b for _, b in boxes) == rh
        for c in range(2):
            for r0, b in boxes:
                dst = c * cs + r0 * 16
                assert dst % 128 == 0 and r0 * 16 + b * 16 <= cs
        assert 2 * rh * 16 + 288 * cout <= stage  # the stage's transaction bytes
        a_end = _kmajor((2 * g["wp"] + 2 + 128 * (S - 1)) * 16, cs, 128, 128).max() + 2
        assert a_end <= 2 * cs
        assert tiles * 128 * S >= g["rows"] - 2 * g["plane"]


@pytest.mark.parametrize("cout,cin", NET_WGRAD)
def test_wgrad_tma_plan_bounds_at_128(cout, cin):
    """The TMA weight gradient's plan: chunk strides of whole 128-byte
    lines, every box (8 channels x 128 rows, the 2-row tail of the input
    halo) 128-byte aligned inside its chunk and region, and the MMAs' reads
    inside the allocation."""
    for n in (128, 64, 32):
        kt, csa, csb, ab, bb, nstg, smem, tmem_cols, chunks, steps = _plan(3, cin, cout, 1, n, n, n)
        g = _grid(1, n, n, n)
        nca, ncb = cout // 8, cin // 8
        assert smem <= SMEM_MAX and tmem_cols >= 3 * cin and kt % 128 == 0
        assert csa % 128 == 0 and csb % 128 == 0 and ab % 128 == 0 and bb % 128 == 0
        for buf in range(nstg):
            a0, b0 = buf * ab, nstg * ab + buf * bb
            for c in range(nca):
                for r0 in range(0, kt, 128):
                    dst = a0 + c * csa + r0 * 16
                    assert dst % 128 == 0 and r0 * 16 + 128 * 16 <= csa and dst + 2048 <= a0 + ab
            for c in range(ncb):
                for r0 in range(0, kt, 128):
                    dst = b0 + c * csb + r0 * 16
                    assert dst % 128 == 0 and dst + 2048 <= b0 + bb
                tail = b0 + c * csb + kt * 16
                assert tail % 128 == 0 and kt * 16 + 2 * 16 <= csb and tail + 32 <= b0 + bb
            ks = kt // 16 - 1
            assert _mnmajor(a0 + ks * 256, 128, csa, 64).max() + 2 <= smem
            assert _mnmajor(b0 + (ks * 16 + 2) * 16, 128, csb, cin).max() + 2 <= smem
        total = -(-(g["rows"] - 2 * g["plane"]) // kt)
        assert chunks * steps >= total and (chunks - 1) * steps < total


def test_wgrad_tma_emulation_reproduces_weight_gradient():
    """The TMA staging loads whole boxes: dY rows at or past the end of the
    summed range are the last z border plane (zero by the layout) or lie
    past the tensor (read as zero), and input rows before the first row
    read as zero.  With the TMA plan's layout and those reads the MMAs
    reproduce the weight gradient."""
    rng = np.random.default_rng(2)
    nb, d, h, w, cout, c1, c2 = 2, 3, 4, 5, 16, 16, 16
    cin = c1 + c2
    kt, csa, csb, ab, bb, nstg, smem, tmem_cols, chunks, steps = _plan(3, cin, cout, nb, d, h, w)
    g = _grid(nb, d, h, w)
    dY = _padded(rng, nb, d, h, w, cout)
    X = np.concatenate([_padded(rng, nb, d, h, w, c1), _padded(rng, nb, d, h, w, c2)], 1)
    nca, ncb = cout // 8, cin // 8
    r0, r1 = g["plane"], g["rows"] - g["plane"]

    def box(sm, dst, T, x, y, rows):
        for r in range(rows):
            row = y + r
            ok = 0 <= row < g["rows"]
            sm.cp16(dst + r * 16, T[row, x:x + 8] if ok else np.zeros(8))

    dW = np.zeros((cout, 27, cin))
    for gidx in range(9):
        dzi, dyi = divmod(gidx, 3)
        off = (dzi - 1) * g["plane"] + (dyi - 1) * g["wp"]
        for cy in range(chunks):
            qbeg = r0 + cy * steps * kt
            T = 0 if r1 - qbeg <= 0 else min(steps, -(-(r1 - qbeg) // kt))
            acc = np.zeros((3, 64, cin))
            sm = Smem(smem)
            sm.v[:] = 0.0  # rows above cout read whatever lies there; not read back
            for it in range(T):
                buf = it % nstg
                a0, b0 = buf * ab, nstg * ab + buf * bb
                q0 = qbeg + it * kt
                hb = q0 + off - 1
                for c in range(nca):
                    for rr in range(0, kt, 128):
                        box(sm, a0 + c * csa + rr * 16, dY, 8 * c, q0 + rr, 128)
                for c in range(ncb):
                    for rr in range(0, kt, 128):
                        box(sm, b0 + c * csb + rr * 16, X, 8 * c, hb + rr, 128)
                    box(sm, b0 + c * csb + kt * 16, X, 8 * c, hb + kt, 2)
                for ks in range(kt // 16):
                    A = sm.read(_mnmajor(a0 + ks * 256, 128, csa, 64))
                    for j in range(3):
                        B = sm.read(_mnmajor(b0 + (ks * 16 + j) * 16, 128, csb, cin))
                        acc[j] += A @ B.T
            for j in range(3):
                dW[:, gidx * 3 + j] += acc[j, :cout]
    ref = np.zeros((cout, 27, cin))
    for tap in range(27):
        dz, dy, dx = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        o = dz * g["plane"] + dy * g["wp"] + dx
        p = np.arange(r0, r1)
        ok = (p + o >= 0) & (p + o < g["rows"])
        ref[:, tap] = dY[p[ok]].T @ X[p[ok] + o]
    assert np.abs(dW - ref).max() <= 1e-12 * np.abs(ref).max()
