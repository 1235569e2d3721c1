"""FP64 CPU restatement of the reconstruction iteration (TEST INFRASTRUCTURE).

Used by tests/ only, as the checker of yoricktrtt_b200/recon.py: the same
objective (weighted least squares + smoothed isotropic TV of the B-spline
samples, Tomography_3D/Ytrtt3D_optim.i:128-234) and the same VMLM-B rules,
in numpy FP64 with the FP64 oracle projectors.  Parity with the reference
is unpinned here: the reference takes VMLM-B (OptimPack), TV (YTotVar) and
the spline sampling (SPL) from packages that are not in its repository.
"""
from __future__ import annotations

import math

import numpy as np


def spline_sample(x: np.ndarray) -> np.ndarray:
    """Separable [1/6, 2/3, 1/6] convolution along every axis, zero outside."""
    z = x.astype(np.float64).copy()
    for ax in range(x.ndim):
        src = z
        z = (2.0 / 3.0) * src
        lo = [slice(None)] * x.ndim
        hi = [slice(None)] * x.ndim
        lo[ax] = slice(1, None)
        hi[ax] = slice(None, -1)
        z[tuple(lo)] += src[tuple(hi)] / 6.0
        z[tuple(hi)] += src[tuple(lo)] / 6.0
    return z


def tv(z: np.ndarray, eps: float):
    """(sum sqrt(|grad z|^2 + eps^2) - eps, gradient), forward differences,
    arrays ordered [k][j][i] (or [j][i])."""
    d = []
    for ax in range(z.ndim):
        dd = np.zeros_like(z)
        sl_hi = [slice(None)] * z.ndim
        sl_lo = [slice(None)] * z.ndim
        sl_hi[ax] = slice(1, None)
        sl_lo[ax] = slice(None, -1)
        dd[tuple(sl_lo)] = z[tuple(sl_hi)] - z[tuple(sl_lo)]
        d.append(dd)
    s = np.sqrt(sum(dd * dd for dd in d) + eps * eps)
    f = float(np.sum(s - eps))
    g = np.zeros_like(z)
    for ax, dd in enumerate(d):
        q = dd / s
        g -= q
        sl_hi = [slice(None)] * z.ndim
        sl_lo = [slice(None)] * z.ndim
        sl_hi[ax] = slice(1, None)
        sl_lo[ax] = slice(None, -1)
        g[tuple(sl_hi)] += q[tuple(sl_lo)]
    return f, g


def objective(project, backproject, y, w=None, mu=0.0, eps=1e-3, spline=True):
    """fg(x) for f = 1/2 ||Hx - y||^2_W + mu TV(S x)."""
    def fg(x):
        r = project(x) - y
        wr = r if w is None else w * r
        f = 0.5 * float(np.sum(wr * r))
        g = backproject(wr)
        if mu > 0:
            z = spline_sample(x) if spline else x
            ft, gz = tv(z, eps)
            f += mu * ft
            g = g + mu * (spline_sample(gz) if spline else gz)
        return f, g
    return fg


def vmlmb(fg, x0, lower=0.0, upper=None, mem=5, maxiter=100, frtol=1e-6, armijo=1e-4,
          max_backtrack=30):
    """Same rules as yoricktrtt_b200.recon.vmlmb, in FP64."""
    lo = -math.inf if lower is None else float(lower)
    hi = math.inf if upper is None else float(upper)

    def clip(v):
        return np.clip(v, lo, hi)

    x = clip(np.array(x0, dtype=np.float64))
    f, g = fg(x)
    fs = [f]
    S, Y = [], []
    its = 0
    for it in range(1, maxiter + 1):
        free = np.ones_like(x)
        if lo > -math.inf:
            free[(x <= lo) & (g > 0)] = 0.0
        if hi < math.inf:
            free[(x >= hi) & (g < 0)] = 0.0
        pg = g * free
        pgn = math.sqrt(float(np.sum(pg * pg)))
        if pgn == 0.0:
            break
        q = pg.copy()
        used = []
        for s, yv in reversed(list(zip(S, Y))):
            sf, yf = s * free, yv * free
            sy = float(np.sum(sf * yf))
            if sy <= 0.0:
                continue
            a = float(np.sum(sf * q)) / sy
            q -= a * yf
            used.append((sf, yf, sy, a))
        if used:
            sf, yf, sy, _ = used[0]
            q *= sy / float(np.sum(yf * yf))
            for sf, yf, sy, a in reversed(used):
                b = float(np.sum(yf * q)) / sy
                q += (a - b) * sf
            d = -(q * free)
            alpha = 1.0
        else:
            d = -pg
            xn = math.sqrt(float(np.sum(x * x)))
            alpha = (0.1 * xn if xn > 0 else 1.0) / pgn
        gd = float(np.sum(g * d))
        if gd >= 0.0:
            S.clear()
            Y.clear()
            d = -pg
            xn = math.sqrt(float(np.sum(x * x)))
            alpha = (0.1 * xn if xn > 0 else 1.0) / pgn
            gd = float(np.sum(g * d))
        for _ in range(max_backtrack):
            xt = clip(x + alpha * d)
            ft, gt = fg(xt)
            if ft <= f + armijo * float(np.sum(g * (xt - x))):
                break
            denom = 2.0 * (ft - f - gd * alpha)
            aq = -gd * alpha * alpha / denom if denom > 0 else 0.5 * alpha
            alpha = min(max(aq, 0.1 * alpha), 0.5 * alpha)
        else:
            break
        s = xt - x
        yv = gt - g
        if float(np.sum(s * yv)) > 0.0:
            S.append(s)
            Y.append(yv)
            if len(S) > mem:
                S.pop(0)
                Y.pop(0)
        fprev = f
        x, f, g = xt, ft, gt
        its = it
        fs.append(f)
        if abs(fprev - f) <= frtol * max(abs(fprev), abs(f)):
            break
    return x, fs, its
