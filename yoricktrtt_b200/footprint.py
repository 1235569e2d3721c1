"""Tabulated B-spline footprint used by the table-mode projectors.

Restates ``_monodim_bspline`` + ``_cumsum`` + ``_make_footprint``
(``Ytrtt_tomobj.i:140-196, 296-337``): a degree-``deg`` centred B-spline is
sampled on ``m`` points ``coord[i] = i*step - (n-1)/2`` with ``n = 2*deg+3``
and ``step = (n-1)/(m-1)``; ``cum`` is its trapezoid partial sum.  The
projectors look ``cum`` up at ``floor`` of a continuous table index, so the
table *is* the footprint model of ``trtt_PB2D/FB2D/PB3D/CB3D``.

The reference draws the samples through an external spline package that is
not in its repository; the samples here come from the closed-form B-spline
(recursion on the degree), which is the function that package evaluates.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def bspline(deg: int, x: np.ndarray) -> np.ndarray:
    """Centred B-spline of degree ``deg`` at ``x`` by the recursion
    b_n(x) = ((n+1)/2 + x) b_{n-1}(x+1/2)/n + ((n+1)/2 - x) b_{n-1}(x-1/2)/n,
    with b_0 the unit box on [-1/2, 1/2)."""
    x = np.asarray(x, dtype=np.float64)
    memo: dict[tuple[int, int], np.ndarray] = {}

    def f(d: int, s2: int) -> np.ndarray:  # b_d(x + s2/2)
        key = (d, s2)
        if key in memo:
            return memo[key]
        xs = x + 0.5 * s2
        if d == 0:
            out = ((xs >= -0.5) & (xs < 0.5)).astype(np.float64)
        else:
            out = ((0.5 * (d + 1) + xs) * f(d - 1, s2 + 1)
                   + (0.5 * (d + 1) - xs) * f(d - 1, s2 - 1)) / d
        memo[key] = out
        return out

    return f(int(deg), 0)


@dataclass
class FootprintTable:
    """The five footprint arguments of the table-mode projectors
    (``plugin/trtt_3D_projectors.h:299``): footprint, cum_footprint,
    size_footprint, step_footprint, coord_footprint."""

    deg: int
    footprint: np.ndarray
    cum: np.ndarray
    coord: np.ndarray
    step: float

    @property
    def size(self) -> int:
        return int(self.cum.shape[0])


def make_footprint(deg: int, m: int) -> FootprintTable:
    """Build the table of a degree-``deg`` B-spline with ``m`` samples."""
    if m < 2:
        raise ValueError("size_footprint must be >= 2")
    if not 0 <= deg <= 9:
        raise ValueError("spline degree must be in 0..9")
    n = 2 * deg + 3
    step = float(n - 1) / float(m - 1)
    coord = np.arange(m, dtype=np.float64) * step - 0.5 * (n - 1)
    fp = bspline(deg, coord)
    cum = np.zeros(m)
    # sequential trapezoid sum, same rounding sequence as the C oracle
    inc = 0.5 * step * (fp[:-1] + fp[1:])
    acc = 0.0
    for i in range(1, m):
        acc = acc + inc[i - 1]
        cum[i] = acc
    return FootprintTable(deg, fp, cum, coord, step)
