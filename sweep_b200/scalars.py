"""Finite-difference coefficient tables of the stencils (the values of the
reference's ``src/sweep/scalars.py:25-93`` and
``src/sweep/propagator/_c.py:1134-1156``, derived here in closed form with
exact rational arithmetic).

Centred differences of half-width n have the closed-form weights

* first derivative:  g_k = (-1)^(k+1) (n!)^2 / (k (n-k)! (n+k)!)
* second derivative: c_k = 2 (-1)^(k+1) (n!)^2 / (k^2 (n-k)! (n+k)!),
  centre c_0 = -2 sum_k c_k,

for k = 1..n (the weight of u(x + k h) and of u(x - k h)).  The stencils run
in float32 in difference form, sum_k c_k (u(x + k h) - u(x)) + ..., which is
exact for a constant field only if the float32 taps sum to the float32 centre
exactly.  So the float32 table rounds the centre and the inner taps, and the
last tap takes whatever makes c_0 / 2 = c_1 + ... + c_n hold exactly (for
order 8 that is the reference kernels' constant ((c0 / 2 - c1) - c2) - c3,
operators/laplace.cuh:331-335).
"""
from __future__ import annotations

from fractions import Fraction
from math import factorial

import numpy as np


def _centred(n: int, second: bool) -> list:
    """Exact centred weights k = 1..n of the first (second=False) or second
    derivative."""
    out = []
    for k in range(1, n + 1):
        w = Fraction((-1) ** (k + 1) * factorial(n) ** 2, factorial(n - k) * factorial(n + k))
        out.append(2 * w / (k * k) if second else w / k)
    return out


def _f32(x: Fraction) -> np.float32:
    return np.float32(float(x))


def laplacian_taps_fp32(n: int):
    """float32 ``(centre, taps)`` of the half-width-n second derivative,
    ``centre`` = |c_0| > 0, with ``centre == 2 * sum(taps)`` exactly."""
    c = _centred(n, True)
    centre = _f32(2 * sum(c))
    taps = np.array([_f32(x) for x in c], np.float32)
    last = Fraction(float(centre)) / 2 - sum(Fraction(float(t)) for t in taps[:-1])
    taps[-1] = _f32(last)
    if Fraction(float(taps[-1])) != last:
        raise RuntimeError(f"no exactly zero-sum float32 stencil of half-width {n}")
    return centre, taps


def staggered_grid_coes(M: int) -> np.ndarray:
    """Staggered first-derivative weights a_1..a_M (float32) of the half-cell
    stencil sum_m a_m (u(x + (m - 1/2) h) - u(x - (m - 1/2) h)) / h: the
    Lagrange-derivative weights on the points +-(2m - 1) / 2."""
    a = np.zeros(M, dtype=np.float32)
    for m in range(1, M + 1):
        am = (-1) ** (m + 1) / (2 * m - 1)
        prod = 1.0
        for n in range(1, M + 1):
            if n != m:
                num = (2 * n - 1) ** 2
                prod *= abs(num / (num - (2 * m - 1) ** 2))
        a[m - 1] = am * prod
    return a


def centred_tables(M: int):
    """``(lap, grad)`` float32 tables of length M+1 for the 2nd-order-in-time
    equations: ``lap[0]`` the centre magnitude, ``lap[1..M]`` the
    second-derivative taps, ``grad[1..M]`` the centred first-derivative taps."""
    centre, taps = laplacian_taps_fp32(M)
    lap = np.zeros(M + 1, np.float32)
    lap[0] = centre
    lap[1:] = taps
    grad = np.zeros(M + 1, np.float32)
    grad[1:] = [_f32(x) for x in _centred(M, False)]
    return lap, grad
