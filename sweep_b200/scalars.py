"""Finite-difference coefficient tables, restated from the reference's
``src/sweep/scalars.py:25-93`` and ``src/sweep/propagator/_c.py:1134-1156``."""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np


def fd_coefficients(derivative_order: int = 2, accuracy_order: int = 2) -> np.ndarray:
    """Centred Taylor coefficients of the positive taps (float64)."""
    n = accuracy_order // 2
    pts = np.arange(-n, n + 1, dtype=np.float64)
    mat = np.array([pts ** i for i in range(2 * n + 1)])
    rhs = np.zeros(2 * n + 1)
    rhs[derivative_order] = math.factorial(derivative_order)
    return np.linalg.solve(mat, rhs)[-n:]


def second_derivative_coefficients_fp32(accuracy_order: int):
    """float32 ``(c0, c)`` whose stencil sums to exactly zero: the float32
    rounding residual of ``c0 + 2 sum(c)`` goes into the last tap."""
    c = fd_coefficients(2, accuracy_order)
    c0 = np.float32(-2 * c.sum())
    c = c.astype(np.float32)
    residual = Fraction(float(c0)) + 2 * sum(Fraction(float(x)) for x in c)
    if residual:
        target = Fraction(float(c[-1])) - residual / 2
        c[-1] = np.float32(float(target))
        if Fraction(float(c[-1])) != target:
            raise RuntimeError(f"no zero-sum float32 stencil of order {accuracy_order}")
    return c0, c


def staggered_grid_coes(M: int) -> np.ndarray:
    """Staggered first-derivative coefficients a_1..a_M (float32)."""
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
    equations: ``lap[0] = -c0``, ``lap[1..M]`` the second-derivative taps,
    ``grad[1..M]`` the centred first-derivative taps."""
    c0, c = second_derivative_coefficients_fp32(2 * M)
    lap = np.zeros(M + 1, np.float32)
    lap[0] = -c0
    lap[1:] = c
    grad = np.zeros(M + 1, np.float32)
    grad[1:] = fd_coefficients(1, 2 * M).astype(np.float32)
    return lap, grad
