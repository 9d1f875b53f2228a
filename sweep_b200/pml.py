"""CPML damping profiles on the runtime grid, restated from the reference's
``src/sweep/equations/pml.py:81-269`` (``setup_pml``, ``set_cpml_profiles_r``,
``set_cpml_profiles_s``).  Built in float32 numpy exactly as the reference
builds them (``src/sweep/propagator/base.py:1006-1069``: ``max_vel`` 4500 m/s
and ``pml_freq`` 25 Hz by default, ``r_val`` 1e-3, ``n_power`` 2)."""
from __future__ import annotations

import math

import numpy as np


def setup_pml(width, start, max_pml, dt, n, max_vel, pml_freq, offset=0.0,
              r_val=0.001, n_power=2, eps=1e-9):
    """``(a, b)`` of one axis: a = exp(-(sigma + alpha) dt) inside the band
    (0 outside), b = sigma / (sigma + alpha) (a - 1)."""
    dtype = np.float32
    alpha0 = math.pi * pml_freq
    if max_pml == 0:
        return np.zeros(n, dtype), np.zeros(n, dtype)
    sigma0 = -(1 + n_power) * max_vel * math.log(r_val) / (2 * max_pml)
    x = np.arange(n, dtype=dtype) + dtype(offset)
    f0 = (dtype(start[0]) - x) / dtype(width[0]) if width[0] else np.zeros_like(x)
    f1 = (x - dtype(start[1])) / dtype(width[1]) if width[1] else np.zeros_like(x)
    frac = np.clip(np.maximum(f0, f1), 0.0, 1.0)
    sigma = dtype(sigma0) * (frac ** n_power)
    alpha = dtype(alpha0) * (dtype(1.0) - frac)
    sa = sigma + alpha
    sa = np.where(np.abs(sa) < eps, dtype(eps), sa)
    a = np.exp(-sa * abs(dt)).astype(dtype, copy=False)
    b = (sigma / sa) * (a - dtype(1.0))
    a = a.copy()
    a[frac == 0] = dtype(0.0)
    return a, b.astype(dtype, copy=False)


def cpml_profiles_r(pads, M, dt, spacing, shape, max_vel=4500.0, pml_freq=25.0):
    """Regular-grid profiles, per axis in shape order: ``(a, b, db/daxis)``.

    ``pads`` = flat ``[lo0, hi0, lo1, hi1, ...]`` PML widths, ``shape`` the
    runtime shape (physical + 2 pad + 2 M per axis)."""
    out = []
    for d, n in enumerate(shape):
        w = pads[2 * d: 2 * d + 2]
        start = [float(M + w[0]), float(n - 1 - M - w[1])]
        max_pml = max(w[0] * spacing[d], w[1] * spacing[d])
        a, b = setup_pml(w, start, max_pml, dt, n, max_vel, pml_freq)
        db = np.gradient(b, spacing[d]).astype(np.float32)
        out.append((a, b, db))
    return out


def cpml_profiles_s(pads, M, dt, spacing, shape, max_vel=4500.0, pml_freq=25.0):
    """Staggered-grid profiles, per axis in shape order: ``(a, b, a_half, b_half)``
    (integer and half-integer positions)."""
    out = []
    for d, n in enumerate(shape):
        w = pads[2 * d: 2 * d + 2]
        start = [M + w[0], n - 1 - M - w[1]]
        max_pml = max(w[0] * spacing[d], w[1] * spacing[d])
        a, b = setup_pml(w, start, max_pml, dt, n, max_vel, pml_freq, offset=0.0)
        ah, bh = setup_pml(w, start, max_pml, dt, n, max_vel, pml_freq, offset=0.5)
        out.append((a, b, ah, bh))
    return out
