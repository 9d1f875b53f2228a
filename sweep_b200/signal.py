"""Source wavelets (reference ``src/sweep/signal.py:10-21``)."""
import numpy as np


def ricker(t, f):
    """Ricker wavelet ``(1 - 2 (pi f t)^2) exp(-(pi f t)^2)``; shift ``t`` for a delay."""
    a = (np.pi * f * np.asarray(t)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)
