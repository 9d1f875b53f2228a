"""Shared helpers of the parity tests: float64 metrics (float32 norms of
elastic gradients underflow) and golden-fixture loading."""
from pathlib import Path

import numpy as np

GOLD = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def load(case):
    return np.load(GOLD / f"{case}.npz")
