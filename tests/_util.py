"""Shared helpers for the tests (inputs, tolerances, comparisons)."""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "fft_golden.npz"

# relative L2 tolerances of the parity bar: FP32 2e-6, FP64 1e-13
TOL = {np.float32: 2e-6, np.float64: 1e-13}


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def uniform_cx(rng, *shape):
    return rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)


def normal_cx(rng, *shape, sigma=1.0):
    return sigma * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


def golden():
    return np.load(GOLDEN)
