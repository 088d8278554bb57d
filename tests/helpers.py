"""Shared test helpers: golden fixtures and error measures."""
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, f"{name}.npz")) as z:
        return {k: z[k] for k in z.files}


def rel_err(a, b) -> float:
    """max |a - b| / max |b|"""
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) / scale


def rms_rel(a, b) -> float:
    """RMS over rows of |a_i - b_i| divided by the RMS of |b_i| (the force-error measure)."""
    a = np.asarray(a, float).reshape(-1, 3)
    b = np.asarray(b, float).reshape(-1, 3)
    return float(np.sqrt(np.mean(np.sum((a - b) ** 2, axis=1))) / np.sqrt(np.mean(np.sum(b ** 2, axis=1))))


def tensor_rel(a, b) -> float:
    """max |a_kl - b_kl| / max |b_kl| over a 3x3 stress tensor."""
    a = np.asarray(a, float).ravel()
    b = np.asarray(b, float).ravel()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
