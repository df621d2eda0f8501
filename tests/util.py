"""Shared helpers for the parity tests."""
from __future__ import annotations

import numpy as np


def interior(a: np.ndarray) -> np.ndarray:
    return a[2:-2, 2:-2]


def field_errors(gpu: np.ndarray, ref: np.ndarray, sea_level: float = 0.0) -> dict:
    """Per-field max abs difference and the reference's max magnitude over interior cells.

    Fields: eta = w - sea level, hu, hv."""
    g = interior(np.asarray(gpu, dtype=np.float64))
    r = interior(np.asarray(ref, dtype=np.float64))
    out = {}
    for k, name in enumerate(("eta", "hu", "hv")):
        a = g[..., k] - (sea_level if k == 0 else 0.0)
        b = r[..., k] - (sea_level if k == 0 else 0.0)
        out[name] = (float(np.max(np.abs(a - b))), float(np.max(np.abs(b))))
    return out


def rel_ok(errs: dict, rtol: float, atol: float = 0.0) -> bool:
    return all(e <= rtol * scale + atol for e, scale in errs.values())


def eta_rms(gpu: np.ndarray, ref: np.ndarray) -> float:
    d = interior(np.asarray(gpu, dtype=np.float64))[..., 0] - interior(np.asarray(ref, dtype=np.float64))[..., 0]
    return float(np.sqrt(np.mean(d * d)))
