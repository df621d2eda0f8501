"""Shared helpers for the parity tests."""
from __future__ import annotations

import numpy as np


def interior(a: np.ndarray) -> np.ndarray:
    return a[2:-2, 2:-2]


def field_errors(gpu: np.ndarray, ref: np.ndarray, sea_level: float = 0.0) -> dict:
    """Per-field max abs difference over interior cells, with the scale it is judged against:
    max |eta| for eta = w - sea level, and the momentum scale max(|hu|, |hv|) for hu and hv
    (in a one-dimensional run hv is rounding noise, so its own maximum is no scale)."""
    g = interior(np.asarray(gpu, dtype=np.float64))
    r = interior(np.asarray(ref, dtype=np.float64))
    mom = float(max(np.max(np.abs(r[..., 1])), np.max(np.abs(r[..., 2]))))
    out = {}
    for k, name in enumerate(("eta", "hu", "hv")):
        a = g[..., k] - (sea_level if k == 0 else 0.0)
        b = r[..., k] - (sea_level if k == 0 else 0.0)
        scale = float(np.max(np.abs(b))) if k == 0 else mom
        out[name] = (float(np.max(np.abs(a - b))), scale)
    return out


def rel_ok(errs: dict, rtol: float, atol: float = 0.0) -> bool:
    return all(e <= rtol * scale + atol for e, scale in errs.values())


def eta_rms(gpu: np.ndarray, ref: np.ndarray) -> float:
    d = interior(np.asarray(gpu, dtype=np.float64))[..., 0] - interior(np.asarray(ref, dtype=np.float64))[..., 0]
    return float(np.sqrt(np.mean(d * d)))


def surface_rms(gpu: np.ndarray, ref: np.ndarray, bed: np.ndarray) -> float:
    """RMS over interior cells of the free-surface difference, the surface being max(w, B): the water
    level where a cell holds water and the bed where it is dry.  Below the bed, w is no surface: a
    sponge over dry land keeps pulling it toward sea level (w = sl + gamma (w - sl)) while the depth
    stays 0, and single- and double-precision runs of that decay part by centimetres without moving
    any water."""
    b = interior(np.asarray(bed, dtype=np.float64))
    g = np.maximum(interior(np.asarray(gpu, dtype=np.float64))[..., 0], b)
    r = np.maximum(interior(np.asarray(ref, dtype=np.float64))[..., 0], b)
    d = g - r
    return float(np.sqrt(np.mean(d * d)))
