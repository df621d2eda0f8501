"""Storage precision of the time-invariant Thomas factors, measured on the C4 systems.

The mixed form keeps the factors (c', 1/den, m) of each tridiagonal system in FP32.  Storing them in
FP16 would save 6 of the 32 bytes per cell of a solve; this file measures what it would cost in
accuracy.  It takes rows and columns of the dispersive systems of a C4 member (the coefficients the
FP64 oracle builds as engine.cpp:2612-2887 does), factors each system in FP64, rounds the factors
to FP32 or to FP16, and solves in FP32 against the FP64 solution for three right-hand sides: a smooth
wave, white noise, and the matrix applied to a wave-shaped field.  One FP32 iterative-refinement step
(residual with the FP32 matrix, a second solve with the FP16 factors) is measured as well.

Measured (C4 member 5, 256 x 256, depth 15 m offshore, dx 1 m, K1 up to 90; two rows and two
columns, three right-hand sides each): FP32 factors give at most 1.8e-7 relative error per solve,
FP16 factors 2.6e-4..4.1e-4, and FP16 with one refinement step at most 1.1e-6.  FP16 alone thus
perturbs every dispersive increment by about 3e-4 of itself, three orders of magnitude above FP32.  The refinement step repairs it but needs the FP32 matrix (12 bytes per cell)
and a second sweep over the factors (6 more), more than the 6 bytes FP16 saves, so the solves keep
FP32 factors.  The test asserts those orders of magnitude.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from celeris_b200 import cases


def _thomas(A, B, C):
    n = len(B)
    cp, inv, m = np.zeros(n), np.zeros(n), np.zeros(n)
    cprev = 0.0
    for i in range(n):
        den = B[i] - A[i] * cprev
        iv = 1.0 / den
        cprev = C[i] * iv
        cp[i], inv[i], m[i] = cprev, iv, -A[i] * iv
    return cp, inv, m


def _solve(cp, inv, m, r, dt):
    n = len(r)
    y = np.zeros(n, dt)
    acc = dt(0)
    for i in range(n):   # y_i = inv_i r_i + m_i y_{i-1}, as the solver kernels sweep it
        acc = dt(inv[i]) * dt(r[i]) + dt(m[i]) * acc
        y[i] = acc
    x = np.zeros(n, dt)
    acc = dt(0)
    for i in range(n - 1, -1, -1):   # x_i = y_i - c'_i x_{i+1}
        acc = y[i] - dt(cp[i]) * acc
        x[i] = acc
    return x


def _matvec(A, B, C, x):
    y = B * x
    y[1:] += A[1:] * x[:-1]
    y[:-1] += C[:-1] * x[1:]
    return y


@pytest.fixture(scope="module")
def systems():
    p, z, bnx, bny = cases.config4(1, 1, first_member=5)[0]
    o = O.Oracle(p, z, bnx, bny, "f64")
    ax, ay = o.coefs()
    out = []
    for row in (p.ny // 4, p.ny // 2):          # x systems (rows)
        out.append(tuple(ax[row + 2, 2:-2, k] for k in range(3)))
    for col in (p.nx // 8, p.nx // 3):          # y systems (columns)
        out.append(tuple(ay[2:-2, col + 2, k] for k in range(3)))
    return out


def test_fp16_factors_cost_accuracy_that_one_refinement_step_restores(systems):
    rng = np.random.default_rng(7)
    worst = {"f32": 0.0, "f16": 0.0, "f16_refined": 0.0}
    best_f16 = 1.0
    for A, B, C in systems:
        n = len(B)
        assert ((B - 1) / 2).max() > 10                    # deep water: strongly dispersive rows
        cp, inv, m = _thomas(A, B, C)
        wave = np.sin(np.arange(n) * 2 * np.pi / 40.0)
        for r in (wave * 1e-3, rng.standard_normal(n) * 1e-3, _matvec(A, B, C, wave * 1e-3)):
            x = _solve(cp, inv, m, r, np.float64)
            nx = np.linalg.norm(x)
            f32 = [a.astype(np.float32) for a in (cp, inv, m)]
            f16 = [a.astype(np.float16).astype(np.float32) for a in (cp, inv, m)]
            r32 = r.astype(np.float32)
            x32 = _solve(*f32, r32, np.float32).astype(np.float64)
            x16 = _solve(*f16, r32, np.float32).astype(np.float64)
            A32, B32, C32 = (a.astype(np.float32) for a in (A, B, C))
            res = (r32 - _matvec(A32, B32, C32, x16.astype(np.float32))).astype(np.float32)
            x16r = x16 + _solve(*f16, res, np.float32).astype(np.float64)
            e = {"f32": np.linalg.norm(x32 - x) / nx, "f16": np.linalg.norm(x16 - x) / nx,
                 "f16_refined": np.linalg.norm(x16r - x) / nx}
            for k in worst:
                worst[k] = max(worst[k], e[k])
            best_f16 = min(best_f16, e["f16"])
    print({k: f"{v:.2e}" for k, v in worst.items()}, f"best f16 {best_f16:.2e}")
    assert worst["f32"] < 1e-6
    assert best_f16 > 1e-5                 # FP16 factors: every case at least 1e-5 off
    assert worst["f16"] > 100 * worst["f32"]
    assert worst["f16_refined"] < 2e-6    # one FP32 refinement step brings it back near FP32
