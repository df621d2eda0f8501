"""Oracle for the irregular-wave spectrum generator (test infrastructure only).

A numpy restatement of the reference's generateSpectrumWaves (engine.cpp:3559-3776) in double
precision, used by tests/ to check the library's ``cel_spectrum_waves``.  Grids are accumulated in
float32 as the reference's float loops accumulate them (engine.cpp:3588-3593, 3623-3628), so both
sides get the same number of frequencies and directions.  The reference seeds ``rand()`` with the
clock; the restatement draws the same seeded splitmix64 sequence as the library, so phases can be
compared exactly.  Parity is unpinned by reference outputs: the generator sits in engine.cpp, which
does not build here, and the reference ships no generated file for a known input.
"""
from __future__ import annotations

import math

import numpy as np

PI_R = 3.1415   # the generator's value of pi (engine.cpp:3597, 3647, 3766-3769)
MASK = (1 << 64) - 1


def splitmix64(state: int):
    state = (state + 0x9E3779B97F4A7C15) & MASK
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return state, z ^ (z >> 31)


def spectrum_waves(hs: float, tp: float, mean_theta: float, depth: float, seed: int = 0):
    """Returns an (n, 4) array of {amplitude, period, theta (rad), phase}."""
    f32 = np.float32
    hs, tp, th_p, h = f32(hs), f32(tp), f32(mean_theta), f32(depth)
    gamma_s, spread_o, del_f, del_t, trunc = 3.3, 50.0, f32(0.005), f32(5.0), 0.05
    f_peak = f32(f32(1.0) / tp)
    Hs = float(min(hs, h * f32(0.5)))                         # engine.cpp:3579
    beta = 0.0624 / (0.23 + 0.033 * gamma_s - 0.185 / (1.9 + gamma_s))   # engine.cpp:3583
    # grids (float accumulation)
    f, v = [], max(del_f, f32(f_peak - f32(5) * del_f))
    f_end = f32(f_peak + f32(5) * del_f)
    while v <= f_end:
        f.append(v)
        v = f32(v + del_f)
    th, v = [], f32(f32(-20) + th_p)
    th_end = f32(f32(20) + th_p)
    while v <= th_end:
        th.append(v)
        v = f32(v + del_t)
    f = np.array(f, dtype=np.float64)
    th = np.array(th, dtype=np.float64)
    nf, nt = len(f), len(th)
    fp = float(f_peak)
    # frequency spectrum, JONSWAP shape with gamma 3.3 (engine.cpp:3596-3618; phiK is not applied)
    frat = f / fp
    sigma = np.where(f <= fp, 0.07, 0.09)
    E = beta * Hs * Hs / (f * frat ** 4) * np.exp(-1.25 / frat ** 4) * gamma_s ** np.exp(-(frat - 1) ** 2 / (2 * sigma ** 2))
    # cos^2s spreading, s = 50 (f/fp)^5 below the peak and 50 (f/fp)^-2.5 above (engine.cpp:3630-3648)
    s = np.where(frat < 1.0, spread_o * frat ** 5, spread_o * frat ** -2.5)
    ang = 0.5 * ((th[None, :] - float(th_p)) * PI_R / 180.0)
    D = np.cos(ang) ** (2 * s[:, None])
    D = D / D.sum(axis=1, keepdims=True)          # the normalisation removes beta_s (engine.cpp:3650-3659)
    ED = E[:, None] * D
    # truncation on column floor(nt/2 + 0.5) at 5 % of its maximum (engine.cpp:3697-3723)
    jc = int(math.floor(nt / 2.0 + 0.5))
    keep = np.nonzero(ED[:, jc] > trunc * ED[:, jc].max())[0]
    count = len(keep)
    out = []
    state = seed
    for k, i in enumerate(keep):
        # widths at grid position k of the full grid (engine.cpp:3754-3760)
        if k == 0:
            dfk = f[1] - f[0]
        elif k == count - 1:
            dfk = f[count - 1] - f[count - 2]
        else:
            dfk = (f[k + 1] - f[k]) / 2 + (f[k] - f[k - 1]) / 2
        for j in range(nt):
            state, r = splitmix64(state)
            rq = f32(f32(r % 10000) / f32(10000.0))
            phase = float(f32(float(f32(rq * f32(2))) * PI_R))
            out.append((math.sqrt(2 * ED[i, j] * dfk), 1.0 / f[i], th[j] * PI_R / 180.0, phase))
    return np.array(out)
