"""Seeded synthetic cases for the five benchmark configurations (C1-C5).

Each builder returns ``(params, z, bnx, bny)``: a filled :class:`abi.Params` and the bathymetry
grid ``z`` (float32, ``bny x bnx``) laid out like the reference's ``.cbf`` content — a grid that
spans x in [-W/2, W/2] and y in [0, L] (terrain_heightfield.cpp:213-242).  The grid equals the
mesh (``bnx = nx``, ``bny = ny``), so the library's bathymetry preparation samples it exactly at
the grid points.  Seeds follow ``12345 + 1000*config + member``.  No public dataset is involved:
all inputs are generated here from the configuration text.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

G = 9.81


def _grid_x(nx: int, dx: float) -> np.ndarray:
    return np.arange(nx, dtype=np.float64) * dx  # physical x from the west edge


def _set_side(b: abi.Boundary, kind: int, width: int, sea_level: float = 0.0,
              amplitude: float = 0.0, period: float = 0.0, theta_rad: float = 0.0) -> None:
    b.type = kind
    b.width = width
    b.sea_level = sea_level
    b.amplitude = amplitude
    b.period = period
    b.theta = theta_rad


def _bumps(rng: np.random.Generator, X: np.ndarray, Y: np.ndarray, xwet: float, L: float,
           count_range=(1, 4), height=(2.0, 8.0), sigma=(20.0, 80.0)) -> np.ndarray:
    out = np.zeros_like(X)
    n = int(rng.integers(count_range[0], count_range[1] + 1))
    for _ in range(n):
        hb = rng.uniform(*height)
        sg = rng.uniform(*sigma)
        xc = rng.uniform(0.0, max(xwet, 1.0))
        yc = rng.uniform(0.0, L)
        out += hb * np.exp(-((X - xc) ** 2 + (Y - yc) ** 2) / (2.0 * sg * sg))
    return out


def jonswap_components(n: int, hs: float, tp: float, gamma: float, rng: np.random.Generator,
                       fmin_ratio: float = 0.5, fmax_ratio: float = 3.0) -> np.ndarray:
    """``n`` JONSWAP components (amplitude, period, theta=0, phase) with Hs = 4 sqrt(m0)."""
    fp = 1.0 / tp
    f = np.linspace(fmin_ratio * fp, fmax_ratio * fp, n)
    df = f[1] - f[0]
    sig = np.where(f <= fp, 0.07, 0.09)
    r = np.exp(-((f - fp) ** 2) / (2.0 * sig * sig * fp * fp))
    S = G * G * (2 * math.pi) ** -4 * f ** -5 * np.exp(-1.25 * (fp / f) ** 4) * gamma ** r
    m0 = np.sum(S) * df
    S *= (hs / 4.0) ** 2 / m0
    amp = np.sqrt(2.0 * S * df)
    phase = rng.uniform(0.0, 2 * math.pi, n)
    return np.stack([amp, 1.0 / f, np.zeros(n), phase], axis=1)


def config1(nx: int = 512, ny: int = 64, flat_until: float = 44.0, correction_steps: int = 1):
    """C1 small flume: 512x64 cells, dx=dy=0.5 m, h=10 m flat then a 1:20 beach.

    The flat section ends at 44 m (not 64 m) so the 1:20 beach rises above still water
    inside the 255.5 m domain (shoreline at 244 m)."""
    dx = 0.5
    p = abi.default_params()
    p.nx, p.ny = nx, ny
    p.width, p.length = dx * (nx - 1), dx * (ny - 1)
    p.correction_steps = correction_steps
    p.timestep = 0.2 * dx / math.sqrt(G * 10.0)
    p.theta = 2.0
    p.manning = 0
    p.friction = 0.0
    _set_side(p.west, abi.CEL_BC_SINEWAVE, 2, amplitude=0.1, period=8.0)
    _set_side(p.east, abi.CEL_BC_SOLID, 2)
    _set_side(p.south, abi.CEL_BC_SOLID, 2)
    _set_side(p.north, abi.CEL_BC_SOLID, 2)
    x = _grid_x(nx, dx)
    b = np.where(x < flat_until, -10.0, -10.0 + (x - flat_until) / 20.0)
    z = np.tile(b, (ny, 1)).astype(np.float32)
    return p, z, nx, ny


def config2(nx: int = 2048, ny: int = 2048, n_waves: int = 64, member: int = 0, correction_steps: int = 1):
    """C2: 2048^2, dx=1 m; 1:30 slope from 15 m plus 1-4 Gaussian shoals; 64 JONSWAP
    components on the west boundary; 40-cell sponges N/E/S; Manning 0.02; breaking on."""
    rng = np.random.default_rng(12345 + 2000 + member)
    dx = 1.0
    p = abi.default_params()
    p.nx, p.ny = nx, ny
    p.width, p.length = dx * (nx - 1), dx * (ny - 1)
    p.correction_steps = correction_steps
    p.timestep = 0.2 * dx / math.sqrt(G * 15.0)
    p.manning = 1
    p.friction = 0.02
    p.dissipation_threshold = 0.25
    _set_side(p.west, abi.CEL_BC_IRREGULAR, 2)
    comps = jonswap_components(n_waves, 1.0, 10.0, 3.3, rng)
    p.west.n_waves = n_waves
    for i in range(n_waves):
        for k in range(4):
            p.west.waves[i][k] = float(comps[i, k])
    for side in (p.north, p.east, p.south):
        _set_side(side, abi.CEL_BC_SPONGE, 40)
    x = _grid_x(nx, dx)
    y = _grid_x(ny, dx)
    X, Y = np.meshgrid(x, y)
    B = -15.0 + X / 30.0 + _bumps(rng, X, Y, 450.0, p.length)
    return p, B.astype(np.float32), nx, ny


def config3(nx: int = 1024, ny: int = 1024, correction_steps: int = 1, wavemaker: bool = False):
    """C3: solitary wave H/d=0.1 in d=0.32 m (dx=0.025 m at 1024^2) running up a truncated
    cone (base radius 3.6 m, top radius 1.1 m, height 0.625 m) centred in the domain; solid
    walls.  ``wavemaker=True`` gives the sinusoidal wave-maker variant (west SineWave)."""
    span = 0.025 * 1023
    dx = span / (nx - 1)
    p = abi.default_params()
    p.nx, p.ny = nx, ny
    p.width, p.length = span, span
    p.correction_steps = correction_steps
    d = 0.32
    p.timestep = 0.2 * dx / math.sqrt(G * (d + 0.032))
    for side in (p.west, p.east, p.south, p.north):
        _set_side(side, abi.CEL_BC_SOLID, 2)
    if wavemaker:
        _set_side(p.west, abi.CEL_BC_SINEWAVE, 2, amplitude=0.01, period=2.0)
    else:
        p.n_solitons = 1
        s = p.solitons[0]
        s.H, s.theta, s.xc, s.yc, s.length = 0.032, 0.0, 3.0, span / 2.0, 1e30
    x = _grid_x(nx, dx)
    y = _grid_x(ny, dx)
    X, Y = np.meshgrid(x, y)
    r = np.hypot(X - span / 2.0, Y - span / 2.0)
    cone = np.clip((3.6 - r) / (3.6 - 1.1), 0.0, 1.0) * 0.625
    B = -d + cone
    return p, B.astype(np.float32), nx, ny


C4_SIZES = [(256, 256), (512, 256), (1024, 512), (1024, 1024), (2048, 512)]


def ensemble_member(nx: int, ny: int, rng: np.random.Generator, correction_steps: int = 1,
                    manning: float = 0.0, breaking: bool = False):
    """One member of the C4/C5 ensembles: dx=1 m, 15 m offshore, slope U[1/50,1/15] rising
    eastward, 1-4 bumps, west SineWave a~U[0.05,0.5] T~U[5,15], N/S solid, E 40-cell sponge."""
    dx = 1.0
    p = abi.default_params()
    p.nx, p.ny = nx, ny
    p.width, p.length = dx * (nx - 1), dx * (ny - 1)
    p.correction_steps = correction_steps
    p.timestep = 0.2 * dx / math.sqrt(G * 15.0)
    if manning > 0:
        p.manning = 1
        p.friction = manning
    slope = rng.uniform(1.0 / 50.0, 1.0 / 15.0)
    amp = rng.uniform(0.05, 0.5)
    per = rng.uniform(5.0, 15.0)
    _set_side(p.west, abi.CEL_BC_SINEWAVE, 2, amplitude=amp, period=per)
    _set_side(p.north, abi.CEL_BC_SOLID, 2)
    _set_side(p.south, abi.CEL_BC_SOLID, 2)
    _set_side(p.east, abi.CEL_BC_SPONGE, min(40, max(2, nx // 4)))
    x = _grid_x(nx, dx)
    y = _grid_x(ny, dx)
    X, Y = np.meshgrid(x, y)
    B = -15.0 + slope * X + _bumps(rng, X, Y, 15.0 / slope, p.length)
    return p, B.astype(np.float32), nx, ny


def c4_sizes(members: int = 64, first_member: int = 0) -> list:
    """(nx, ny) of C4 members first_member .. first_member+members-1, without building them."""
    return [C4_SIZES[int(np.random.default_rng(12345 + 4000 + m).integers(0, len(C4_SIZES)))]
            for m in range(first_member, first_member + members)]


def c5_sizes(members: int = 1024, first_member: int = 0) -> list:
    """(nx, ny) of C5 members first_member .. first_member+members-1, without building them."""
    sizes = list(range(128, 513, 32))
    out = []
    for m in range(first_member, first_member + members):
        rng = np.random.default_rng(12345 + 5000 + m)
        nx = sizes[int(rng.integers(0, len(sizes)))]
        out.append((nx, sizes[int(rng.integers(0, len(sizes)))]))
    return out


def config4(members: int = 64, correction_steps: int = 1, first_member: int = 0):
    """C4: 64 domains with sizes drawn by seed from C4_SIZES (``first_member`` offsets the seeds,
    e.g. per rank of a multi-GPU run)."""
    out = []
    for m in range(first_member, first_member + members):
        rng = np.random.default_rng(12345 + 4000 + m)
        nx, ny = C4_SIZES[int(rng.integers(0, len(C4_SIZES)))]
        out.append(ensemble_member(nx, ny, rng, correction_steps))
    return out


def config5(members: int = 1024, correction_steps: int = 1, first_member: int = 0):
    """C5: 1024 domains, nx and ny i.i.d. uniform over {128, 160, ..., 512}; Manning 0.02."""
    sizes = list(range(128, 513, 32))
    out = []
    for m in range(first_member, first_member + members):
        rng = np.random.default_rng(12345 + 5000 + m)
        nx = sizes[int(rng.integers(0, len(sizes)))]
        ny = sizes[int(rng.integers(0, len(sizes)))]
        out.append(ensemble_member(nx, ny, rng, correction_steps, manning=0.02, breaking=True))
    return out


def small_case(nx: int = 40, ny: int = 24, kind: str = "mixed", seed: int = 0, correction_steps: int = 1):
    """Small cases for parity tests; ``kind`` selects the boundary mix."""
    rng = np.random.default_rng(777 + seed)
    dx = 1.0
    p = abi.default_params()
    p.nx, p.ny = nx, ny
    p.width, p.length = dx * (nx - 1), dx * (ny - 1)
    p.correction_steps = correction_steps
    p.timestep = 0.2 * dx / math.sqrt(G * 6.0)
    x = _grid_x(nx, dx)
    y = _grid_x(ny, dx)
    X, Y = np.meshgrid(x, y)
    B = -5.0 + 0.12 * X + 1.5 * np.exp(-((X - 0.3 * nx) ** 2 + (Y - 0.5 * ny) ** 2) / (2 * (0.15 * nx) ** 2))
    if kind == "solid":
        for s in (p.west, p.east, p.south, p.north):
            _set_side(s, abi.CEL_BC_SOLID, 2)
        p.n_solitons = 1
        p.solitons[0].H, p.solitons[0].theta, p.solitons[0].xc, p.solitons[0].yc, p.solitons[0].length = \
            0.4, 0.3, 0.3 * nx, 0.5 * ny, 1e30
    elif kind == "sponge":
        _set_side(p.west, abi.CEL_BC_SINEWAVE, 2, amplitude=0.3, period=6.0, theta_rad=0.2)
        _set_side(p.east, abi.CEL_BC_SPONGE, 6)
        _set_side(p.north, abi.CEL_BC_SPONGE, 5)
        _set_side(p.south, abi.CEL_BC_SOLID, 2)
        p.manning = 1
        p.friction = 0.025
    elif kind == "irregular":
        _set_side(p.west, abi.CEL_BC_IRREGULAR, 2)
        comps = jonswap_components(8, 0.5, 6.0, 3.3, rng)
        p.west.n_waves = 8
        for i in range(8):
            for k in range(4):
                p.west.waves[i][k] = float(comps[i, k])
        _set_side(p.south, abi.CEL_BC_IRREGULAR, 2)
        p.south.n_waves = 3
        for i in range(3):
            p.south.waves[i][0], p.south.waves[i][1], p.south.waves[i][2], p.south.waves[i][3] = \
                0.05, 5.0 + i, 1.2, 0.3 * i
        _set_side(p.east, abi.CEL_BC_SPONGE, 4)
        _set_side(p.north, abi.CEL_BC_SOLID, 2)
    elif kind == "uts":
        _set_side(p.west, abi.CEL_BC_UTS, 2)
        _set_side(p.east, abi.CEL_BC_SOLID, 3)
        _set_side(p.south, abi.CEL_BC_SOLID, 2)
        _set_side(p.north, abi.CEL_BC_UTS, 2)
    else:  # mixed
        _set_side(p.west, abi.CEL_BC_SINEWAVE, 2, amplitude=0.25, period=5.0)
        _set_side(p.east, abi.CEL_BC_SPONGE, 5)
        _set_side(p.south, abi.CEL_BC_SOLID, 2)
        _set_side(p.north, abi.CEL_BC_SOLID, 2)
        p.n_solitons = 1
        p.solitons[0].H, p.solitons[0].theta, p.solitons[0].xc, p.solitons[0].yc, p.solitons[0].length = \
            0.3, 0.0, 0.4 * nx, 0.5 * ny, 0.3 * ny
    B = B + 0.05 * rng.standard_normal(B.shape)
    return p, B.astype(np.float32), nx, ny


def attach_uts(p: abi.Params, side: str, rows: np.ndarray) -> list:
    """Attach a (t, eta, hu, hv) table to a side; returns the ctypes buffer to keep alive."""
    import ctypes as C
    b = getattr(p, side)
    buf = (C.c_double * rows.size)(*rows.astype(np.float64).ravel().tolist())
    b.n_uts = rows.shape[0]
    b.uts = C.cast(buf, C.POINTER(C.c_double))
    return [buf]
