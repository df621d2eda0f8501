"""ctypes binding of the CPU oracle (test infrastructure only).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this module; the product
(celeris_b200/) never does.  ``Oracle(params, z, bnx, bny, real="f64")`` wraps one instance of
the C++ transcription in oracle/celeris_oracle.hpp (``real="f32"`` for the FP32 build).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))
from celeris_b200 import abi  # noqa: E402  (struct definitions only)

_libs: dict = {}


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(real: str) -> C.CDLL:
    if real not in _libs:
        if real == "ref":
            # the reference's own compute.hlsl driven by the oracle's schedule (ref_build.py)
            path = os.path.join(_HERE, "_ref", "libref_shader.so")
            if not os.path.exists(path):
                raise FileNotFoundError("oracle/_ref/libref_shader.so is not built (python oracle/ref_build.py)")
        else:
            path = os.path.join(_HERE, "_build", f"liboracle_{real}.so")
            if not os.path.exists(path):
                build()
        L = C.CDLL(path)
        vp, i, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
        fp = C.POINTER(C.c_float)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [C.POINTER(abi.Params), fp, i, i, fp]
        L.orc_destroy.argtypes = [vp]
        L.orc_reset_timestep.argtypes = [vp, C.POINTER(abi.Stats)]
        L.orc_timestep.argtypes = [vp]
        L.orc_timesteps.argtypes = [vp, i, C.POINTER(abi.Stats)]
        L.orc_physical_steps.argtypes = [vp, i, C.POINTER(abi.Stats)]
        L.orc_get_state.argtypes = [vp, dp]
        L.orc_set_state.argtypes = [vp, dp]
        L.orc_get_aux.argtypes = [vp, dp]
        L.orc_get_bottom.argtypes = [vp, dp]
        L.orc_get_coefs.argtypes = [vp, dp, dp]
        L.orc_time_scheme.argtypes = [vp]
        L.orc_total_time.argtypes = [vp]
        L.orc_total_time.restype = C.c_double
        L.orc_passes.argtypes = [vp]
        L.orc_add_solitary_wave.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_new_terrain.argtypes = [vp, C.POINTER(C.c_float), i, i]
        L.orc_rebootstrap.argtypes = [vp]
        L.orc_cr_solve.argtypes = [i, dp, dp, dp, dp, dp]
        L.orc_time_physical_steps.argtypes = [vp, i]
        L.orc_time_physical_steps.restype = C.c_double
        L.orc_threads.restype = i
        _libs[real] = L
    return _libs[real]


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    def __init__(self, params: abi.Params, z: np.ndarray, bnx: int, bny: int, real: str = "f64",
                 hot: np.ndarray | None = None):
        self.L = _lib(real)
        self.nx, self.ny = params.nx, params.ny
        self.NX, self.NY = self.nx + 4, self.ny + 4
        self._z = np.ascontiguousarray(z, dtype=np.float32)
        hp = None
        if hot is not None:
            self._hot = np.ascontiguousarray(hot, dtype=np.float32)
            hp = self._hot.ctypes.data_as(C.POINTER(C.c_float))
        self.h = self.L.orc_create(C.byref(params), self._z.ctypes.data_as(C.POINTER(C.c_float)), bnx, bny, hp)

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reset_timestep(self) -> dict:
        s = abi.Stats()
        self.L.orc_reset_timestep(self.h, C.byref(s))
        return s.as_dict()

    def timestep(self):
        self.L.orc_timestep(self.h)

    def timesteps(self, n: int) -> dict:
        s = abi.Stats()
        self.L.orc_timesteps(self.h, n, C.byref(s))
        return s.as_dict()

    def physical_steps(self, n: int) -> dict:
        s = abi.Stats()
        self.L.orc_physical_steps(self.h, n, C.byref(s))
        return s.as_dict()

    def state(self) -> np.ndarray:
        out = np.zeros((self.NY, self.NX, 4), dtype=np.float64)
        self.L.orc_get_state(self.h, _dp(out))
        return out

    def set_state(self, st: np.ndarray):
        a = np.ascontiguousarray(st, dtype=np.float64)
        self.L.orc_set_state(self.h, _dp(a))

    def aux(self) -> np.ndarray:
        out = np.zeros((self.NY, self.NX, 4), dtype=np.float64)
        self.L.orc_get_aux(self.h, _dp(out))
        return out

    def bottom(self) -> np.ndarray:
        out = np.zeros((self.NY, self.NX, 3), dtype=np.float64)
        self.L.orc_get_bottom(self.h, _dp(out))
        return out

    def coefs(self):
        ax = np.zeros((self.NY, self.NX, 3), dtype=np.float64)
        ay = np.zeros((self.NY, self.NX, 3), dtype=np.float64)
        self.L.orc_get_coefs(self.h, _dp(ax), _dp(ay))
        return ax, ay

    @property
    def time_scheme(self) -> int:
        return self.L.orc_time_scheme(self.h)

    @property
    def total_time(self) -> float:
        return self.L.orc_total_time(self.h)

    @property
    def passes(self) -> int:
        return self.L.orc_passes(self.h)

    def add_solitary_wave(self, H, theta_deg, xc, yc):
        self.L.orc_add_solitary_wave(self.h, H, theta_deg, xc, yc)

    def rebootstrap(self):
        """Recompute the Pass1 faces from the current state at the next pass."""
        self.L.orc_rebootstrap(self.h)

    def new_terrain(self, z: np.ndarray):
        """newTerrainSettings with a new bathymetry grid (same layout as the creation grid)."""
        z = np.ascontiguousarray(z, dtype=np.float32)
        self.L.orc_new_terrain(self.h, z.ctypes.data_as(C.POINTER(C.c_float)), z.shape[1], z.shape[0])

    def time_physical_steps(self, n: int) -> float:
        return self.L.orc_time_physical_steps(self.h, n)


def cr_solve(a, b, c, d, real: str = "f64") -> np.ndarray:
    L = _lib(real)
    n = len(b)
    arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (a, b, c, d)]
    x = np.zeros(n)
    L.orc_cr_solve(n, *[_dp(v) for v in arrs], _dp(x))
    return x


def threads(real: str = "f32") -> int:
    return _lib(real).orc_threads()
