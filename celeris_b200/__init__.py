"""celeris_b200: B200-native Celeris Boussinesq timestep path (host-side Python mirror).

The computation lives in the CUDA/C++ library ``_build/libceleris_b200.so`` behind the C ABI of
``include/celeris_b200.h``; this module only marshals arguments.  :class:`Engine` mirrors the
reference's ``ShallowWaterEngine`` (remesh, resetTimestep, timestep, state access) and
:class:`Batch` advances many domains together.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .abi import (CEL_BC_IRREGULAR, CEL_BC_SINEWAVE, CEL_BC_SOLID, CEL_BC_SPONGE, CEL_BC_UTS,  # noqa: F401
                  CEL_FORM_FUSED, CEL_FORM_MIXED, CEL_FORM_PLAIN, CelError, Params, Stats, check,
                  default_params, lib)

FORMS = {"plain": CEL_FORM_PLAIN, "fused": CEL_FORM_FUSED, "mixed": CEL_FORM_MIXED}


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def params_from_cml(path: str) -> Params:
    p = Params()
    check(lib().cel_params_from_cml(path.encode(), C.byref(p)))
    return p


def read_cbf(path: str) -> np.ndarray:
    bnx, bny = C.c_int(), C.c_int()
    check(lib().cel_read_cbf(path.encode(), None, 0, C.byref(bnx), C.byref(bny)))
    z = np.zeros((bny.value, bnx.value), dtype=np.float32)
    check(lib().cel_read_cbf(path.encode(), _fp(z), z.size, C.byref(bnx), C.byref(bny)))
    return z


class Engine:
    """One domain (``cel_engine``)."""

    def __init__(self, params: Params, z: np.ndarray | None = None, form: str | int = "plain"):
        self._params = params
        f = FORMS[form] if isinstance(form, str) else int(form)
        self.form = f
        h = C.c_void_p()
        if z is None:
            check(lib().cel_create(C.byref(params), None, 0, 0, f, C.byref(h)))
        else:
            self._z = np.ascontiguousarray(z, dtype=np.float32)
            check(lib().cel_create(C.byref(params), _fp(self._z), self._z.shape[1], self._z.shape[0], f, C.byref(h)))
        self.h = h
        nx, ny = C.c_int(), C.c_int()
        check(lib().cel_get_dims(self.h, C.byref(nx), C.byref(ny)))
        self.nx, self.ny = nx.value, ny.value

    def close(self):
        if getattr(self, "h", None):
            lib().cel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def shape(self):
        return (self.ny + 4, self.nx + 4)

    def remesh(self):
        check(lib().cel_remesh(self.h))

    def set_stream(self, stream_ptr: int | None):
        check(lib().cel_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def state(self) -> np.ndarray:
        out = np.zeros(self.shape + (4,), dtype=np.float32)
        check(lib().cel_get_state(self.h, _fp(out)))
        return out

    def set_state(self, rgba: np.ndarray):
        a = np.ascontiguousarray(rgba, dtype=np.float32)
        assert a.shape == self.shape + (4,)
        check(lib().cel_set_state(self.h, _fp(a)))

    def bottom(self) -> np.ndarray:
        out = np.zeros(self.shape + (3,), dtype=np.float32)
        check(lib().cel_get_bottom(self.h, _fp(out)))
        return out

    def aux(self) -> np.ndarray:
        out = np.zeros(self.shape + (4,), dtype=np.float32)
        check(lib().cel_get_aux(self.h, _fp(out)))
        return out

    def reset_timestep(self, realworld_dt: float = 0.0, elapsed: float = 0.0) -> dict:
        s = Stats()
        check(lib().cel_reset_timestep(self.h, realworld_dt, elapsed, C.byref(s)))
        return s.as_dict()

    def timestep(self):
        check(lib().cel_timestep(self.h))

    def timesteps(self, n: int):
        check(lib().cel_timesteps(self.h, n))

    def physical_steps(self, n: int):
        check(lib().cel_physical_steps(self.h, n))

    def stats(self) -> dict:
        s = Stats()
        check(lib().cel_get_stats(self.h, C.byref(s)))
        return s.as_dict()

    def add_solitary_wave(self, H: float, theta_deg: float, xc: float, yc: float):
        check(lib().cel_add_solitary_wave(self.h, H, theta_deg, xc, yc))

    def water_height(self, x: float, y: float) -> float:
        """getWaterHeight at world point (x, y): terrain height + the 4x4 block's mean depth."""
        out = C.c_float()
        check(lib().cel_get_water_height(self.h, x, y, C.byref(out)))
        return np.float32(out.value)

    def set_bathymetry(self, z: np.ndarray):
        """newTerrainSettings with a new bathymetry grid (the .cbf layout, rows = y)."""
        z = np.ascontiguousarray(z, dtype=np.float32)
        check(lib().cel_set_bathymetry(self.h, _fp(z), z.shape[1], z.shape[0]))

    def synchronize(self):
        check(lib().cel_synchronize(self.h))

    def kernel_timing(self, enable: bool = True):
        check(lib().cel_engine_kernel_timing(self.h, int(enable)))

    def kernel_times(self) -> dict:
        return _kernel_times(self.h, 0)


def _kernel_times(handle, is_batch: int) -> dict:
    cap = 64
    names = (C.c_char * 64 * cap)()
    ms = (C.c_double * cap)()
    n_l = (C.c_longlong * cap)()
    n = C.c_int()
    check(lib().cel_kernel_times(handle, is_batch, C.cast(names, C.POINTER(C.c_char * 64)), ms, n_l, cap, C.byref(n)))
    return {names[i].value.decode(): (ms[i], n_l[i]) for i in range(n.value)}


class Batch:
    """Many domains advanced together (``cel_batch``)."""

    def __init__(self, members, form: str | int = "mixed", lanes: int = 0):
        """``lanes``: how many lanes the members are split into (0 = the library's default)."""
        f = FORMS[form] if isinstance(form, str) else int(form)
        self.form = f
        self.members = list(members)
        n = len(self.members)
        self._params = [m[0] for m in self.members]
        self._z = [np.ascontiguousarray(m[1], dtype=np.float32) for m in self.members]
        pp = (C.POINTER(Params) * n)(*[C.pointer(p) for p in self._params])
        zz = (C.POINTER(C.c_float) * n)(*[_fp(z) for z in self._z])
        bnx = (C.c_int * n)(*[z.shape[1] for z in self._z])
        bny = (C.c_int * n)(*[z.shape[0] for z in self._z])
        h = C.c_void_p()
        check(lib().cel_batch_create_lanes(n, pp, zz, bnx, bny, f, int(lanes), C.byref(h)))
        self.h = h
        self.n = n
        self.shapes = [(p.ny + 4, p.nx + 4) for p in self._params]

    def close(self):
        if getattr(self, "h", None):
            lib().cel_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cells(self) -> int:
        return int(lib().cel_batch_cells(self.h))

    @property
    def lanes(self) -> int:
        return int(lib().cel_batch_lanes(self.h))

    def set_stream(self, stream_ptr: int | None):
        check(lib().cel_batch_set_stream(self.h, C.c_void_p(stream_ptr or 0)))

    def use_graph(self, enable: bool = True):
        check(lib().cel_batch_use_graph(self.h, int(enable)))

    @property
    def launches_per_step(self) -> int:
        return int(lib().cel_batch_launches_per_step(self.h))

    def set_timestep(self, dt: np.ndarray):
        """Per-member time step from a float32 array (pinned memory makes the copy async)."""
        check(lib().cel_batch_set_timestep(self.h, C.cast(C.c_void_p(dt.ctypes.data if isinstance(dt, np.ndarray) else int(dt)), C.POINTER(C.c_float))))

    def step(self, n: int = 1):
        check(lib().cel_batch_step(self.h, n))

    def stats(self) -> list:
        """Statistics of each member at the start of the most recent step (fused into that step)."""
        arr = (Stats * self.n)()
        check(lib().cel_batch_stats(self.h, arr))
        return [arr[i].as_dict() for i in range(self.n)]

    def stats_current(self) -> list:
        """Statistics of each member's current state (an extra pass over the state)."""
        arr = (Stats * self.n)()
        check(lib().cel_batch_stats_current(self.h, arr))
        return [arr[i].as_dict() for i in range(self.n)]

    def state(self, i: int) -> np.ndarray:
        out = np.zeros(self.shapes[i] + (4,), dtype=np.float32)
        check(lib().cel_batch_get_state(self.h, i, _fp(out)))
        return out

    def state_parts(self, i: int):
        """Member i's state as (hi, lo) float textures; hi + lo is the compensated state (lo = 0 in
        the FP32 forms)."""
        hi = np.zeros(self.shapes[i] + (4,), dtype=np.float32)
        lo = np.zeros(self.shapes[i] + (4,), dtype=np.float32)
        check(lib().cel_batch_get_state_parts(self.h, i, _fp(hi), _fp(lo)))
        return hi, lo

    def set_state(self, i: int, rgba: np.ndarray):
        a = np.ascontiguousarray(rgba, dtype=np.float32)
        check(lib().cel_batch_set_state(self.h, i, _fp(a)))

    def aux(self, i: int) -> np.ndarray:
        out = np.zeros(self.shapes[i] + (4,), dtype=np.float32)
        check(lib().cel_batch_get_aux(self.h, i, _fp(out)))
        return out

    def add_solitary_wave(self, i: int, H: float, theta_deg: float, xc: float, yc: float):
        check(lib().cel_batch_add_solitary_wave(self.h, i, H, theta_deg, xc, yc))

    def set_bathymetry(self, i: int, z: np.ndarray):
        z = np.ascontiguousarray(z, dtype=np.float32)
        check(lib().cel_batch_set_bathymetry(self.h, i, _fp(z), z.shape[1], z.shape[0]))

    def set_tuning(self, band_width: int = 0, strip_height: int = 0, chunks: int = 0):
        """Column-solver band width (1/8/16/32), stencil strip height and the column solver's chunks
        per column (0 keeps the current value)."""
        check(lib().cel_batch_set_tuning(self.h, band_width, strip_height, chunks))

    @property
    def col_chunks(self) -> int:
        """Chunks per column of the column solver (rows per chunk = ceil(ny / chunks))."""
        return int(lib().cel_batch_col_chunks(self.h))

    @property
    def tuning(self) -> tuple:
        """(column band width, strip height)."""
        tx, ty, rp = C.c_int(), C.c_int(), C.c_int()
        check(lib().cel_batch_get_tuning(self.h, C.byref(tx), C.byref(ty), C.byref(rp)))
        return tx.value, ty.value

    @property
    def stencil_rows(self) -> int:
        tx, ty, rp = C.c_int(), C.c_int(), C.c_int()
        check(lib().cel_batch_get_tuning(self.h, C.byref(tx), C.byref(ty), C.byref(rp)))
        return rp.value

    def set_stencil_rows(self, rows_per_step: int):
        """1: one row per stencil step; 2: two rows as paired f32x2 arithmetic."""
        check(lib().cel_batch_set_stencil_rows(self.h, rows_per_step))

    @property
    def stencil_width(self) -> int:
        return int(lib().cel_batch_stencil_width(self.h))

    def set_stencil_width(self, threads: int):
        """Threads per stencil CTA (128 or 96; 96 with two rows per step)."""
        check(lib().cel_batch_set_stencil_width(self.h, threads))

    def autotune(self, steps: int = 5) -> dict:
        """Times each candidate for `steps` steps and keeps the fastest (the members advance)."""
        tx, ty, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib().cel_batch_autotune(self.h, steps, C.byref(tx), C.byref(ty), C.byref(ms)))
        return {"band_width": tx.value, "strip_height": ty.value, "ms_per_step": ms.value}

    def kernel_timing(self, enable: bool = True):
        check(lib().cel_batch_kernel_timing(self.h, int(enable)))

    def kernel_times(self) -> dict:
        return _kernel_times(self.h, 1)


def byte_model(form: str | int, correction_steps: int):
    f = FORMS[form] if isinstance(form, str) else int(form)
    a, b = C.c_double(), C.c_double()
    check(lib().cel_byte_model(f, correction_steps, C.byref(a), C.byref(b)))
    return a.value, b.value


# ---- file output in the reference's text formats (host side) ------------------------------------
def _texels(params: Params, a: np.ndarray, comps: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.shape != (params.ny + 4, params.nx + 4, comps):
        raise ValueError(f"expected a ({params.ny + 4}, {params.nx + 4}, {comps}) array, got {a.shape}")
    return a


def log_dump(params: Params, rgba: np.ndarray, total_time: float, elapsed: float = 0.0):
    """Appends the time axis, ranges and gauges of ``params.log`` for one state."""
    a = _texels(params, rgba, 4)
    check(lib().cel_log_dump(C.byref(params), _fp(a), total_time, elapsed))


def write_inundation(params: Params, aux: np.ndarray, path: str | None = None):
    a = _texels(params, aux, 4)
    check(lib().cel_write_inundation(C.byref(params), _fp(a), path.encode() if path else None))


def write_bathymetry(params: Params, bottom: np.ndarray, path: str | None = None):
    a = _texels(params, bottom, 3)
    check(lib().cel_write_bathymetry(C.byref(params), _fp(a), path.encode() if path else None))


def write_hotstart(params: Params, rgba: np.ndarray, path: str):
    a = _texels(params, rgba, 4)
    check(lib().cel_write_hotstart(C.byref(params), _fp(a), path.encode()))


def spectrum_waves(hs: float, tp: float, mean_theta_deg: float, depth: float, seed: int = 0,
                   gravity: float = 9.81, path: str | None = None) -> abi.Boundary:
    """Irregular-wave components of a directional spectrum (the reference's generateSpectrumWaves),
    as a boundary's wave table; set ``type``, ``width`` and ``sea_level`` on the result."""
    s = abi.Spectrum(hs, tp, mean_theta_deg, depth)
    b = abi.Boundary()
    check(lib().cel_spectrum_waves(C.byref(s), gravity, seed, C.byref(b), path.encode() if path else None))
    return b
