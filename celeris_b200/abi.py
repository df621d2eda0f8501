"""ctypes mirror of include/celeris_b200.h (structs and the library loader).

The Python side is plumbing for tests and the benchmark: every computation runs in the
C++/CUDA library ``celeris_b200/_build/libceleris_b200.so`` behind the C ABI.  Loading fails
loudly if the library has not been built; there is no Python fallback.
"""
from __future__ import annotations

import ctypes as C
import os

CEL_MAX_WAVES = 1000
CEL_MAX_SOLITONS = 100
CEL_MAX_LOG_RANGES = 100
CEL_MAX_GAUGES = 1000

CEL_BC_SOLID, CEL_BC_SPONGE, CEL_BC_SINEWAVE, CEL_BC_IRREGULAR, CEL_BC_UTS = range(5)
CEL_FORM_PLAIN, CEL_FORM_FUSED, CEL_FORM_MIXED = 0, 1, 2
SCHEME_EULER, SCHEME_PREDICTOR, SCHEME_CORRECTOR, SCHEME_PREDICTOR_ADAPTIVE = range(4)

BC_NAMES = {"Solid": CEL_BC_SOLID, "Sponge": CEL_BC_SPONGE, "SineWave": CEL_BC_SINEWAVE,
            "IrregularWaves": CEL_BC_IRREGULAR, "UniformTimeSeries": CEL_BC_UTS}


class Boundary(C.Structure):
    _fields_ = [
        ("type", C.c_int),
        ("width", C.c_int),
        ("sea_level", C.c_double),
        ("amplitude", C.c_double),
        ("period", C.c_double),
        ("theta", C.c_double),
        ("n_waves", C.c_int),
        ("waves", (C.c_double * 4) * CEL_MAX_WAVES),
        ("n_uts", C.c_int),
        ("uts", C.POINTER(C.c_double)),
    ]


class Soliton(C.Structure):
    _fields_ = [("H", C.c_double), ("theta", C.c_double), ("xc", C.c_double),
                ("yc", C.c_double), ("length", C.c_double)]


class LogRange(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("x0", C.c_int), ("y0", C.c_int), ("x1", C.c_int), ("y1", C.c_int)]


class Log(C.Structure):
    _fields_ = [
        ("do_log", C.c_int), ("log_step", C.c_int),
        ("path", C.c_char * 1024), ("time_axis_name", C.c_char * 256), ("gauges_name", C.c_char * 256),
        ("n_ranges", C.c_int), ("ranges", LogRange * CEL_MAX_LOG_RANGES),
        ("n_gauges", C.c_int), ("gauges", (C.c_int * 2) * CEL_MAX_GAUGES),
    ]


class Params(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("width", C.c_double), ("length", C.c_double),
        ("still_water_elevation", C.c_double),
        ("boussinesq", C.c_int),
        ("epsilon", C.c_double), ("theta", C.c_double),
        ("correction_steps", C.c_int),
        ("timestep", C.c_double),
        ("adaptive", C.c_int),
        ("ema_alpha", C.c_double), ("min_timestep_ratio", C.c_double),
        ("manning", C.c_int), ("friction", C.c_double),
        ("gravity", C.c_double),
        ("dissipation_threshold", C.c_double), ("whitewater_decay", C.c_double),
        ("west", Boundary), ("east", Boundary), ("south", Boundary), ("north", Boundary),
        ("n_solitons", C.c_int),
        ("solitons", Soliton * CEL_MAX_SOLITONS),
        ("bathymetry_path", C.c_char * 1024),
        ("hotstart_path", C.c_char * 1024),
        ("project_name", C.c_char * 256),
        ("log", Log),
    ]


class Spectrum(C.Structure):
    _fields_ = [("significant_waveheight", C.c_double), ("peak_period", C.c_double),
                ("mean_theta", C.c_double), ("depth_at_source", C.c_double)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "mass", "x_momentum", "y_momentum", "kinetic_energy", "potential_energy", "total_energy",
        "max_speed", "max_depth", "max_froude", "cfl_rate", "cfl_number", "timestep", "total_time",
        "mass_full")] + [("time_scheme", C.c_int), ("health", C.c_int)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


def default_params() -> Params:
    """InitSetting defaults (reference settings.hpp:370-438) plus gravity 9.81."""
    p = Params()
    p.nx = p.ny = 100
    p.width = p.length = 100.0
    p.still_water_elevation = 0.0
    p.boussinesq = 1
    p.epsilon = 5e-8
    p.theta = 2.0
    p.correction_steps = 0
    p.timestep = 1e-4
    p.adaptive = 0
    p.ema_alpha = 0.5
    p.min_timestep_ratio = 0.05
    p.manning = 0
    p.friction = 0.0
    p.gravity = 9.81
    p.dissipation_threshold = 0.25
    p.whitewater_decay = 0.25
    for side in (p.west, p.east, p.south, p.north):
        side.type = CEL_BC_SOLID
        side.width = 2
    p.log.log_step = 100
    p.log.path = b"NA"
    p.log.time_axis_name = b"time_axis"
    p.log.gauges_name = b"gauges"
    return p


_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libceleris_b200.so")
_lib = None


def lib() -> C.CDLL:
    """Loads the CUDA library (raises if it is missing: no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"celeris_b200 library not built: {LIB_PATH} (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L: C.CDLL) -> None:
    vp = C.c_void_p
    i = C.c_int
    fp = C.POINTER(C.c_float)
    sig = {
        "cel_last_error": (C.c_char_p, []),
        "cel_version": (C.c_char_p, []),
        "cel_params_default": (i, [C.POINTER(Params)]),
        "cel_params_from_cml": (i, [C.c_char_p, C.POINTER(Params)]),
        "cel_read_irregular_waves": (i, [C.c_char_p, C.POINTER(Boundary)]),
        "cel_read_uts": (i, [C.c_char_p, C.POINTER(Boundary)]),
        "cel_params_release": (None, [C.POINTER(Params)]),
        "cel_params_size": (C.c_size_t, []),
        "cel_spectrum_waves": (i, [C.POINTER(Spectrum), C.c_double, C.c_ulonglong, C.POINTER(Boundary), C.c_char_p]),
        "cel_log_dump": (i, [C.POINTER(Params), fp, C.c_float, C.c_float]),
        "cel_write_inundation": (i, [C.POINTER(Params), fp, C.c_char_p]),
        "cel_write_bathymetry": (i, [C.POINTER(Params), fp, C.c_char_p]),
        "cel_write_hotstart": (i, [C.POINTER(Params), fp, C.c_char_p]),
        "cel_read_cbf": (i, [C.c_char_p, fp, C.c_size_t, C.POINTER(i), C.POINTER(i)]),
        "cel_create": (i, [C.POINTER(Params), fp, i, i, i, C.POINTER(vp)]),
        "cel_destroy": (i, [vp]),
        "cel_remesh": (i, [vp]),
        "cel_set_stream": (i, [vp, vp]),
        "cel_get_dims": (i, [vp, C.POINTER(i), C.POINTER(i)]),
        "cel_set_state": (i, [vp, fp]),
        "cel_get_state": (i, [vp, fp]),
        "cel_get_bottom": (i, [vp, fp]),
        "cel_get_aux": (i, [vp, fp]),
        "cel_reset_timestep": (i, [vp, C.c_float, C.c_float, C.POINTER(Stats)]),
        "cel_timestep": (i, [vp]),
        "cel_timesteps": (i, [vp, i]),
        "cel_physical_steps": (i, [vp, i]),
        "cel_get_stats": (i, [vp, C.POINTER(Stats)]),
        "cel_add_solitary_wave": (i, [vp, C.c_double, C.c_double, C.c_double, C.c_double]),
        "cel_get_water_height": (i, [vp, C.c_float, C.c_float, fp]),
        "cel_synchronize": (i, [vp]),
        "cel_set_bathymetry": (i, [vp, fp, i, i]),
        "cel_batch_set_bathymetry": (i, [vp, i, fp, i, i]),
        "cel_batch_add_solitary_wave": (i, [vp, i, C.c_double, C.c_double, C.c_double, C.c_double]),
        "cel_batch_create": (i, [i, C.POINTER(C.POINTER(Params)), C.POINTER(fp), C.POINTER(i),
                                 C.POINTER(i), i, C.POINTER(vp)]),
        "cel_batch_create_lanes": (i, [i, C.POINTER(C.POINTER(Params)), C.POINTER(fp), C.POINTER(i),
                                       C.POINTER(i), i, i, C.POINTER(vp)]),
        "cel_batch_lanes": (i, [vp]),
        "cel_batch_destroy": (i, [vp]),
        "cel_batch_set_stream": (i, [vp, vp]),
        "cel_batch_step": (i, [vp, i]),
        "cel_batch_stats": (i, [vp, C.POINTER(Stats)]),
        "cel_batch_stats_current": (i, [vp, C.POINTER(Stats)]),
        "cel_batch_get_tuning": (i, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "cel_batch_col_chunks": (i, [vp]),
        "cel_batch_set_stencil_rows": (i, [vp, i]),
        "cel_batch_set_stencil_width": (i, [vp, i]),
        "cel_batch_stencil_width": (i, [vp]),
        "cel_batch_autotune": (i, [vp, i, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]),
        "cel_batch_get_state": (i, [vp, i, fp]),
        "cel_batch_get_state_parts": (i, [vp, i, fp, fp]),
        "cel_batch_set_state": (i, [vp, i, fp]),
        "cel_batch_get_aux": (i, [vp, i, fp]),
        "cel_batch_use_graph": (i, [vp, i]),
        "cel_batch_cells": (C.c_longlong, [vp]),
        "cel_batch_set_timestep": (i, [vp, fp]),
        "cel_batch_launches_per_step": (i, [vp]),
        "cel_set_tuning": (i, [vp, i, i, i]),
        "cel_batch_set_tuning": (i, [vp, i, i, i]),
        "cel_batch_kernel_timing": (i, [vp, i]),
        "cel_engine_kernel_timing": (i, [vp, i]),
        "cel_kernel_times": (i, [vp, i, C.POINTER(C.c_char * 64), C.POINTER(C.c_double),
                                 C.POINTER(C.c_longlong), i, C.POINTER(i)]),
        "cel_byte_model": (i, [i, i, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "cel_selftest_reciprocal": (i, [C.POINTER(C.c_float), C.POINTER(C.c_float), i]),
        "cel_stats_noalloc": (i, [vp, vp, C.POINTER(Params), vp, C.POINTER(Stats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


class CelError(RuntimeError):
    pass


def check(status: int) -> None:
    if status != 0:
        msg = lib().cel_last_error()
        raise CelError(f"celeris_b200 error {status}: {msg.decode() if msg else ''}")


# Exported symbol list of include/celeris_b200.h (checked by the CPU test suite)
EXPORTED = [
    "cel_last_error", "cel_version", "cel_params_default", "cel_params_from_cml",
    "cel_read_irregular_waves", "cel_read_uts", "cel_params_release", "cel_params_size", "cel_read_cbf",
    "cel_log_dump", "cel_write_inundation", "cel_write_bathymetry", "cel_write_hotstart", "cel_spectrum_waves",
    "cel_create", "cel_destroy", "cel_remesh", "cel_set_stream", "cel_get_dims",
    "cel_set_state", "cel_get_state", "cel_get_bottom", "cel_get_aux",
    "cel_reset_timestep", "cel_timestep", "cel_timesteps", "cel_physical_steps", "cel_get_stats",
    "cel_add_solitary_wave", "cel_get_water_height", "cel_synchronize", "cel_set_bathymetry",
    "cel_batch_set_bathymetry", "cel_batch_add_solitary_wave",
    "cel_batch_create", "cel_batch_create_lanes", "cel_batch_lanes", "cel_batch_destroy", "cel_batch_set_stream",
    "cel_batch_step",
    "cel_batch_stats", "cel_batch_stats_current", "cel_batch_get_state", "cel_batch_get_state_parts", "cel_batch_set_state", "cel_batch_get_aux",
    "cel_batch_use_graph", "cel_batch_cells", "cel_batch_set_timestep", "cel_batch_launches_per_step", "cel_set_tuning", "cel_batch_set_tuning",
    "cel_batch_get_tuning", "cel_batch_col_chunks", "cel_batch_set_stencil_rows", "cel_batch_set_stencil_width", "cel_batch_stencil_width",
    "cel_batch_autotune",
    "cel_batch_kernel_timing", "cel_engine_kernel_timing", "cel_kernel_times", "cel_byte_model", "cel_selftest_reciprocal", "cel_stats_noalloc",
]
