"""Writes ``ref_spectrum.npz``: the reference's own spectrum wave-maker (engine.cpp:3559-3776,
generateSpectrumWaves, built by ``python oracle/ref_build.py`` into oracle/_ref/libref_spectrum.so)
run on the settings of ``CASES``, as it writes its component file (six significant digits per
value).  Each case stores the file's rows {amplitude, period, theta (rad), phase}; the phases come
from the C library's rand() seeded with 1, which the product does not reproduce (it draws seeded
phases of its own), so tests compare the other three columns and the phase quantisation.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_spectrum.so")

# (significant wave height m, peak period s, mean direction deg, depth at source m)
CASES = [(1.0, 10.0, 0.0, 15.0), (2.5, 14.0, 12.5, 20.0), (0.4, 6.0, -30.0, 3.0), (3.0, 8.0, 0.0, 4.0),
         (0.8, 5.0, 45.0, 10.0), (1.5, 12.0, -7.5, 2.0)]
GRAVITY = 9.81


def reference_rows(lib, hs, tp, th, h, seed=1) -> np.ndarray:
    lib.ref_spectrum_file.argtypes = [C.c_double] * 5 + [C.c_uint, C.c_char_p, C.c_char_p, C.c_int]
    d = tempfile.mkdtemp()
    buf = C.create_string_buffer(4096)
    if lib.ref_spectrum_file(hs, tp, th, h, GRAVITY, seed, d.encode(), buf, 4096) != 0:
        raise RuntimeError("reference generator refused the case")
    rows, started = [], False
    with open(buf.value.decode()) as f:
        for line in f:
            if line.startswith("===="):
                started = True
            elif started and line.strip():
                rows.append([float(x) for x in line.split()])
    return np.array(rows, dtype=np.float64)


def main() -> None:
    if not os.path.exists(LIB):
        sys.exit("oracle/_ref/libref_spectrum.so is not built (python oracle/ref_build.py)")
    lib = C.CDLL(LIB)
    out = {"cases": np.array(CASES, dtype=np.float64)}
    for k, case in enumerate(CASES):
        out[f"case{k}"] = reference_rows(lib, *case)
    np.savez_compressed(os.path.join(HERE, "ref_spectrum.npz"), **out)
    print(f"wrote {len(CASES)} cases")


if __name__ == "__main__":
    main()
