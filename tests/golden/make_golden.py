"""Writes the golden fixtures in this folder from the reference's own code.

Run in a tree where ``python oracle/ref_build.py`` has built ``oracle/_ref/`` from the reference
sources (compute.hlsl compiled as C++; terrain_heightfield.cpp and settings.cpp compiled as they
are).  Outputs:

* ``ref_states.npz``: for each case of ``golden_cases.NAMES``, the state, aux and statistics the
  reference's shader code gives after ``STEPS`` physical steps (plus, for ``mixed``, after a
  runtime solitary wave and 3 more steps).
* ``ref_bottom.npz``: the reference's BY/BX/BA for the seeded grid of ``bottom_case()`` read
  from a ``.cbf`` file, together with that grid.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), HERE]

from golden_cases import NAMES, STEPS, bottom_case, golden_case, write_cbf  # noqa: E402
from oracle import Oracle  # noqa: E402

STAT_KEYS = ["mass", "x_momentum", "y_momentum", "kinetic_energy", "potential_energy", "max_speed", "max_depth",
             "max_froude", "cfl_rate", "timestep", "total_time"]


def main() -> None:
    out = {}
    for name in NAMES:
        p, z, bnx, bny, keep = golden_case(name)
        ref = Oracle(p, z, bnx, bny, real="ref")
        s = ref.physical_steps(STEPS)
        out[f"{name}/state"] = ref.state().astype(np.float32)
        out[f"{name}/aux"] = ref.aux().astype(np.float32)
        out[f"{name}/stats"] = np.array([s[k] for k in STAT_KEYS])
        if name == "mixed":
            ref.add_solitary_wave(0.2, 30.0, 15.0, 10.0)
            ref.physical_steps(3)
            out[f"{name}/state_soliton"] = ref.state().astype(np.float32)
    out["stat_keys"] = np.array(STAT_KEYS)
    np.savez_compressed(os.path.join(HERE, "ref_states.npz"), **out)

    b = bottom_case()
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_host.so"))
    lib.ref_bottom.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.POINTER(C.c_float)]
    bot = np.zeros((b["ny"] + 4, b["nx"] + 4, 3), dtype=np.float32)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "grid.cbf")
        write_cbf(path, b["z"])
        lib.ref_bottom(path.encode(), b["nx"], b["ny"], b["width"], b["length"], b["swl"], b["gravity"],
                       bot.ctypes.data_as(C.POINTER(C.c_float)))
    np.savez_compressed(os.path.join(HERE, "ref_bottom.npz"), z=b["z"], bottom=bot)
    print("wrote", os.listdir(HERE))


if __name__ == "__main__":
    main()
