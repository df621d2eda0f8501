"""The oracle pinned to the reference's own code (CPU).

The fixtures in tests/golden/ were written by tests/golden/make_golden.py from the reference's
compute.hlsl compiled as C++ and its terrain_heightfield.cpp/settings.cpp compiled as they are
(oracle/ref_build.py).  The FP32 oracle must reproduce them bit for bit; the FP64 oracle must
stay within FP32 rounding of them.  When oracle/_ref/ is built in this tree, the live reference
build is compared too.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from golden_cases import NAMES, STEPS, bottom_case, golden_case, write_cbf  # noqa: E402

import celeris_b200 as cb  # noqa: E402
from celeris_b200 import abi  # noqa: E402
from oracle import Oracle  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "ref_states.npz"))
BOTTOM = np.load(os.path.join(HERE, "golden", "ref_bottom.npz"))
REF_SHADER = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_shader.so")


def _run(name, real):
    p, z, bnx, bny, keep = golden_case(name)
    o = Oracle(p, z, bnx, bny, real=real)
    s = o.physical_steps(STEPS)
    return o, s, keep


@pytest.mark.parametrize("name", NAMES)
def test_fp32_oracle_reproduces_reference_shader(name):
    o, s, _ = _run(name, "f32")
    np.testing.assert_array_equal(o.state().astype(np.float32), GOLD[f"{name}/state"])
    np.testing.assert_array_equal(o.aux().astype(np.float32), GOLD[f"{name}/aux"])
    keys = list(GOLD["stat_keys"])
    np.testing.assert_array_equal(np.array([s[k] for k in keys]), GOLD[f"{name}/stats"])
    if name == "mixed":
        o.add_solitary_wave(0.2, 30.0, 15.0, 10.0)
        o.physical_steps(3)
        np.testing.assert_array_equal(o.state().astype(np.float32), GOLD["mixed/state_soliton"])


@pytest.mark.parametrize("name", ["solid", "mixed", "irregular", "adaptive_manning"])
def test_fp64_oracle_close_to_reference_shader(name):
    o, _, _ = _run(name, "f64")
    ref = GOLD[f"{name}/state"].astype(np.float64)
    got = o.state()
    eta_rms = np.sqrt(np.mean((got[2:-2, 2:-2, 0] - ref[2:-2, 2:-2, 0]) ** 2))
    assert eta_rms < 1e-5, eta_rms                       # FP32 rounding over 20 steps
    scale = max(1e-3, np.abs(ref[2:-2, 2:-2, 1:3]).max())
    assert np.abs(got[2:-2, 2:-2, 1:3] - ref[2:-2, 2:-2, 1:3]).max() < 1e-4 * scale


def test_oracle_bottom_matches_reference_sampling():
    b = bottom_case()
    p = abi.default_params()
    p.nx, p.ny, p.width, p.length = b["nx"], b["ny"], b["width"], b["length"]
    for real in ("f32", "f64"):
        o = Oracle(p, b["z"], b["bnx"], b["bny"], real=real)
        np.testing.assert_array_equal(o.bottom().astype(np.float32), BOTTOM["bottom"])


def test_cbf_reader_reads_reference_layout(tmp_path, celeris):
    b = bottom_case()
    path = str(tmp_path / "grid.cbf")
    write_cbf(path, b["z"])
    np.testing.assert_array_equal(cb.read_cbf(path), BOTTOM["z"])


@pytest.mark.skipif(not os.path.exists(REF_SHADER), reason="oracle/_ref not built in this tree")
@pytest.mark.parametrize("name", ["mixed", "uts"])
def test_live_reference_build_matches_fixture(name):
    o, _, _ = _run(name, "ref")
    np.testing.assert_array_equal(o.state().astype(np.float32), GOLD[f"{name}/state"])


@pytest.mark.skipif(not os.path.exists(REF_SHADER), reason="oracle/_ref not built in this tree")
def test_terrain_change_matches_reference_shader():
    """After a mid-run newTerrainSettings the FP32 oracle and the reference's shader build step on
    identically (coefficients of the old bottom, new bottom textures, re-bootstrap)."""
    p, z, bnx, bny, keep = golden_case("mixed")
    ny, nx = z.shape
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
    z2 = (z + 1.0 * np.exp(-((X - 0.5 * nx) ** 2 + (Y - 0.5 * ny) ** 2) / (2 * (0.15 * nx) ** 2))).astype(np.float32)
    out = []
    for real in ("f32", "ref"):
        o = Oracle(p, z, bnx, bny, real=real)
        o.physical_steps(10)
        o.new_terrain(z2)
        o.physical_steps(10)
        out.append(o.state().astype(np.float32))
    np.testing.assert_array_equal(out[0], out[1])


# the reference's example inputs, copied next to its checkers by oracle/ref_build.py
EXAMPLES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "examples")


@pytest.mark.skipif(not (os.path.exists(REF_SHADER) and os.path.isdir(EXAMPLES)),
                    reason="oracle/_ref or the reference's example folder is not present")
def test_fp32_oracle_matches_reference_shader_on_the_reference_examples():
    """The reference's own example inputs (conical island, irregular and time-series wave-makers,
    the tutorial case, the flume), 8 physical steps: the FP32 oracle and the reference's shader
    build agree bit for bit."""
    import glob
    import celeris_b200 as cb
    ran = 0
    for path in sorted(glob.glob(os.path.join(EXAMPLES, "**", "*.cml"), recursive=True)):
        p = cb.params_from_cml(path)
        if not os.path.exists(p.bathymetry_path.decode()):
            continue
        z = cb.read_cbf(p.bathymetry_path.decode())
        states = []
        for real in ("f32", "ref"):
            o = Oracle(p, z, z.shape[1], z.shape[0], real=real)
            o.physical_steps(8)
            states.append(o.state().astype(np.float32))
        np.testing.assert_array_equal(states[0], states[1], err_msg=path)
        ran += 1
    assert ran >= 4
