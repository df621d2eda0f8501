"""CPU-side checks of the C-ABI library: it loads, exports every symbol declared in
include/celeris_b200.h, parses settings, and refuses to run without a GPU (no CPU fallback)."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from celeris_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "celeris_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const char\*|int|void|long long|size_t)\s+(cel_\w+)\s*\(", txt, re.M)))


def test_header_symbol_list_matches_binding():
    assert header_symbols() == sorted(abi.EXPORTED)


def test_library_exports_every_symbol(celeris):
    L = celeris.lib()
    for name in header_symbols():
        assert hasattr(L, name), name


def test_no_device_is_an_error_not_a_fallback(celeris):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from celeris_b200 import cases
    p, z, bnx, bny = cases.small_case(16, 12, "solid")
    with pytest.raises(celeris.CelError):
        celeris.Engine(p, z, "plain")


def test_defaults_match_initsetting(celeris):
    p = abi.Params()
    assert celeris.lib().cel_params_default(C.byref(p)) == 0
    assert (p.nx, p.ny, p.width, p.length) == (100, 100, 100.0, 100.0)
    assert p.boussinesq == 1 and p.epsilon == 5e-8 and p.theta == 2 and p.timestep == 1e-4
    assert p.west.type == abi.CEL_BC_SOLID and p.west.width == 2


CML = """<?xml version="1.0" ?>
<Experiment>
  <name>unit test case</name>
  <!-- comment with <tags> inside -->
  <model type = "BSNQ">
    <parameters epsilon = 5e-12 Theta = 1.5 correctionStepsNum = 2 timestep = 0.005></parameters>
    <friction type = "Manning" coef = 0.02></friction>
  </model>
  <fieldDimensions width = 200 length = 5 stillWaterElevation = 0.25></fieldDimensions>
  <gridSize nx = 160 ny = 9></gridSize>
  <bathymetryFilePath> bathy.cbf </bathymetryFilePath>
  <hotStartFilePath> N/A </hotStartFilePath>
  <solitaryWave H = 0.05 theta = 30 xc = 45 yc = 2 ></solitaryWave>
  <solitaryWave H = 0.02 theta = 0 xc = 10 yc = 2 length = 3></solitaryWave>
  <westBoundary type = "SineWave" seaLevel = 0 widthNum = 2>
    <sineWave amplitude = 0.1 period = 8 theta = 10></sineWave>
  </westBoundary>
  <eastBoundary  type = "Sponge" seaLevel = 0.1 widthNum = 40></eastBoundary>
  <southBoundary type = "IrregularWaves" seaLevel = 0 widthNum = 2>
    <filePath> waves.txt </filePath>
  </southBoundary>
  <northBoundary type = "UniformTimeSeries" seaLevel = 0 widthNum = 2>
    <filePath>uts.txt</filePath>
  </northBoundary>
  <graphics><surfaceShading type = 2><dissipationIntensity show = true threshold = 0.3 decay = 0.2></dissipationIntensity></surfaceShading></graphics>
</Experiment>
"""


def test_cml_parser(tmp_path, celeris):
    (tmp_path / "case.cml").write_text(CML)
    (tmp_path / "waves.txt").write_text("# header\n[NumberOfWaves] 2\n=====\n0.04 2 .785 0.0\n0.03 3 -.785 1.5\n")
    (tmp_path / "uts.txt").write_text("comment\n====\n0 0 0 0\n1 0.1 0.2 0.3\n2 0 0 0\n")
    z = np.arange(12, dtype=np.float32).reshape(3, 4)
    with open(tmp_path / "bathy.cbf", "w") as f:
        f.write("[nx] 4\n[ny] 3\n\n====\n")
        for row in z:
            f.write(" ".join(f"{v:.3f}" for v in row) + "\n")
    p = celeris.params_from_cml(str(tmp_path / "case.cml"))
    assert (p.nx, p.ny, p.width, p.length, p.still_water_elevation) == (160, 9, 200.0, 5.0, 0.25)
    assert p.epsilon == 5e-12 and p.theta == 1.5 and p.correction_steps == 2 and p.timestep == 0.005
    assert p.manning == 1 and p.friction == 0.02 and p.boussinesq == 1
    assert p.n_solitons == 2 and abs(p.solitons[0].theta - np.pi / 6) < 1e-12 and p.solitons[0].length == 1e30
    assert p.solitons[1].length == 3
    assert p.west.type == abi.CEL_BC_SINEWAVE and abs(p.west.theta - np.pi / 18) < 1e-12 and p.west.period == 8
    assert p.east.type == abi.CEL_BC_SPONGE and p.east.width == 40 and p.east.sea_level == 0.1
    assert p.south.type == abi.CEL_BC_IRREGULAR and p.south.n_waves == 2 and p.south.waves[1][3] == 1.5
    assert p.north.type == abi.CEL_BC_UTS and p.north.n_uts == 3 and p.north.uts[5] == 0.1
    assert p.dissipation_threshold == 0.3 and p.whitewater_decay == 0.2
    assert p.bathymetry_path.decode().endswith("bathy.cbf")
    np.testing.assert_array_equal(celeris.read_cbf(p.bathymetry_path.decode()), z.round(3))
    celeris.lib().cel_params_release(C.byref(p))


def test_cml_errors(tmp_path, celeris):
    (tmp_path / "bad.cml").write_text("<Experiment><gridSize nx = 10 ny = 10></Experiment>")
    with pytest.raises(celeris.CelError):
        celeris.params_from_cml(str(tmp_path / "bad.cml"))
    with pytest.raises(celeris.CelError):
        celeris.params_from_cml(str(tmp_path / "missing.cml"))
    (tmp_path / "bt.cml").write_text('<E><westBoundary type = "Wall" widthNum = 2></westBoundary></E>')
    with pytest.raises(celeris.CelError):
        celeris.params_from_cml(str(tmp_path / "bt.cml"))


def test_byte_model(celeris):
    # the paired-row stencil reads the corner grid (4 B) instead of BA, BX, BY (12 B)
    s, t = celeris.byte_model("fused", 1)
    assert s == 104 and t == (104 + 48) + (128 + 48)
    s2, t2 = celeris.byte_model("mixed", 1)
    assert s2 == 112 and t2 == (112 + 64) + (136 + 64)


def test_new_entry_points_refuse_null_handles(celeris):
    """Argument checks come before any device work, so they hold on a machine without a GPU."""
    L = celeris.lib()
    z = (C.c_float * 16)()
    f = C.c_float()
    assert L.cel_set_bathymetry(None, z, 4, 4) == 1
    assert L.cel_batch_set_bathymetry(None, 0, z, 4, 4) == 1
    assert L.cel_batch_add_solitary_wave(None, 0, 0.1, 0.0, 1.0, 1.0) == 1
    assert L.cel_get_water_height(None, 0.0, 0.0, C.byref(f)) == 1
    assert L.cel_batch_set_stencil_width(None, 96) == 1
    assert L.cel_batch_stencil_width(None) == 0
    assert L.cel_spectrum_waves(None, 9.81, 0, None, None) == 1
    assert L.cel_log_dump(None, None, 0.0, 0.0) == 1
    assert L.cel_write_hotstart(None, None, None) == 1
    assert L.cel_batch_lanes(None) == 0
    # a negative lane count is refused before any device work
    p = abi.Params()
    assert L.cel_params_default(C.byref(p)) == 0
    pp = (C.POINTER(abi.Params) * 1)(C.pointer(p))
    zz = (C.POINTER(C.c_float) * 1)(C.cast(z, C.POINTER(C.c_float)))
    dims = (C.c_int * 1)(4)
    h = C.c_void_p()
    assert L.cel_batch_create_lanes(1, pp, zz, dims, dims, 2, -1, C.byref(h)) == 1
    assert b"lanes" in L.cel_last_error()


# the reference's example inputs, copied next to its checkers by oracle/ref_build.py
EXAMPLES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "examples")


@pytest.mark.skipif(not os.path.isdir(EXAMPLES), reason="the reference's example folder is not present")
def test_reference_example_inputs_parse(celeris):
    """Every .cml the reference ships parses, with the files it names (.cbf grids, irregular-wave
    components, time series) read where they exist."""
    import glob
    seen = {}
    for path in sorted(glob.glob(os.path.join(EXAMPLES, "**", "*.cml"), recursive=True)):
        p = celeris.params_from_cml(path)
        assert p.nx >= 2 and p.ny >= 2 and p.width > 0 and p.length > 0, path
        bp = p.bathymetry_path.decode()
        if os.path.exists(bp):
            z = celeris.read_cbf(bp)
            assert z.size > 0 and np.isfinite(z).all(), bp
        seen[os.path.basename(path)] = p
    assert len(seen) >= 5
    irr = seen.get("conical_island - irregular.cml")
    if irr is not None:
        assert irr.west.type == abi.CEL_BC_IRREGULAR and irr.west.n_waves > 0
    uts = seen.get("conical_island - UniformTimeSeries.cml")
    if uts is not None:
        assert uts.west.type == abi.CEL_BC_UTS and uts.west.n_uts > 1
    ready = seen.get("conical_island_ready.cml")
    if ready is not None:
        assert ready.log.do_log == 1 and ready.log.n_gauges == 5 and ready.log.n_ranges == 2


def test_cpp_engine_adapter_compiles_and_links(tmp_path, celeris):
    """include/celeris_b200_engine.hpp, the ShallowWaterEngine stand-in a host program includes,
    compiles against the C header and links the built library.  Without a GPU, creating an engine
    throws the library's message as a C++ exception; with one, the engine is created."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(abi.LIB_PATH)
    (tmp_path / "case.cml").write_text("<E><gridSize nx = 4 ny = 4></gridSize></E>")
    (tmp_path / "host.cpp").write_text(r"""
#include "celeris_b200_engine.hpp"
#include <cstdio>
int main(int argc, char** argv) {
    std::vector<float> z(16, -1.0f);
    try {
        CelerisB200Engine e(argv[1], z, 4, 4);
        std::printf("created %d\n", e.params().nx);
    } catch (const std::exception& ex) {
        std::printf("error: %s\n", ex.what());
    }
    std::printf("version %s\n", cel_version());
    return 0;
}
""")
    exe = tmp_path / "host"
    cmd = [gxx, "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(root, "include"), str(tmp_path / "host.cpp"),
           "-L", libdir, "-lceleris_b200", "-Wl,-rpath," + libdir, "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe), str(tmp_path / "case.cml")], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    assert lines[0] == "created 4" or lines[0].startswith("error: "), lines
    assert lines[-1].startswith("version ")
