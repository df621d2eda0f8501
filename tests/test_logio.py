"""File output in the reference's text formats, checked on the CPU through the C ABI.

Covers the <logData> parser (main.cpp:825-887), the time-axis / range / gauge dump
(engine.cpp:628-675), the inundation map (engine.cpp:781-817), the bathymetry grid
(engine.cpp:750-779) and hot-start files (read by engine.cpp:2943-2966).  The expected text is
built here with C's %g rules (6 significant digits), which is what the reference's ofstream writes
for a float.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from celeris_b200 import abi


def g6(v) -> str:
    return "%g" % float(np.float32(v))


CML = """<?xml version="1.0" ?>
<Experiment>
  <gridSize nx = 20 ny = 12></gridSize>
  <logData doLog = true logStep = 20>
    <logPath>log/</logPath>
    <timeAxis filename = "t_axis"></timeAxis>
    <range filename = "island">
      <bottomLeft x = 3 y = 4></bottomLeft>
      <topRight x = 6 y = 5></topRight>
    </range>
    <range filename = "centerline">
      <bottomLeft x = 0 y = 8></bottomLeft>
      <topRight x = 23 y = 8></topRight>
    </range>
    <gauges filename = "gauges">
      2,2,
      5,7,
      23,15
    </gauges>
  </logData>
</Experiment>
"""


def parse(tmp_path, text, name="case.cml"):
    import celeris_b200 as cb
    (tmp_path / name).write_text(text)
    return cb.params_from_cml(str(tmp_path / name))


def test_params_struct_size_matches_binding(celeris):
    assert celeris.lib().cel_params_size() == C.sizeof(abi.Params)


def test_log_defaults(celeris):
    p = abi.Params()
    assert celeris.lib().cel_params_default(C.byref(p)) == 0
    assert p.log.do_log == 0 and p.log.log_step == 100
    assert (p.log.path, p.log.time_axis_name, p.log.gauges_name) == (b"NA", b"time_axis", b"gauges")
    assert p.log.n_ranges == 0 and p.log.n_gauges == 0


def test_logdata_parsed(tmp_path, celeris):
    p = parse(tmp_path, CML)
    lg = p.log
    assert lg.do_log == 1 and lg.log_step == 20
    assert lg.path.decode() == str(tmp_path) + "/log/"
    assert lg.time_axis_name == b"t_axis" and lg.gauges_name == b"gauges"
    assert lg.n_ranges == 2
    r0, r1 = lg.ranges[0], lg.ranges[1]
    assert (r0.name, r0.x0, r0.y0, r0.x1, r0.y1) == (b"island", 3, 4, 6, 5)
    assert (r1.name, r1.x0, r1.y0, r1.x1, r1.y1) == (b"centerline", 0, 8, 23, 8)
    assert [tuple(lg.gauges[k]) for k in range(lg.n_gauges)] == [(2, 2), (5, 7), (23, 15)]


@pytest.mark.parametrize("text, pairs", [
    ("1,2,3,4", [(1, 2), (3, 4)]),
    # a trailing comma: the round that fails keeps the previous pair (main.cpp:866-876)
    ("1,2,3,4,", [(1, 2), (3, 4), (3, 4)]),
    # a missing comma: the separator read takes the first digit of the next number
    ("5,7,\n19,15\n66,14", [(5, 7), (19, 15), (6, 14)]),
    ("  ", []),
])
def test_gauge_list_stream_semantics(tmp_path, celeris, text, pairs):
    p = parse(tmp_path, f"<E><gridSize nx = 70 ny = 20></gridSize><logData doLog = false logStep = 1>"
                        f"<gauges filename = \"g\">{text}</gauges></logData></E>")
    assert [tuple(p.log.gauges[k]) for k in range(p.log.n_gauges)] == pairs


def test_empty_log_path_is_the_cml_folder(tmp_path, celeris):
    p = parse(tmp_path, "<E><logData doLog = true logStep = 5><logPath> </logPath></logData></E>")
    assert p.log.path.decode() == str(tmp_path)
    assert p.log.do_log == 1 and p.log.log_step == 5


def make_state(p, seed=0):
    rng = np.random.default_rng(seed)
    s = rng.normal(0, 1, (p.ny + 4, p.nx + 4, 4)).astype(np.float32)
    s[2, 2, :] = [1e-5, -0.0, 123456789.0, 0.1]   # exponent form, negative zero, rounding (gauge 2,2)
    return s


def test_log_dump_writes_the_reference_format(tmp_path, celeris):
    p = parse(tmp_path, CML)
    os.makedirs(p.log.path.decode(), exist_ok=True)
    s1, s2 = make_state(p, 1), make_state(p, 2)
    celeris.log_dump(p, s1, 0.125, 3.5)
    celeris.log_dump(p, s2, np.float32(0.1) * 3, 7.25)      # appends
    d = p.log.path.decode() + "/"
    assert open(d + "t_axis.txt").read() == f"0.125\n{g6(np.float32(0.1) * 3)}\n"
    assert open(d + "t_axis-elapsed.txt").read() == "3.5\n7.25\n"

    def lines(s, pts):
        return "".join(f"{i}\t{j}\t" + "\t".join(g6(v) for v in s[j, i]) + "\n" for i, j in pts)

    island = [(i, j) for j in (4, 5) for i in range(3, 7)]
    center = [(i, 8) for i in range(24)]
    gauges = [(2, 2), (5, 7), (23, 15)]
    assert open(d + "island.txt").read() == lines(s1, island) + lines(s2, island)
    assert open(d + "centerline.txt").read() == lines(s1, center) + lines(s2, center)
    assert open(d + "gauges.txt").read() == lines(s1, gauges) + lines(s2, gauges)
    assert open(d + "gauges.txt").read().startswith("2\t2\t1e-05\t-0\t1.23457e+08\t0.1\n")


def test_log_dump_refuses_points_outside_the_texture(tmp_path, celeris):
    p = parse(tmp_path, CML)
    p.log.gauges[2][0] = p.nx + 4          # one past the last texel column
    with pytest.raises(celeris.CelError, match="outside"):
        celeris.log_dump(p, make_state(p), 0.0)
    p = parse(tmp_path, CML)
    p.log.ranges[1].x1 = p.nx + 4
    with pytest.raises(celeris.CelError, match="centerline"):
        celeris.log_dump(p, make_state(p), 0.0)
    p = parse(tmp_path, CML)
    p.log.log_step = 0
    with pytest.raises(celeris.CelError, match="logStep"):
        celeris.log_dump(p, make_state(p), 0.0)


def test_log_dump_reports_an_unwritable_folder(tmp_path, celeris):
    p = parse(tmp_path, CML)              # the log/ folder is not created
    with pytest.raises(celeris.CelError, match="cannot open"):
        celeris.log_dump(p, make_state(p), 0.0)


def test_inundation_map_format(tmp_path, celeris):
    p = parse(tmp_path, CML)
    aux = make_state(p, 3)
    path = tmp_path / "inund.txt"
    celeris.write_inundation(p, aux, str(path))
    txt = path.read_text()
    head = ("[nx] 20\n[ny] 12\n\n\n# This file contains the maximum depth of inundation on each point, in meters."
            "\n\n====================================\n")
    assert txt.startswith(head)
    rows = txt[len(head):].split("\n")[:-1]
    assert len(rows) == p.ny
    for j, row in zip(range(2, p.ny + 2), rows):
        # columns 2..nx+2 inclusive, each followed by a tab (engine.cpp:808-814)
        assert row == "".join(g6(aux[j, i, 0]) + "\t" for i in range(2, p.nx + 3))


def test_inundation_default_name_is_timestamped(tmp_path, celeris):
    p = parse(tmp_path, CML)
    os.makedirs(p.log.path.decode(), exist_ok=True)
    celeris.write_inundation(p, make_state(p))
    names = os.listdir(p.log.path.decode())
    assert len(names) == 1 and names[0].endswith("-inundation.txt") and names[0].count("-") == 5


def test_bathymetry_file_reads_back(tmp_path, celeris):
    p = parse(tmp_path, CML)
    b3 = np.random.default_rng(4).uniform(-2, 1, (p.ny + 4, p.nx + 4, 3)).astype(np.float32)
    path = tmp_path / "dump.cbf"
    celeris.write_bathymetry(p, b3, str(path))
    z = celeris.read_cbf(str(path))
    assert z.shape == (p.ny, p.nx)
    want = np.array([[float(g6(v)) for v in row] for row in b3[2:-2, 2:-2, 2]], dtype=np.float32)
    np.testing.assert_array_equal(z, want)


def test_hotstart_file_keeps_every_bit(tmp_path, celeris):
    p = parse(tmp_path, CML)
    s = make_state(p, 5)
    path = tmp_path / "hot.txt"
    celeris.write_hotstart(p, s, str(path))
    rows = np.loadtxt(path, dtype=np.float64)
    assert rows.shape == ((p.nx + 4) * (p.ny + 4), 6)
    jj, ii = np.meshgrid(np.arange(p.ny + 4), np.arange(p.nx + 4), indexing="ij")
    np.testing.assert_array_equal(rows[:, 0], ii.ravel())
    np.testing.assert_array_equal(rows[:, 1], jj.ravel())
    back = rows[:, 2:].astype(np.float32).reshape(p.ny + 4, p.nx + 4, 4)
    np.testing.assert_array_equal(back.view(np.uint32), s.view(np.uint32))
