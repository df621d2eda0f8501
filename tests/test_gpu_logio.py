"""Logging while stepping, and hot starts, on the GPU.

Engines and batch members with <logData> doLog set write the time axis, ranges and gauges after
every logStep-th physical step, as the reference's timestep() does (engine.cpp:1488-1493).  The
files are compared with the text the same writer gives for the state of a second, silent run
after the same number of steps.  A hot-start file written from a stepped state must start a new
engine in exactly that state.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from celeris_b200 import cases

pytestmark = pytest.mark.gpu

STEPS, EVERY = 7, 3


def g6(v) -> str:
    return "%g" % float(np.float32(v))


def set_log(p, folder, every):
    p.log.do_log, p.log.log_step = 1, every
    p.log.path = folder.encode()
    p.log.n_ranges = 1
    r = p.log.ranges[0]
    r.name, r.x0, r.y0, r.x1, r.y1 = b"strip", 0, 9, p.nx + 3, 9
    p.log.n_gauges = 3
    for k, (x, y) in enumerate([(2, 2), (10, 7), (p.nx + 1, p.ny + 1)]):
        p.log.gauges[k][0], p.log.gauges[k][1] = x, y


def expected_lines(s, pts):
    return "".join(f"{i}\t{j}\t" + "\t".join(g6(v) for v in s[j, i]) + "\n" for i, j in pts)


def check_folder(folder, p, states, times):
    pts_r = [(i, 9) for i in range(p.nx + 4)]
    pts_g = [(2, 2), (10, 7), (p.nx + 1, p.ny + 1)]
    assert open(os.path.join(folder, "strip.txt")).read() == "".join(expected_lines(s, pts_r) for s in states)
    assert open(os.path.join(folder, "gauges.txt")).read() == "".join(expected_lines(s, pts_g) for s in states)
    assert open(os.path.join(folder, "time_axis.txt")).read() == "".join(g6(t) + "\n" for t in times)
    el = open(os.path.join(folder, "time_axis-elapsed.txt")).read().split()
    assert len(el) == len(states) and all(float(v) >= 0 for v in el)


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_engine_logs_every_log_step(tmp_path, celeris, form):
    p, z, _, _ = cases.small_case(48, 20, "sponge")
    silent = celeris.Engine(p, z, form)
    states = []
    for s in range(1, STEPS + 1):
        silent.physical_steps(1)
        if s % EVERY == 0:
            states.append(silent.state())
    set_log(p, str(tmp_path), EVERY)
    eng = celeris.Engine(p, z, form)
    eng.physical_steps(STEPS)
    dt = np.float32(p.timestep)
    if form == "plain":        # float clock, as the reference's total_time
        t, times = np.float32(0), []
        for s in range(1, STEPS + 1):
            if s % EVERY == 0:
                times.append(t)
            t = np.float32(t + dt)
    else:                      # FP64 clock rounded to float
        times = [np.float32((s - 1) * np.float64(dt)) for s in range(1, STEPS + 1) if s % EVERY == 0]
    check_folder(str(tmp_path), p, states, times)


def test_batch_member_logs_on_its_own_schedule(tmp_path, celeris):
    pa, za, _, _ = cases.small_case(48, 20, "sponge")
    pb, zb, _, _ = cases.small_case(40, 24, "solid")
    silent = celeris.Batch([(pa, za), (pb, zb)], "mixed")
    silent.use_graph(True)
    states = []
    for s in range(1, STEPS + 1):
        silent.step(1)
        if s % 2 == 0:
            states.append(silent.state(0))
    set_log(pa, str(tmp_path), 2)
    b = celeris.Batch([(pa, za), (pb, zb)], "mixed")
    b.use_graph(True)
    b.step(STEPS)
    dt = np.float32(pa.timestep)
    times = [np.float32((s - 1) * np.float64(dt)) for s in range(1, STEPS + 1) if s % 2 == 0]
    check_folder(str(tmp_path), pa, states, times)
    np.testing.assert_array_equal(b.state(1), silent.state(1))


def test_engine_creation_rejects_a_gauge_outside_the_texture(tmp_path, celeris):
    p, z, _, _ = cases.small_case(48, 20, "sponge")
    set_log(p, str(tmp_path), 2)
    p.log.gauges[1][1] = p.ny + 4
    for form in ("plain", "fused"):
        with pytest.raises(celeris.CelError, match="gauge"):
            celeris.Engine(p, z, form)


@pytest.mark.parametrize("form", ["plain", "fused", "mixed"])
def test_hotstart_round_trip(tmp_path, celeris, form):
    p, z, _, _ = cases.small_case(48, 20, "sponge")
    a = celeris.Engine(p, z, form)
    a.physical_steps(25)
    s = a.state()
    path = str(tmp_path / "hot.txt")
    celeris.write_hotstart(p, s, path)
    p.hotstart_path = path.encode()
    b = celeris.Engine(p, z, form)
    got = b.state()
    # equal values (the mixed form keeps -0 as hi + lo = -0 + +0, which reads back as +0)
    np.testing.assert_array_equal(got[..., :3], s[..., :3])
