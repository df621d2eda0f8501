"""Failure detection, injected from the host.

A non-finite value put into one member's state (through the public state upload) must come back
as CEL_ERR_NUMERIC in that member's statistics and in no other member's, while the other members
advance exactly as they would have without it.  A cell whose water level lies below its bed (a
negative depth) is a dry cell, as the reference's Pass3 clamps it (max(0, w - B)): it raises no
flag and the state stays finite.  No GPU fault is involved: the kernels only read the values.
"""
from __future__ import annotations

import numpy as np
import pytest

from celeris_b200 import cases

pytestmark = pytest.mark.gpu

CEL_ERR_NUMERIC = 5


def _members():
    return [cases.small_case(40 + 8 * i, 24 + 4 * i, k, correction_steps=1)
            for i, k in enumerate(["mixed", "sponge", "solid"])]


@pytest.mark.parametrize("form", ["plain", "fused", "mixed"])
def test_engine_reports_an_injected_nan(celeris, form):
    p, z, bnx, bny = _members()[0]
    e = celeris.Engine(p, z, form)
    e.physical_steps(5)
    assert e.reset_timestep()["health"] == 0
    s = e.state()
    s[12, 20, 1] = np.nan          # hu of one interior cell
    e.set_state(s)
    e.physical_steps(2)
    assert e.reset_timestep()["health"] == CEL_ERR_NUMERIC


@pytest.mark.parametrize("form", ["fused", "mixed"])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_flags_only_the_member_with_the_nan(celeris, form, graph):
    members = _members()
    clean = celeris.Batch([(m[0], m[1]) for m in members], form)
    hit = celeris.Batch([(m[0], m[1]) for m in members], form)
    for b in (clean, hit):
        b.use_graph(graph)
        b.step(5)
    s = hit.state(1)
    s[15, 22, 0] = np.inf          # w of one interior cell of member 1
    hit.set_state(1, s)
    clean.set_state(1, clean.state(1))   # the same upload path without the fault
    for b in (clean, hit):
        b.step(3)
    st = hit.stats_current()
    assert [x["health"] for x in st] == [0, CEL_ERR_NUMERIC, 0]
    assert [x["health"] for x in hit.stats()] == [0, CEL_ERR_NUMERIC, 0]   # the step's own totals
    for i in (0, 2):
        np.testing.assert_array_equal(hit.state(i), clean.state(i))
    assert all(x["health"] == 0 for x in clean.stats_current())


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_negative_depth_is_a_dry_cell(celeris, form):
    p, z, bnx, bny = _members()[1]
    e = celeris.Engine(p, z, form)
    e.physical_steps(5)
    s, bot = e.state(), e.bottom()
    y, x = 14, 20
    assert s[y, x, 0] - bot[y, x, 2] > 0.5          # a wet cell
    s[y, x, 0] = bot[y, x, 2] - 0.5                 # water level half a metre below the bed
    e.set_state(s)
    st = e.reset_timestep()
    assert st["health"] == 0
    e.physical_steps(20)
    assert e.reset_timestep()["health"] == 0
    assert np.isfinite(e.state()).all()
