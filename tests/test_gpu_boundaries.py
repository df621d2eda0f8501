"""GPU parity of the boundary strips in the cases the small mixes do not reach.

* a side where one batch member has a solid strip 3 cells wide (so the whole side runs in two
  phases: compute into scratch, then copy back) and another member an irregular wave-maker;
* an irregular wave-maker of 100 components (more than one per lane of the warp-split sum);
* the compensated form's strips: sponge, sine and irregular values are evaluated in FP64 and kept
  as a float pair; its water volume follows the FP64 oracle on open-boundary cases closer than the
  FP32 form's.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from celeris_b200 import abi, cases
from util import eta_rms, field_errors, rel_ok

pytestmark = pytest.mark.gpu


def _solid3_west(nx=48, ny=30):
    p, z, bnx, bny = cases.small_case(nx, ny, "solid", correction_steps=1)
    p.west.type, p.west.width = abi.CEL_BC_SOLID, 3
    return p, z, bnx, bny


def _irregular_west(nx=56, ny=36, n_waves=8, seed=1):
    p, z, bnx, bny = cases.small_case(nx, ny, "irregular", seed=seed, correction_steps=1)
    if n_waves != p.west.n_waves:
        comps = cases.jonswap_components(n_waves, 0.4, 6.0, 3.3, np.random.default_rng(99))
        p.west.n_waves = n_waves
        for i in range(n_waves):
            for k in range(4):
                p.west.waves[i][k] = float(comps[i, k])
    return p, z, bnx, bny


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_two_phase_side_with_a_wavemaker_member(celeris, form):
    """One lane holds a member whose west wall is 3 cells wide (two-phase west side) and a member
    with an irregular wave-maker on the west: the wave-maker's cells go through the scratch strip
    and come back unchanged, so the batch equals the members stepped alone."""
    members = [_solid3_west(), _irregular_west()]
    batch = celeris.Batch([(m[0], m[1]) for m in members], form, lanes=1)
    batch.use_graph(True)
    batch.step(25)
    for i, (p, z, bnx, bny) in enumerate(members):
        e = celeris.Engine(p, z, form)
        e.physical_steps(25)
        np.testing.assert_array_equal(batch.state(i), e.state())
    # and the wave-maker member against the FP64 oracle
    p, z, bnx, bny = members[1]
    ref = O.Oracle(p, z, bnx, bny, "f64")
    ref.physical_steps(25)
    assert eta_rms(batch.state(1), ref.state()) <= 1e-4


def test_many_component_wavemaker(celeris):
    """100 components on a 130-row west side (the reference's tree has 128 leaves): the plain form
    bit for bit against the FP32 transcription; the fused forms against the FP64 oracle, in the
    interior and on the wave-maker strip itself."""
    p, z, bnx, bny = _irregular_west(nx=60, ny=130, n_waves=100)
    r32 = O.Oracle(p, z, bnx, bny, "f32")
    r64 = O.Oracle(p, z, bnx, bny, "f64")
    eng = celeris.Engine(p, z, "plain")
    r32.physical_steps(30)
    r64.physical_steps(30)
    eng.physical_steps(30)
    a, b = eng.state(), r32.state()
    assert np.array_equal(a[..., :3].astype(np.float64), b[..., :3]), field_errors(a, b)
    ref = r64.state()
    amp = float(sum(p.west.waves[i][0] for i in range(100)))
    for form, tol in (("fused", 2e-6), ("mixed", 1e-7)):
        e = celeris.Engine(p, z, form)
        e.physical_steps(30)
        s = e.state()
        # west strip (columns 0, 1; rows 2 .. ny+1): the summed wave-maker values
        d = np.abs(s[2:-2, 0:2, :3].astype(np.float64) - ref[2:-2, 0:2, :3])
        assert d.max() <= tol * amp, (form, d.max())
        assert eta_rms(s, ref) <= 1e-4, form


@pytest.mark.parametrize("kind", ["sponge", "mixed", "irregular"])
def test_compensated_strips_keep_the_volume(celeris, kind):
    """Open boundaries (sine or irregular wave-makers, sponges) on small run-up cases: the
    compensated form's total water volume against the FP64 oracle after 400 steps, and the FP32
    form's for scale.  Measured: 2.7e-9 to 5.1e-9 for the compensated form against 9.6e-9 to
    1.6e-7 for FP32; the strips add no error of their own (their values are FP64), what remains
    comes from the single-precision fluxes and increments of the cells next to the run-up front."""
    p, z, bnx, bny = cases.small_case(70, 45, kind, correction_steps=1)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    ref.physical_steps(400)
    m_ref = ref.reset_timestep()["mass_full"]
    diffs = {}
    for form in ("mixed", "fused"):
        b = celeris.Batch([(p, z)], form)
        b.use_graph(True)
        b.step(400)
        m = b.stats_current()[0]["mass_full"]
        diffs[form] = abs(m - m_ref) / m_ref
    print(kind, diffs)
    assert diffs["mixed"] <= 1e-8, diffs
    assert diffs["mixed"] <= diffs["fused"], diffs
