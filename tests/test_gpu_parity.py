"""GPU parity: the CUDA forms against the CPU oracle on the same seeded inputs.

* plain FP32 form vs the FP32 transcription: the same passes and CR levels in the same order
  (compiled without FMA), so fields agree to 1e-5 relative (the gate for the plain form);
* fused FP32 and mixed forms vs the FP64 oracle: eta RMS error within 1e-4 m;
* batches give the same fields as single-domain fused engines.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as O
from celeris_b200 import cases
from util import eta_rms, field_errors, rel_ok

pytestmark = pytest.mark.gpu

KINDS = ["solid", "mixed", "sponge", "irregular", "uts", "nlsw"]


def _uts_rows():
    t = np.linspace(0.0, 40.0, 81)
    return np.stack([t, 0.2 * np.sin(2 * np.pi * t / 5.0), 0.3 * np.sin(2 * np.pi * t / 5.0),
                     0.05 * np.cos(2 * np.pi * t / 5.0)], axis=1)


def _case(kind, nx=40, ny=24, N=1):
    # "nlsw": the mixed boundary case with model type NLSW (identity tridiagonal systems)
    p, z, bnx, bny = cases.small_case(nx, ny, "mixed" if kind == "nlsw" else kind, correction_steps=N)
    if kind == "nlsw":
        # NLSW keeps the dispersion terms explicitly (engine.cpp:2625, 4127): stable at depth / dx ~ 1,
        # so a 4 m grid with the Courant number kept
        p.boussinesq = 0
        p.width, p.length, p.timestep = 4 * p.width, 4 * p.length, 4 * p.timestep
    if N == 0:
        # Pure AB3 (no corrector) at Courant 0.2 is unstable on these steep run-up cases in the
        # FP64 oracle as well; half the step keeps the method inside its stability region.
        p.timestep *= 0.5
    keep = []
    if kind == "uts":
        keep += cases.attach_uts(p, "west", _uts_rows())
        keep += cases.attach_uts(p, "north", _uts_rows())
    return p, z, bnx, bny, keep


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("N", [0, 1, 2])
def test_plain_matches_fp32_transcription(celeris, kind, N):
    p, z, bnx, bny, keep = _case(kind, N=N)
    ref = O.Oracle(p, z, bnx, bny, "f32")
    eng = celeris.Engine(p, z, "plain")
    # state, bottom and aux agree before the first step
    np.testing.assert_array_equal(eng.bottom().astype(np.float64), ref.bottom())
    np.testing.assert_allclose(eng.state()[..., :3], ref.state()[..., :3], rtol=0, atol=1e-6)
    ref.physical_steps(150)
    eng.physical_steps(150)
    a, b = eng.state(), ref.state()
    errs = field_errors(a, b)
    assert rel_ok(errs, 1e-5, 1e-9), errs
    # with correctly rounded transcendentals on both sides the two FP32 paths agree bit for bit
    assert np.array_equal(a[2:-2, 2:-2, :3].astype(np.float64), b[2:-2, 2:-2, :3]), errs
    aux_g, aux_r = eng.aux(), ref.aux()
    np.testing.assert_allclose(aux_g[2:-2, 2:-2, 0], aux_r[2:-2, 2:-2, 0], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("kind", ["mixed", "sponge"])
def test_plain_pass_by_pass(celeris, kind):
    p, z, bnx, bny, keep = _case(kind, N=1)
    ref = O.Oracle(p, z, bnx, bny, "f32")
    eng = celeris.Engine(p, z, "plain")
    for k in range(8):
        s_ref = ref.reset_timestep()
        s_gpu = eng.reset_timestep()
        assert s_gpu["time_scheme"] == s_ref["time_scheme"]
        assert abs(s_gpu["mass"] - s_ref["mass"]) <= 1e-5 * abs(s_ref["mass"])
        ref.timestep()
        eng.timestep()
        errs = field_errors(eng.state(), ref.state())
        assert rel_ok(errs, 1e-6, 1e-9), (k, errs)


@pytest.mark.parametrize("form", ["fused", "mixed"])
@pytest.mark.parametrize("kind", KINDS)
def test_fused_forms_vs_fp64_oracle(celeris, form, kind):
    p, z, bnx, bny, keep = _case(kind, nx=70, ny=45, N=1)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    eng = celeris.Engine(p, z, form)
    ref.physical_steps(200)
    eng.physical_steps(200)
    a, b = eng.state(), ref.state()
    assert np.isfinite(a).all()
    rms = eta_rms(a, b)
    assert rms <= 1e-4, rms
    errs = field_errors(a, b)
    assert rel_ok(errs, 2e-3, 1e-6), errs


def test_batch_equals_single_engines(celeris):
    members = [_case(k, nx=40 + 8 * i, ny=24 + 4 * i, N=1)[:4] for i, k in enumerate(["solid", "mixed", "sponge", "irregular"])]
    batch = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    batch.step(30)
    for i, (p, z, bnx, bny) in enumerate(members):
        e = celeris.Engine(p, z, "mixed")
        e.physical_steps(30)
        np.testing.assert_array_equal(batch.state(i), e.state())


TINY = [(2, 2), (3, 5), (7, 2), (2, 9)]


@pytest.mark.parametrize("nx, ny", TINY)
def test_smallest_domains(celeris, nx, ny):
    """The smallest grids the parameters accept (nx, ny >= 2: a 2-texel ghost frame around as
    little as 2 x 2 interior cells), with systems of 2 and 3 unknowns and strips wider than the
    domain: plain against the FP32 transcription bit for bit, the fused forms against the FP64
    oracle."""
    for kind in ("solid", "sponge", "mixed"):
        p, z, bnx, bny, keep = _case(kind, nx=nx, ny=ny, N=1)
        r32 = O.Oracle(p, z, bnx, bny, "f32")
        eng = celeris.Engine(p, z, "plain")
        r32.physical_steps(40)
        eng.physical_steps(40)
        a, b = eng.state(), r32.state()
        errs = field_errors(a, b)
        assert rel_ok(errs, 1e-5, 1e-9), (kind, errs)
        assert np.array_equal(a[2:-2, 2:-2, :3].astype(np.float64), b[2:-2, 2:-2, :3]), (kind, errs)
        r64 = O.Oracle(p, z, bnx, bny, "f64")
        r64.physical_steps(40)
        for form in ("fused", "mixed"):
            e = celeris.Engine(p, z, form)
            e.physical_steps(40)
            s = e.state()
            assert np.isfinite(s).all(), (kind, form)
            assert eta_rms(s, r64.state()) <= 1e-4, (kind, form)


def test_batch_of_smallest_domains_equals_single_engines(celeris):
    """Tiny members beside a larger one in one batch, replayed from graphs."""
    members = [_case(k, nx=nx, ny=ny, N=1)[:4] for (nx, ny), k in zip(TINY, ["solid", "sponge", "mixed", "solid"])]
    members.append(_case("irregular", nx=40, ny=24, N=1)[:4])
    batch = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    batch.use_graph(True)
    batch.step(30)
    for i, (p, z, bnx, bny) in enumerate(members):
        e = celeris.Engine(p, z, "mixed")
        e.physical_steps(30)
        np.testing.assert_array_equal(batch.state(i), e.state())


@pytest.mark.parametrize("adaptive", [False, True])
def test_lanes_change_concurrency_not_results(celeris, adaptive):
    """The same ensemble split into 1, 2 and 3 lanes (each lane its own stream, launches and
    graphs, members assigned by cell count): every member's state, statistics and clock agree
    bit for bit, under graph replay and with the caller's per-member time steps."""
    members = [_case(k, nx=40 + 12 * i, ny=24 + 6 * (i % 3), N=1)[:4]
               for i, k in enumerate(["solid", "mixed", "sponge", "irregular", "mixed"])]
    for m in members:
        m[0].adaptive = int(adaptive)
    runs = []
    for lanes in (1, 2, 3):
        b = celeris.Batch([(m[0], m[1]) for m in members], "mixed", lanes=lanes)
        assert b.lanes == lanes
        b.use_graph(True)
        b.step(12)
        if not adaptive:
            b.set_timestep(np.array([0.9 * m[0].timestep for m in members], dtype=np.float32))
        b.step(13)
        runs.append((b, [b.state(i) for i in range(len(members))], b.stats()))
    _, s1, t1 = runs[0]
    for b, s, t in runs[1:]:
        for i in range(len(members)):
            np.testing.assert_array_equal(s[i], s1[i])
            assert t[i]["mass_full"] == t1[i]["mass_full"]
            assert t[i]["total_time"] == t1[i]["total_time"]
            assert t[i]["timestep"] == t1[i]["timestep"]


def test_refused_time_steps_change_no_lane(celeris):
    """A per-member time step array with one invalid entry is refused as a whole: no lane takes
    the valid entries (the bad entry is tried at every member, so it lands in every lane)."""
    members = [_case(k, nx=40 + 8 * i, ny=24, N=1)[:4] for i, k in enumerate(["solid", "mixed", "sponge"])]
    a = celeris.Batch([(m[0], m[1]) for m in members], "mixed", lanes=2)
    b = celeris.Batch([(m[0], m[1]) for m in members], "mixed", lanes=2)
    a.step(5)
    b.step(5)
    half = np.array([0.5 * m[0].timestep for m in members], dtype=np.float32)
    for j in range(len(members)):
        bad = half.copy()
        bad[j] = -1.0
        with pytest.raises(celeris.CelError, match="> 0"):
            a.set_timestep(bad)
    a.step(5)
    b.step(5)
    for i in range(len(members)):
        np.testing.assert_array_equal(a.state(i), b.state(i))


def test_batch_member_index_checks(celeris):
    """Member indices are the caller's whatever the lane split; one outside [0, n) is an argument
    error for every per-member call, and the batch stays usable."""
    members = [_case(k, nx=40, ny=24, N=1)[:4] for k in ["solid", "mixed", "sponge"]]
    b = celeris.Batch([(m[0], m[1]) for m in members], "mixed", lanes=2)
    z = members[0][1]
    L = celeris.lib()
    buf = np.zeros((28, 44, 4), dtype=np.float32)
    for i in (-1, 3):
        assert L.cel_batch_get_state(b.h, i, buf.ctypes.data_as(C.POINTER(C.c_float))) == 1
        assert b"range" in L.cel_last_error()
        with pytest.raises(celeris.CelError, match="range"):
            b.add_solitary_wave(i, 0.1, 0.0, 10.0, 10.0)
        with pytest.raises(celeris.CelError, match="range"):
            b.set_bathymetry(i, z)
    b.step(3)
    assert all(st["health"] == 0 for st in b.stats())


def test_lanes_follow_the_callers_stream(celeris):
    """A 2-lane batch moved onto a caller's stream mid-run and back (lane 0 runs on it, lane 1
    forks from it and joins it; the switch drains lane 1 and recaptures lane 0's graphs): the
    same fields as a batch that stays on its own stream."""
    import torch
    members = [_case(k, nx=48 + 8 * i, ny=32, N=1)[:4] for i, k in enumerate(["solid", "mixed", "sponge", "irregular"])]
    ref = celeris.Batch([(m[0], m[1]) for m in members], "mixed", lanes=2)
    ref.use_graph(True)
    ref.step(30)
    b = celeris.Batch([(m[0], m[1]) for m in members], "mixed", lanes=2)
    b.use_graph(True)
    b.step(10)
    s = torch.cuda.Stream()
    b.set_stream(s.cuda_stream)
    b.step(10)
    done = torch.cuda.Event()
    done.record(s)
    done.synchronize()
    after = b.stats()
    b.set_stream(None)
    b.step(10)
    for i in range(len(members)):
        np.testing.assert_array_equal(b.state(i), ref.state(i))
    assert all(st["health"] == 0 for st in after)


def test_batch_graph_replay_matches_direct(celeris):
    members = [_case(k, nx=48, ny=32, N=1)[:4] for k in ["mixed", "sponge", "irregular"]]
    b1 = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    b2 = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    b2.use_graph(True)
    b1.step(25)
    b2.step(25)
    for i in range(len(members)):
        np.testing.assert_array_equal(b1.state(i), b2.state(i))
    s1, s2 = b1.stats(), b2.stats()
    for a, b in zip(s1, s2):
        assert a["mass_full"] == b["mass_full"]
        assert abs(a["total_time"] - b["total_time"]) < 1e-12


def test_flume_config1_plain_1000_steps(celeris):
    """C1 (512x64 flume, sine wave-maker): plain FP32 GPU vs the FP32 transcription after
    1000 physical steps, 1e-5 relative in eta/hu/hv; mass agrees too."""
    p, z, bnx, bny = cases.config1()
    ref = O.Oracle(p, z, bnx, bny, "f32")
    eng = celeris.Engine(p, z, "plain")
    s_ref = ref.physical_steps(1000)
    eng.physical_steps(1000)
    errs = field_errors(eng.state(), ref.state())
    assert rel_ok(errs, 1e-5, 1e-9), errs
    s_gpu = eng.reset_timestep()
    s_ref = ref.reset_timestep()
    assert abs(s_gpu["mass_full"] - s_ref["mass_full"]) <= 1e-6 * s_ref["mass_full"]


def test_tall_domain_narrow_column_bands(celeris):
    """ny above ~3,500 rows makes the column solver use 8-column bands (64 chunks per column)."""
    p, z, bnx, bny = cases.small_case(36, 3700, "solid", correction_steps=1)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    b = celeris.Batch([(p, z)], "mixed")
    ref.physical_steps(60)
    b.step(60)
    a = b.state(0)
    assert np.isfinite(a).all()
    assert eta_rms(a, ref.state()) <= 1e-4


def test_batch_stats_describe_the_start_of_the_last_step(celeris):
    """cel_batch_stats (gathered by the first pass of a step) equals the statistics of the state
    the step started from (cel_batch_stats_current one step earlier)."""
    members = [_case(k, nx=48, ny=32, N=1)[:4] for k in ["mixed", "sponge"]]
    b1 = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    b2 = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    b1.step(11)
    before = b1.stats_current()
    b2.step(12)
    fused = b2.stats()
    for s, f in zip(before, fused):
        # sums of depth agree to the FP64 reduction order; velocity-derived totals also carry the
        # FP32 difference between the stencil's reciprocal square root and a division
        for k in ("mass", "mass_full", "potential_energy", "max_depth"):
            assert f[k] == pytest.approx(s[k], rel=1e-9, abs=1e-12), k
        for k in ("kinetic_energy", "max_speed", "cfl_rate"):
            assert f[k] == pytest.approx(s[k], rel=1e-6, abs=1e-12), k
        assert f["total_time"] == pytest.approx(s["total_time"], rel=1e-12)


def test_tuning_changes_decomposition_not_results(celeris):
    """Band width, strip height and the column solver's chunks per column (its switch point from
    the carry scan to serial sweeps) only change how the work is split: the fields agree to FP32
    rounding (the column scans group their additions differently)."""
    members = [_case(k, nx=150 + 10 * i, ny=70 + 30 * i, N=1)[:4] for i, k in enumerate(["mixed", "sponge", "irregular"])]
    ref = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    ref.step(30)
    for bw, sh, chunks in [(32, 32, 16), (32, 64, 8), (8, 128, 64), (8, 32, 32), (16, 8, 16), (16, 64, 32), (1, 64, 0),
                           (32, 64, 32), (32, 32, 64), (32, 64, 128),    # cluster solver
                           (16, 64, 1)]:                                  # tile-transposed solver
        b = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
        b.set_tuning(bw, sh, chunks)
        assert b.tuning == (bw, sh)
        assert b.col_chunks == (chunks if bw > 1 else 1)
        b.step(30)
        for i in range(len(members)):
            errs = field_errors(b.state(i), ref.state(i))
            assert rel_ok(errs, 1e-5, 1e-9), (bw, sh, chunks, errs)
    with pytest.raises(celeris.CelError):   # 16 columns x 48 chunks = 768 threads: not a solver size
        celeris.Batch([(m[0], m[1]) for m in members], "mixed").set_tuning(16, 64, 48)
    tall = [_case("mixed", nx=40, ny=520, N=1)[:4]]
    with pytest.raises(celeris.CelError):   # 520 rows > 32 chunks x 16 rows: too tall for the cluster solver
        celeris.Batch([(m[0], m[1]) for m in tall], "mixed").set_tuning(32, 64, 32)
    t = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    got = t.autotune(2)
    assert got["band_width"] in (1, 8, 16, 32) and got["strip_height"] in (32, 64, 128) and got["ms_per_step"] > 0
    assert t.tuning == (got["band_width"], got["strip_height"])
    t.use_graph(True)
    t.step(5)
    assert np.isfinite(t.state(0)).all()


@pytest.mark.parametrize("form", ["fused", "mixed"])
@pytest.mark.parametrize("kind", KINDS)
def test_paired_row_stencil_vs_fp64_oracle(celeris, form, kind):
    """The two-rows-per-step stencil (paired f32x2 arithmetic) against the FP64 oracle."""
    p, z, bnx, bny, keep = _case(kind, nx=70, ny=45, N=1)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    b = celeris.Batch([(p, z)], form)
    b.set_stencil_rows(2)
    assert b.stencil_rows == 2
    ref.physical_steps(200)
    b.step(200)
    a = b.state(0)
    assert np.isfinite(a).all()
    assert eta_rms(a, ref.state()) <= 1e-4
    assert rel_ok(field_errors(a, ref.state()), 2e-3, 1e-6)


def test_paired_row_stencil_matches_single_row(celeris):
    """Both stencils on the same ensemble (odd and even strip heights): the fields agree to FP32
    rounding and the aux texture (max depth, breaking) is identical in coverage."""
    members = [_case(k, nx=150 + 10 * i, ny=71 + 30 * i, N=1)[:4] for i, k in enumerate(["mixed", "sponge", "irregular"])]
    for sh in (32, 33):
        b1 = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
        b2 = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
        b1.set_tuning(16, sh)
        b2.set_tuning(16, sh)
        b2.set_stencil_rows(2)
        b1.step(40)
        b2.step(40)
        for i in range(len(members)):
            assert rel_ok(field_errors(b2.state(i), b1.state(i)), 1e-5, 1e-9), (sh, i)
            a1, a2 = b1.aux(i), b2.aux(i)
            np.testing.assert_allclose(a2[..., 0], a1[..., 0], rtol=1e-4, atol=1e-6)
            assert ((a1[..., 3] > 0) == (a2[..., 3] > 0)).mean() > 0.999
        s1, s2 = b1.stats(), b2.stats()
        for x, y in zip(s1, s2):
            assert y["mass_full"] == pytest.approx(x["mass_full"], rel=1e-9)


@pytest.mark.parametrize("form", ["fused", "mixed"])
@pytest.mark.parametrize("kind, N", [("mixed", 1), ("sponge", 0), ("solid", 1)])
def test_adaptive_batch_vs_fp64_oracle(celeris, form, kind, N):
    """Adaptive time steps chosen on the device (engine.cpp:1698-1726, compute.hlsl:766-780)."""
    p, z, bnx, bny, keep = _case(kind, nx=70, ny=45, N=N)
    p.adaptive = 1
    ref = O.Oracle(p, z, bnx, bny, "f64")
    eng = celeris.Engine(p, z, form)
    ref.physical_steps(150)
    eng.physical_steps(150)
    a, b = eng.state(), ref.state()
    assert np.isfinite(a).all()
    rms = eta_rms(a, b)
    assert rms <= 1e-4, rms
    # the clock is the sum of the chosen steps: the dt sequences agree
    t_ref = ref.reset_timestep()["total_time"]
    t_gpu = eng.stats()["total_time"]
    assert abs(t_gpu - t_ref) <= 1e-5 * t_ref, (t_gpu, t_ref)


def test_adaptive_batch_equals_single_engines_and_graph_replay(celeris):
    members = [_case(k, nx=40 + 8 * i, ny=24 + 4 * i, N=1)[:4] for i, k in enumerate(["solid", "mixed", "sponge"])]
    for m in members:
        m[0].adaptive = 1
    direct = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    direct.step(40)
    graph = celeris.Batch([(m[0], m[1]) for m in members], "mixed")
    graph.use_graph(True)
    graph.step(40)
    sd, sg = direct.stats_current(), graph.stats_current()
    for i, (p, z, bnx, bny) in enumerate(members):
        e = celeris.Engine(p, z, "mixed")
        e.physical_steps(40)
        np.testing.assert_array_equal(direct.state(i), e.state())
        np.testing.assert_array_equal(graph.state(i), e.state())
        assert sd[i]["total_time"] == sg[i]["total_time"] == e.stats()["total_time"]
        assert sd[i]["timestep"] > 0


def test_adaptive_batch_refuses_host_time_steps(celeris):
    p, z, bnx, bny, keep = _case("solid", N=1)
    p.adaptive = 1
    b = celeris.Batch([(p, z)], "mixed")
    with pytest.raises(celeris.CelError, match="adaptive"):
        b.set_timestep(np.array([1e-3], dtype=np.float32))
    q, z2, _, _, _ = _case("solid", N=1)
    with pytest.raises(celeris.CelError, match="adaptive"):
        celeris.Batch([(p, z), (q, z2)], "mixed")


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_spectrum_wavemaker(celeris, form):
    """A west wave-maker driven by the spectrum generator's 90 components (a larger pairwise sum
    tree than the hand-made component lists)."""
    p, z, bnx, bny, keep = _case("irregular", nx=60, ny=40, N=1)
    b = celeris.spectrum_waves(0.3, 6.0, 10.0, 5.0, seed=11)
    assert b.n_waves > 64
    p.west.n_waves = b.n_waves
    for k in range(b.n_waves):
        for q in range(4):
            p.west.waves[k][q] = b.waves[k][q]
    eng = celeris.Engine(p, z, form)
    eng.physical_steps(120)
    a = eng.state()
    if form == "plain":
        ref = O.Oracle(p, z, bnx, bny, "f32")
        ref.physical_steps(120)
        np.testing.assert_array_equal(a[2:-2, 2:-2, :3].astype(np.float64), ref.state()[2:-2, 2:-2, :3])
    else:
        ref = O.Oracle(p, z, bnx, bny, "f64")
        ref.physical_steps(120)
        assert eta_rms(a, ref.state()) <= 1e-4


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_stencil_width_changes_decomposition_not_results(celeris, form):
    """96-thread strips (94 columns) against 128-thread strips (126 columns): every cell is computed
    by the same arithmetic, so the states and aux are identical; the statistics only regroup their
    sums (different partial sums per strip)."""
    members = [_case(k, nx=nx, ny=ny, N=1)[:4]
               for k, nx, ny in (("mixed", 130, 41), ("sponge", 256, 33), ("irregular", 95, 64), ("uts", 190, 20))]
    b1 = celeris.Batch([(m[0], m[1]) for m in members], form)
    b2 = celeris.Batch([(m[0], m[1]) for m in members], form)
    for b in (b1, b2):
        b.set_stencil_rows(2)
    b2.set_stencil_width(96)
    assert (b1.stencil_width, b2.stencil_width) == (128, 96)
    b1.step(30)
    b2.step(30)
    for i in range(len(members)):
        np.testing.assert_array_equal(b2.state(i), b1.state(i))
        np.testing.assert_array_equal(b2.aux(i), b1.aux(i))
    for x, y in zip(b1.stats(), b2.stats()):
        assert y["mass_full"] == pytest.approx(x["mass_full"], rel=1e-12)
        assert y["max_depth"] == x["max_depth"]
    with pytest.raises(celeris.CelError):
        b1.set_stencil_width(64)


_WIDE = {}


def _widest_reference():
    """FP64 oracle state of the widest case after 40 steps (computed once for both forms)."""
    if "state" not in _WIDE:
        p, z, bnx, bny, keep = _wide_case()
        ref = O.Oracle(p, z, bnx, bny, "f64")
        ref.physical_steps(40)
        _WIDE["state"] = ref.state()
    return _WIDE["state"]


def _wide_case():
    # the small cases' 0.12 bed slope would climb ~1900 m over 16000 columns, and single-precision
    # rounding of w = B on that dry land would swamp the comparison: the bed is capped at +1 m
    p, z, bnx, bny, keep = _case("sponge", nx=16000, ny=12, N=1)
    return p, np.minimum(z, 1.0).astype(np.float32), bnx, bny, keep


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_widest_domain(celeris, form):
    """The widest row the fused forms accept (nx = 16000: the row solver keeps a whole row in
    shared memory), against the FP64 oracle; one column past the limit is refused."""
    p, z, bnx, bny, keep = _wide_case()
    eng = celeris.Engine(p, z, form)
    eng.physical_steps(40)
    a = eng.state()
    assert np.isfinite(a).all()
    assert eta_rms(a, _widest_reference()) <= 1e-4
    q, z2, _, _, _ = _case("sponge", nx=16001, ny=12, N=1)
    with pytest.raises(celeris.CelError, match="nx"):
        celeris.Engine(q, z2, form)


def _terrain_change(z):
    """A new bathymetry: the old one with a shoal added and the beach lowered."""
    ny, nx = z.shape
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
    return (z + 1.2 * np.exp(-((X - 0.55 * nx) ** 2 + (Y - 0.4 * ny) ** 2) / (2 * (0.1 * nx) ** 2))
            - 0.3 * (X > 0.8 * nx)).astype(np.float32)


@pytest.mark.parametrize("kind", ["mixed", "sponge"])
def test_new_terrain_plain_matches_fp32_transcription(celeris, kind):
    """newTerrainSettings mid-run (engine.cpp:3313-3379): depth kept, aux cleared, coefficients kept;
    then a remesh rebuilds everything from the new grid."""
    p, z, bnx, bny, keep = _case(kind, nx=48, ny=30, N=1)
    ref = O.Oracle(p, z, bnx, bny, "f32")
    eng = celeris.Engine(p, z, "plain")
    ref.physical_steps(30)
    eng.physical_steps(30)
    z2 = _terrain_change(z)
    ref.new_terrain(z2)
    eng.set_bathymetry(z2)
    np.testing.assert_array_equal(eng.bottom().astype(np.float64), ref.bottom())
    np.testing.assert_array_equal(eng.state()[..., :3].astype(np.float64), ref.state()[..., :3])
    assert not eng.aux()[..., 0].any()
    ref.physical_steps(40)
    eng.physical_steps(40)
    np.testing.assert_array_equal(eng.state()[2:-2, 2:-2, :3].astype(np.float64), ref.state()[2:-2, 2:-2, :3])
    # remesh: a fresh engine on the new grid
    eng.remesh()
    fresh = O.Oracle(p, z2, bnx, bny, "f32")
    np.testing.assert_array_equal(eng.state()[..., :3].astype(np.float64), fresh.state()[..., :3])
    eng.physical_steps(10)
    fresh.physical_steps(10)
    np.testing.assert_array_equal(eng.state()[2:-2, 2:-2, :3].astype(np.float64), fresh.state()[2:-2, 2:-2, :3])


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_new_terrain_fused_forms(celeris, form):
    p, z, bnx, bny, keep = _case("mixed", nx=70, ny=45, N=1)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    eng = celeris.Engine(p, z, form)
    ref.physical_steps(40)
    eng.physical_steps(40)
    z2 = _terrain_change(z)
    ref.new_terrain(z2)
    eng.set_bathymetry(z2)
    np.testing.assert_array_equal(eng.bottom().astype(np.float64), ref.bottom())
    ref.physical_steps(60)
    eng.physical_steps(60)
    assert eta_rms(eng.state(), ref.state()) <= 1e-4
    # the same change on one member of a batch leaves the other members untouched
    q, zq, _, _, _ = _case("sponge", nx=40, ny=24, N=1)
    b = celeris.Batch([(p, z), (q, zq)], form)
    solo = celeris.Batch([(q, zq)], form)
    b.step(5)
    solo.step(5)
    b.set_bathymetry(0, z2)
    b.step(5)
    solo.step(5)
    np.testing.assert_array_equal(b.state(1), solo.state(0))


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_new_terrain_paired_row_stencil(celeris, form):
    """The paired-row stencil rebuilds BA, BX and BY from the corner grid: a terrain change must
    reach its corner plane.  A batch member's terrain changes mid-run and the batch follows the FP64
    oracle through the same change (a stale corner plane would keep the old bed under the new one)."""
    p, z, bnx, bny, keep = _case("mixed", nx=70, ny=45, N=1)
    z2 = _terrain_change(z)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    ref.physical_steps(40)
    ref.new_terrain(z2)
    ref.physical_steps(60)
    b = celeris.Batch([(p, z)], form)
    b.set_stencil_rows(2)
    b.step(40)
    b.set_bathymetry(0, z2)
    b.step(60)
    assert eta_rms(b.state(0), ref.state()) <= 1e-4


def _water_height_expected(state, bottom, p, x, y):
    """getWaterHeight (engine.cpp:4994-5012) restated in float32: GetTerrainHeight's bilinear of BA
    (terrain_heightfield.cpp:313-351) plus the 4x4 block's sum of h (GetStats order) / 16."""
    f = np.float32
    nx, ny, W, L = p.nx, p.ny, f(p.width), f(p.length)
    BA = bottom[..., 2].astype(np.float32)
    tx = f(f(f(x) + W / f(2)) / W * f(nx - 1))
    ty = f(f(y) / L * f(ny - 1))
    tx, ty = f(min(max(tx, f(0)), f(nx - 1)) + f(2)), f(min(max(ty, f(0)), f(ny - 1)) + f(2))
    xd, xu, yd, yu = int(np.floor(tx)), int(np.ceil(tx)), int(np.floor(ty)), int(np.ceil(ty))
    xf, yf = f(tx - f(xd)), f(ty - f(yd))
    lerp = lambda t, a, b: f(a + f(t * f(b - a)))
    terrain = lerp(yf, lerp(xf, BA[yd, xd], BA[yd, xu]), lerp(xf, BA[yu, xd], BA[yu, xu]))
    ix = int(f(f(f(x) + W / f(2)) / W) * f(nx // 4))
    iy = int(f(f(y) / L) * f(ny // 4))
    ix, iy = min(max(ix, 0), nx // 4 - 1), min(max(iy, 0), ny // 4 - 1)
    s = f(0)
    for j in range(2, 6):
        for i in range(2, 6):
            yy, xx = iy * 4 + j, ix * 4 + i
            s = f(s + max(f(0), f(state[yy, xx, 0] - BA[yy, xx])))
    return f(terrain + f(s / f(16)))


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_water_height_follows_get_water_height(celeris, form):
    p, z, bnx, bny, keep = _case("mixed", nx=48, ny=32, N=1)
    eng = celeris.Engine(p, z, form)
    eng.physical_steps(20)
    eng.reset_timestep()
    st, bot = eng.state(), eng.bottom()
    W, L = p.width, p.length
    for x, y in [(0.0, 0.5 * L), (-0.3 * W, 0.21 * L), (0.41 * W, 0.77 * L), (-W / 2, 0.0), (W / 2, L)]:
        want = _water_height_expected(st, bot, p, x, y)
        got = eng.water_height(x, y)
        if form == "plain":
            assert got == want, (x, y, got, want)
        else:
            assert got == pytest.approx(float(want), rel=1e-6, abs=1e-6), (x, y)


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_add_solitary_wave_fused_forms(celeris, form):
    """addSolitaryWave mid-run (engine.cpp:2154-2219) in the fused forms against the FP64 oracle,
    and on one batch member without touching the others.  The reference does not re-bootstrap after
    the wave, so its next pass takes its fluxes from the faces of the state before the wave; the
    fused forms keep no Pass1 textures and take them from the state with the wave, so the oracle is
    told to re-bootstrap for this comparison."""
    p, z, bnx, bny, keep = _case("solid", nx=70, ny=45, N=1)
    ref = O.Oracle(p, z, bnx, bny, "f64")
    eng = celeris.Engine(p, z, form)
    ref.physical_steps(20)
    eng.physical_steps(20)
    ref.add_solitary_wave(0.3, 25.0, 30.0, 20.0)
    ref.rebootstrap()
    eng.add_solitary_wave(0.3, 25.0, 30.0, 20.0)
    assert eta_rms(eng.state(), ref.state()) <= 1e-6
    ref.physical_steps(40)
    eng.physical_steps(40)
    assert eta_rms(eng.state(), ref.state()) <= 1e-4
    q, zq, _, _, _ = _case("sponge", nx=40, ny=24, N=1)
    b = celeris.Batch([(p, z), (q, zq)], form)
    solo = celeris.Batch([(q, zq)], form)
    b.step(3)
    solo.step(3)
    b.add_solitary_wave(0, 0.3, 25.0, 30.0, 20.0)
    b.step(3)
    solo.step(3)
    np.testing.assert_array_equal(b.state(1), solo.state(0))


def test_live_batches_of_different_sizes_step_in_any_order(celeris):
    """Shared-memory limits are per kernel for the whole process: a smaller batch created later
    must not stop a larger one from stepping (row solver and column solver buffers)."""
    big = [_case("sponge", nx=3000, ny=90, N=1)[:2], _case("mixed", nx=70, ny=300, N=1)[:2]]
    small = [_case("solid", nx=40, ny=24, N=1)[:2]]
    b1 = celeris.Batch(big, "mixed")
    b1.step(2)
    b2 = celeris.Batch(small, "mixed")
    b2.step(2)
    b1.step(3)
    ref = celeris.Batch(big, "mixed")
    ref.step(5)
    for i in range(len(big)):
        np.testing.assert_array_equal(b1.state(i), ref.state(i))


def test_adaptive_batch_reports_the_uniform_step_before_its_first_pass(celeris):
    p, z, bnx, bny, keep = _case("solid", N=1)
    p.adaptive = 1
    b = celeris.Batch([(p, z)], "mixed")
    s = b.stats()[0]
    assert s["timestep"] == float(np.float32(p.timestep))
    assert s["total_time"] == 0.0
    b.step(3)
    assert b.stats()[0]["timestep"] > 0


@pytest.mark.parametrize("form", ["fused", "mixed"])
def test_state_parts_sum_to_the_state(celeris, form):
    """cel_batch_get_state_parts: hi + lo is the compensated state (lo = 0 in the FP32 form), and
    cel_batch_get_state returns that sum rounded to float."""
    members = [_case(k, nx=48, ny=32, N=1)[:4] for k in ["mixed", "sponge"]]
    b = celeris.Batch([(m[0], m[1]) for m in members], form)
    b.step(25)
    for i in range(len(members)):
        hi, lo = b.state_parts(i)
        if form == "fused":
            assert not lo.any()
        else:
            assert np.abs(lo[2:-2, 2:-2, :3]).max() > 0      # the low words carry something
            assert np.all(np.abs(lo) <= np.abs(hi) * 2.0 ** -23 + 1e-30)
        np.testing.assert_array_equal((hi.astype(np.float64) + lo).astype(np.float32), b.state(i))
