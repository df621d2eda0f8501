"""The irregular-wave spectrum generator (reference engine.cpp:3559-3776), on the CPU.

Pinned to the reference's own generator: generateSpectrumWaves cut out of engine.cpp and compiled
here (oracle/ref_build.py -> oracle/_ref/libref_spectrum.so), whose component files for a set of
settings are committed as tests/golden/ref_spectrum.npz (tests/golden/make_spectrum_golden.py).
Also against the numpy restatement in oracle/spectrum_oracle.py, which carries the FP64 side.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

import spectrum_oracle as S  # oracle/spectrum_oracle.py

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_spectrum.npz")
REF_LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libref_spectrum.so")

CASES = [(1.0, 10.0, 0.0, 15.0), (2.5, 14.0, 12.5, 20.0), (0.4, 6.0, -30.0, 3.0), (3.0, 8.0, 0.0, 4.0)]


def waves(b):
    return np.array([[b.waves[k][q] for q in range(4)] for k in range(b.n_waves)])


@pytest.mark.parametrize("hs, tp, th, h", CASES)
@pytest.mark.parametrize("seed", [0, 12345])
def test_components_match_the_restatement(celeris, hs, tp, th, h, seed):
    got = waves(celeris.spectrum_waves(hs, tp, th, h, seed=seed))
    ref = S.spectrum_waves(hs, tp, th, h, seed=seed)
    assert got.shape == ref.shape and got.shape[0] % 9 == 0       # 9 directions per kept frequency
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=2e-6)   # amplitude: float storage
    np.testing.assert_allclose(got[:, 1:3], ref[:, 1:3], rtol=1e-6, atol=1e-7)
    np.testing.assert_array_equal(got[:, 3], ref[:, 3])            # phases: same seeded sequence


def test_properties(celeris):
    got = waves(celeris.spectrum_waves(1.0, 10.0, 0.0, 15.0, seed=7))
    thetas = np.unique(np.round(got[:, 2], 6))
    np.testing.assert_allclose(thetas, np.arange(-20, 21, 5) * 3.1415 / 180, atol=2e-6)
    assert (got[:, 0] > 0).all() and (got[:, 3] >= 0).all() and (got[:, 3] < 2 * 3.1415).all()
    # the energy is symmetric about the mean direction
    a = got[:, 0].reshape(-1, 9)
    np.testing.assert_allclose(a, a[:, ::-1], rtol=1e-6)
    # periods bracket the peak period
    assert got[:, 1].min() < 10.0 < got[:, 1].max()
    # another seed changes only the phases
    other = waves(celeris.spectrum_waves(1.0, 10.0, 0.0, 15.0, seed=8))
    np.testing.assert_array_equal(other[:, :3], got[:, :3])
    assert not np.array_equal(other[:, 3], got[:, 3])


def test_wave_height_is_capped_at_half_the_depth(celeris):
    a = waves(celeris.spectrum_waves(5.0, 10.0, 0.0, 4.0))
    b = waves(celeris.spectrum_waves(2.0, 10.0, 0.0, 4.0))
    np.testing.assert_array_equal(a, b)


def test_file_reads_back_as_irregular_waves(tmp_path, celeris):
    from celeris_b200 import abi
    path = str(tmp_path / "irr.txt")
    b = celeris.spectrum_waves(1.0, 10.0, 0.0, 15.0, seed=3, path=path)
    txt = open(path).read()
    assert txt.startswith("[Hs] 1\n[Tp] 10\n[Theta_p] 0\n[h_source] 15\n")
    assert f"[NumberOfWaves] {b.n_waves}\n" in txt
    back = abi.Boundary()
    assert celeris.lib().cel_read_irregular_waves(path.encode(), C.byref(back)) == 0
    assert back.n_waves == b.n_waves
    np.testing.assert_allclose(waves(back), waves(b), rtol=1e-5, atol=1e-6)   # 6 significant digits


def test_zero_inputs_are_refused(celeris):
    with pytest.raises(celeris.CelError):
        celeris.spectrum_waves(1.0, 0.0, 0.0, 15.0)
    with pytest.raises(celeris.CelError):
        celeris.spectrum_waves(1.0, 10.0, 0.0, 0.0)


def _check_against_reference_file(got: np.ndarray, ref: np.ndarray):
    """ref: the reference's component file rows (six significant digits each)."""
    assert got.shape == ref.shape
    np.testing.assert_allclose(got[:, 0], ref[:, 0], rtol=1e-5)              # amplitude
    np.testing.assert_allclose(got[:, 1], ref[:, 1], rtol=1e-5)              # period
    np.testing.assert_allclose(got[:, 2], ref[:, 2], rtol=1e-5, atol=1e-6)   # direction (rad)
    # phases: both sides quantise a random draw as (r % 10000) / 10000 x 2 x 3.1415
    q = 2 * 3.1415 / 10000
    for ph in (got[:, 3], ref[:, 3]):
        steps = ph / q
        assert np.max(np.abs(steps - np.round(steps))) < 1e-2


def test_components_match_the_reference_build_fixtures(celeris):
    g = np.load(GOLDEN)
    for k, case in enumerate(g["cases"]):
        got = waves(celeris.spectrum_waves(*[float(v) for v in case], seed=5))
        _check_against_reference_file(got, g[f"case{k}"])


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="oracle/_ref/libref_spectrum.so is not built")
def test_components_match_the_reference_build_live(celeris):
    """More settings than the fixtures hold, straight against the reference's generator."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_spectrum_golden import reference_rows
    lib = C.CDLL(REF_LIB)
    rng = np.random.default_rng(3)
    for _ in range(12):
        case = (float(rng.uniform(0.2, 4.0)), float(rng.uniform(4.0, 16.0)), float(rng.uniform(-40, 40)),
                float(rng.uniform(1.0, 30.0)))
        got = waves(celeris.spectrum_waves(*case, seed=1))
        _check_against_reference_file(got, reference_rows(lib, *case))
