"""The long-run comparison (tests/long_run.py compare / record) on synthetic records, on the CPU.

It checks the metrics the accuracy record is made of: eta on the free surface max(w, B), so that a
dry cell's w below the bed counts as the bed; the low words of the compensated form added to its
state; run-up from the inundation bits; the volume difference with and without the films thinner
than the reference's minimum depth; and a record of several cases in one JSON file.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import long_run as L  # noqa: E402


def _files(tmp_path, w_gpu_hi, w_gpu_lo=None):
    ny, nx = 8, 10
    B = np.zeros((ny + 4, nx + 4), np.float32)
    B[:, 8:] = 2.0                                     # dry land on the east side
    w_ref = np.full_like(B, 0.5)
    w_ref[:, 8:] = 2.0                                 # dry: w = B
    maxd = np.where(B < 0.5, 0.5, 0.0).astype(np.float32)
    maxd[:, 8] = 0.01                                  # the water reached the first dry column: run-up 2 m
    m_ref = np.array([100.0, 101.0, 102.0])
    ref = tmp_path / "ref.npz"
    np.savez(ref, bottom=B, eta=w_ref.astype(np.float64), maxdepth=maxd, mass=m_ref, every=10, form="fp64-oracle")
    out = {"mixed/eta": w_gpu_hi.astype(np.float32), "mixed/inundated": L._inundated(maxd),
           "mixed/mass": m_ref * (1 + 1e-10)}
    if w_gpu_lo is not None:
        out["mixed/eta_lo"] = w_gpu_lo.astype(np.float32)
    gpu = tmp_path / "gpu.npz"
    np.savez(gpu, every=10, **out)
    return ref, gpu, w_ref, B


def test_dry_cells_below_the_bed_count_as_the_bed(tmp_path):
    ref, gpu, w_ref, B = _files(tmp_path, np.zeros(1))
    w = w_ref.copy()
    w[:, 8:] = -5.0                                    # a sponge pulled dry land's w below the bed
    w[5, 4] += 1e-3                                    # one wet cell differs by 1 mm
    np.savez(gpu, every=10, **{"mixed/eta": w.astype(np.float32),
                               "mixed/inundated": L._inundated(np.where(B < 0.5, 0.5, 0.0) + (np.arange(14) == 8)),
                               "mixed/mass": np.array([100.0, 101.0, 102.0])})
    r = L.compare_files(str(ref), str(gpu), None)["mixed"]
    n = 8 * 10
    assert abs(r["eta_rms_m"] / np.sqrt(1e-6 / n) - 1) < 1e-4  # only the wet cell's (float) 1 mm
    assert r["w_rms_m"] > 1.0                                  # raw w sees the dry land
    assert r["mass_rel_diff_end"] == 0.0
    assert r["runup_m"] == 2.0 and r["runup_err_m"] == 0.0


def test_low_words_join_the_state_and_films_split_the_volume(tmp_path):
    hi, lo = np.full((12, 14), 0.5, np.float32), np.zeros((12, 14), np.float32)
    hi[:, 8:] = 2.0
    lo[2:-2, 8:10] = 5e-5                              # films of 0.05 mm on dry land, in the low words
    lo[3, 3] = 1e-6                                    # and a low word on a wet cell
    ref, gpu, w_ref, B = _files(tmp_path, hi, lo)
    r = L.compare_files(str(ref), str(gpu), None)["mixed"]
    V = 0.5 * 8 * 6                                    # the reference volume (8 rows, wet columns 2 .. 7)
    film = 5e-5 * 8 * 2
    assert abs(r["end_volume_rel_diff"] / ((film + 1e-6) / V) - 1) < 1e-4
    assert abs(r["end_volume_rel_diff_films_excluded"] / (1e-6 / V) - 1) < 1e-2
    assert r["film_depth_sum_m"][0] == 0.0 and abs(r["film_depth_sum_m"][1] - film) < 1e-9


def test_record_collects_cases(tmp_path):
    ref, gpu, w_ref, B = _files(tmp_path, np.full((12, 14), 0.5, np.float32))
    out = tmp_path / "rec.json"

    class A:
        pass
    a = A()
    a.out = str(out)
    a.spec = [f"case one={ref},{gpu},", f"case two!={ref},{gpu},mixed"]
    L.record(a)
    d = json.load(open(out))
    assert [e["case"] for e in d["entries"]] == ["case one", "case two"]
    assert d["entries"][1]["fp64_nonfinite"] is True
    assert "mixed" in d["entries"][0]
