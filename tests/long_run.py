"""Long-run accuracy of the CUDA forms against the FP64 oracle (a measurement, not a pytest test).

The FP64 oracle at 1024^2 x 10,000 steps takes tens of CPU minutes, so the two sides run
separately and meet in .npz files:

  python tests/long_run.py oracle --case c3 --steps 10000 --out ref.npz   # CPU, FP64 oracle
  python tests/long_run.py gpu    --case c3 --steps 10000 --out gpu.npz   # CUDA forms
  python tests/long_run.py compare ref.npz gpu.npz                        # prints one JSON line
  python tests/long_run.py record --out rec.json "C3=ref.npz,gpu.npz," ...  # several into one file

Cases: ``c3`` (1024^2 solitary wave on the truncated cone, solid walls), ``c3wm`` (the same
basin with the sinusoidal wave-maker), ``c1`` (512x64 flume with the sine wave-maker), and
``c4:<i>`` / ``c5:<i>`` for member i of the 64-member C4 or 1024-member C5 ensemble.  For
those the oracle runs member i alone, while ``gpu --case c4`` (or ``c5``) runs the whole
ensemble as one batch (the production configuration, mixed form, graphs, autotuned) and keeps
the members listed with ``--members``.  Every
``--every`` steps the FP64 total water volume (mass_full) is recorded.

Reported per form: eta RMS over the interior (m) on the free surface max(w, B) (the water level
where a cell holds water, the bed where it is dry), max |eta error| (m), the RMS of raw w as well
(it includes dry cells, where w is no surface), max run-up of each side
and its difference (run-up = highest bed elevation among initially dry cells whose recorded
maximum inundation depth exceeds 1e-3 m), relative mass difference from the FP64 oracle at the
end, max over the record, and each side's closed-basin drift |M(t) - M(0)| / M(0).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]

from celeris_b200 import cases  # noqa: E402


def build_case(name: str, n: int | None):
    if name == "c3":
        return cases.config3(n or 1024, n or 1024)
    if name == "c3wm":
        return cases.config3(n or 1024, n or 1024, wavemaker=True)
    if name == "c1":
        return cases.config1()
    if name.startswith("c4:"):
        return cases.config4()[int(name[3:])]
    if name.startswith("c5:"):
        return cases.config5(1, first_member=int(name[3:]))[0]
    raise KeyError(name)


def run_gpu_ensemble(args):
    """The 64-member C4 or 1024-member C5 ensemble as one batch; records the members in --members."""
    import celeris_b200 as cb
    members = cases.config4() if args.case == "c4" else cases.config5()
    keep = [int(k) for k in args.members.split(",")]
    form = args.forms.split(",")[0]   # the ensemble runs one form (fused or mixed)
    b = cb.Batch([(m[0], m[1]) for m in members], form)
    b.use_graph(True)
    tuned = b.autotune(4)
    # autotuning advanced the members: start over from the initial condition with the tuned setup
    b2 = cb.Batch([(m[0], m[1]) for m in members], form)
    b2.set_tuning(tuned["band_width"], tuned["strip_height"], b.col_chunks)
    b2.set_stencil_rows(b.stencil_rows)
    if b.stencil_rows == 2:
        b2.set_stencil_width(b.stencil_width)
    b2.use_graph(True)
    del b
    masses = {k: [b2.stats_current()[k]["mass_full"]] for k in keep}
    done, t0 = 0, time.time()
    while done < args.steps:
        k = min(args.every, args.steps - done)
        b2.step(k)
        done += k
        st = b2.stats_current()
        for i in keep:
            masses[i].append(st[i]["mass_full"])
    out = {}
    for i in keep:
        hi, lo = b2.state_parts(i)
        out[f"m{i}/eta"] = hi[..., 0].astype(np.float32)
        if form == "mixed":
            out[f"m{i}/eta_lo"] = lo[..., 0].astype(np.float32)
        out[f"m{i}/inundated"] = _inundated(b2.aux(i)[..., 0])
        out[f"m{i}/mass"] = np.array(masses[i])
    print(f"ensemble: {args.steps} steps in {time.time() - t0:.1f} s, tuning {tuned}", flush=True)
    np.savez_compressed(args.out, every=args.every, **out)


def run_oracle(args):
    from oracle import Oracle
    p, z, bnx, bny = build_case(args.case, args.n)
    o = Oracle(p, z, bnx, bny, real="f64")
    s0 = o.reset_timestep()
    t0 = time.time()
    masses = [s0["mass_full"]]
    done = 0
    while done < args.steps:
        k = min(args.every, args.steps - done)
        s = o.physical_steps(k)
        done += k
        masses.append(o.reset_timestep()["mass_full"])
        print(f"oracle {done}/{args.steps} steps, {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(args.out, bottom=o.bottom()[..., 2].astype(np.float32),
                        eta=o.state()[..., 0], maxdepth=o.aux()[..., 0], mass=np.array(masses),
                        every=args.every, form="fp64-oracle")


def run_gpu(args):
    if args.case in ("c4", "c5"):
        return run_gpu_ensemble(args)
    import celeris_b200 as cb
    p, z, bnx, bny = build_case(args.case, args.n)
    out = {}
    for form in args.forms.split(","):
        t0 = time.time()
        if form == "plain":
            eng = cb.Engine(p, z, "plain")
            masses = [eng.reset_timestep()["mass_full"]]
            done = 0
            while done < args.steps:
                k = min(args.every, args.steps - done)
                eng.physical_steps(k)
                done += k
                masses.append(eng.reset_timestep()["mass_full"])
            st, aux = eng.state(), eng.aux()
        else:
            b = cb.Batch([(p, z)], form)
            b.use_graph(True)
            masses = [b.stats_current()[0]["mass_full"]]
            done = 0
            while done < args.steps:
                k = min(args.every, args.steps - done)
                b.step(k)
                done += k
                masses.append(b.stats_current()[0]["mass_full"])
            st, aux = b.state(0), b.aux(0)
            hi, lo = b.state_parts(0)
            st = hi
            if form == "mixed":
                out[f"{form}/eta_lo"] = lo[..., 0].astype(np.float32)   # the compensation words
        out[f"{form}/eta"] = st[..., 0].astype(np.float32)        # w (sea level 0)
        out[f"{form}/inundated"] = _inundated(aux[..., 0])          # max inundated depth > 1 mm
        out[f"{form}/mass"] = np.array(masses)
        print(f"{form}: {args.steps} steps in {time.time() - t0:.1f} s", flush=True)
    np.savez_compressed(args.out, every=args.every, **out)


INUNDATED = 1e-3   # m: a cell counts as reached by the water once its max inundated depth passes this
FILM = 1e-4        # m: the reference's minimum depth (compute.hlsl:1062); thinner water is a film


def _inundated(maxdepth: np.ndarray) -> np.ndarray:
    """The cells whose recorded maximum inundated depth passed INUNDATED, as packed bits (small files)."""
    return np.packbits(np.asarray(maxdepth) > INUNDATED)


def _unpack(bits: np.ndarray, shape) -> np.ndarray:
    return np.unpackbits(bits)[: int(np.prod(shape))].reshape(shape).astype(bool)


def runup(bottom: np.ndarray, initial_dry: np.ndarray, reached: np.ndarray) -> float:
    wet = reached & initial_dry
    return float(bottom[wet].max()) if wet.any() else float("nan")


def compare(args):
    print(json.dumps(compare_files(args.ref, args.gpu, args.only)))


def record(args):
    """Compares several (label, FP64 record, GPU record, prefix) sets and writes them as one JSON
    record: a list of {"case", "steps", per-form results}; a label ending in "!" marks a member
    whose FP64 run itself goes non-finite (the comparison then stops at the last finite record)."""
    out = {"generated_by": "tests/long_run.py record", "entries": []}
    for spec in args.spec:
        label, ref, gpu, only = (spec.split("=", 1)[0],) + tuple(spec.split("=", 1)[1].split(","))
        res = compare_files(ref, gpu, only or None)
        res["case"] = label.rstrip("!")
        if label.endswith("!"):
            res["fp64_nonfinite"] = True
        out["entries"].append(res)
    with open(args.out, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['entries'])} entries to {args.out}")


def compare_files(ref_path: str, gpu_path: str, only: str | None) -> dict:
    ref = np.load(ref_path)
    gpu = np.load(gpu_path)
    B = ref["bottom"].astype(np.float64)
    I = (slice(2, -2), slice(2, -2))
    swl = 0.0
    initial_dry = B[I] > swl
    eta_ref = ref["eta"][I] - swl
    res = {"steps_per_record": int(ref["every"]), "records": int(len(ref["mass"]) - 1)}
    m_ref = ref["mass"]
    res["fp64_closed_basin_drift"] = float(np.max(np.abs(m_ref - m_ref[0])) / m_ref[0])
    ru_ref = runup(B[I], initial_dry, ref["maxdepth"][I] > INUNDATED)
    res["fp64_runup_m"] = ru_ref
    forms = sorted({k.split("/")[0] for k in gpu.files if "/" in k})
    if only:
        forms = [f for f in forms if f == only]
    # the free surface max(w, B): the water level where a cell holds water, the bed where it is dry
    # (below the bed, w is no surface: a sponge over dry land pulls it toward sea level)
    surf_ref = np.maximum(eta_ref + swl, B[I])
    for f in forms:
        w = gpu[f"{f}/eta"].astype(np.float64)[I]
        if f"{f}/eta_lo" in gpu.files:
            w = w + gpu[f"{f}/eta_lo"].astype(np.float64)[I]
        d = np.maximum(w, B[I]) - surf_ref
        dw = w - swl - eta_ref
        # the volume apart from films thinner than the reference's minimum depth (1e-4 m,
        # compute.hlsl:1062) in both runs: on dry land both runs gather rounding-level films (the
        # FP64 oracle moves w on every dry cell by about 1e-13 m per step from the first step on),
        # and the compensated form keeps its own, larger ones in the low words
        h_ref = np.maximum(ref["eta"][I].astype(np.float64) - B[I], 0.0)
        h_gpu = np.maximum(w - B[I], 0.0)
        film = (h_ref < FILM) & (h_gpu < FILM)
        m = gpu[f"{f}/mass"]
        n = min(len(m), len(m_ref))
        if f"{f}/inundated" in gpu.files:
            reached = _unpack(gpu[f"{f}/inundated"], B.shape)[I]
        else:
            reached = gpu[f"{f}/maxdepth"][I] > INUNDATED
        ru = runup(B[I], initial_dry, reached)
        res[f] = {
            "eta_rms_m": float(np.sqrt(np.mean(d * d))),
            "eta_max_abs_m": float(np.max(np.abs(d))),
            "w_rms_m": float(np.sqrt(np.mean(dw * dw))),
            "runup_m": ru,
            "runup_err_m": float(abs(ru - ru_ref)),
            "mass_rel_diff_end": float(abs(m[n - 1] - m_ref[n - 1]) / m_ref[n - 1]),
            "mass_rel_diff_max": float(np.max(np.abs(m[:n] - m_ref[:n]) / m_ref[:n])),
            "closed_basin_drift": float(np.max(np.abs(m - m[0])) / m[0]),
            "end_volume_rel_diff": float(abs(h_gpu.sum() - h_ref.sum()) / h_ref.sum()),
            "end_volume_rel_diff_films_excluded": float(abs(h_gpu[~film].sum() - h_ref[~film].sum()) / h_ref.sum()),
            "film_depth_sum_m": [float(h_ref[film].sum()), float(h_gpu[film].sum())],
        }
        if not np.isfinite(m_ref).all():
            last = int(np.argmax(~np.isfinite(m_ref)))
            res[f]["fp64_finite_records"] = last
    res["steps"] = int(ref["every"]) * (len(m_ref) - 1)
    return res


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("oracle", "gpu"):
        s = sub.add_parser(name)
        s.add_argument("--case", default="c3")
        s.add_argument("--n", type=int, default=None)
        s.add_argument("--steps", type=int, default=10000)
        s.add_argument("--every", type=int, default=500)
        s.add_argument("--out", required=True)
        if name == "gpu":
            s.add_argument("--forms", default="mixed,fused,plain")
            s.add_argument("--members", default="0,1,4,5,6", help="c4: ensemble members to record")
    r = sub.add_parser("record")
    r.add_argument("--out", required=True)
    r.add_argument("spec", nargs="+", help="label=ref.npz,gpu.npz,prefix (prefix may be empty)")
    c = sub.add_parser("compare")
    c.add_argument("ref")
    c.add_argument("gpu")
    c.add_argument("--only", default=None, help="compare one record prefix (e.g. m5 for C4 member 5)")
    a = ap.parse_args()
    {"oracle": run_oracle, "gpu": run_gpu, "compare": compare, "record": record}[a.cmd](a)


if __name__ == "__main__":
    main()
