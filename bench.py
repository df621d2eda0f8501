#!/usr/bin/env python
"""Benchmark of the Celeris Boussinesq timestep path on B200 (Gcell-steps/s).

Default workload: configuration C4 — a 64-domain uneven ensemble (sizes drawn by seed from
256^2, 512x256, 1024x512, 1024^2, 2048x512; seeded slopes, bumps and sine wave-makers) advanced
by the batched mixed-precision form (one launch per phase for the domains of each lane, each
physical step a replayed CUDA graph per lane, two lanes side by side on concurrent streams),
with correctionStepsNum = 1 (AB3 predictor + AM4 corrector).

One JSON line on rank 0:
  value     whole-job Gcell-steps/s with the state resident in HBM (device clock, CUDA events,
            max over ranks);
  e2e       the same through the public C ABI with, every step, a host->device upload of the
            per-member time steps from pinned memory and a device->host read of the step's
            statistics (mass, energy, CFL — what resetTimestep reads back every pass);
  roofline  the dominant kernel (the fused stencil) timed live with CUDA events on its stream
            (lanes one after another while timed, so each launch's span is its own);
  cpu_baseline  the FP32 transcription (OpenMP, all host threads) on a bounded sample.
``--impl reference`` times the CPU implementation of the path (the reference's own shader code
compiled for the CPU when that build is present, else the FP32 transcription) on the same
metric, over every member of the workload.  Multi-GPU (torchrun): with ``--scaling weak`` (the
default) rank r runs members r*count .. r*count+count-1 of the seeded list, so each GPU holds a
full ensemble; with ``--scaling strong`` one ensemble is split over the ranks by cost (interior
cells, largest first to the least-loaded rank).  No collective runs inside a step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c4", choices=["c4", "c2", "c3", "c5", "c1"])
    ap.add_argument("--correction-steps", type=int, default=-1, help="override correctionStepsNum (-1 keeps 1)")
    ap.add_argument("--adaptive", action="store_true", help="adaptive time steps chosen on the device")
    ap.add_argument("--form", default="mixed", choices=["mixed", "fused"])
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--lanes", type=int, default=0, help="lanes the batch is split into (0 = the library default)")
    ap.add_argument("--no-plain", action="store_true", help="skip the per-domain plain FP32 comparison")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="0 skips the CPU baseline")
    ap.add_argument("--no-graph", action="store_true", help="direct launches instead of CUDA graphs (profiling)")
    ap.add_argument("--stencil-rows", type=int, default=0, choices=[0, 1, 2],
                    help="force the stencil variant (1 or 2 rows per step) after tuning; 0 keeps the choice")
    ap.add_argument("--stencil-width", type=int, default=0, choices=[0, 96, 128],
                    help="force the stencil strip threads (with two rows per step) after tuning; 0 keeps the choice")
    ap.add_argument("--band-width", type=int, default=0, help="force the column band width after tuning (0 keeps it)")
    ap.add_argument("--strip-height", type=int, default=0, help="force the stencil strip height after tuning (0 keeps it)")
    ap.add_argument("--col-chunks", type=int, default=0,
                    help="force the column solver's chunks per column after tuning (0 keeps it; 32/64/128 with "
                         "--band-width 32: the cluster solver)")
    ap.add_argument("--tune-steps", type=int, default=6, help="steps per autotuner candidate (0 keeps the defaults)")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="weak: a full ensemble per GPU; strong: one ensemble split over the GPUs by cost")
    ap.add_argument("--accuracy-steps", type=int, default=-1,
                    help="FP64-oracle check of one sampled member after the run (-1: when the oracle can "
                         "finish it in about a minute, 0: skip)")
    return ap.parse_args()


def members_for(cfg: str, rank: int, count: int, world: int = 1, scaling: str = "weak"):
    """This rank's members and the workload's name.  Weak scaling gives every rank its own seeded
    block of `count` members; strong scaling splits one ensemble of `count` members over `world`
    ranks by cost (celeris_b200.shards)."""
    from celeris_b200 import cases
    if scaling == "strong" and cfg in ("c4", "c5"):
        from celeris_b200.shards import partition_by_cost
        sizes = cases.c4_sizes(count) if cfg == "c4" else cases.c5_sizes(count)
        mine = partition_by_cost([nx * ny for nx, ny in sizes], world)[rank]
        build = cases.config4 if cfg == "c4" else cases.config5
        return [build(1, 1, first_member=k)[0] for k in mine], \
            f"{cfg.upper()} {count}-domain ensemble split over {world} GPU(s) by cost (members {mine[0]}..)"
    if cfg == "c4":
        return cases.config4(count, 1, first_member=rank * count), \
            f"C4 {count}-domain uneven ensemble (256^2..2048x512, dx=1 m, slope+bumps, sine wave-maker, N/S solid, E sponge)"
    if cfg == "c5":
        return cases.config5(count, 1, first_member=rank * count), f"C5 {count}-domain ensemble (128..512 sides)"
    if cfg == "c2":
        return [cases.config2(member=rank)], "C2 2048^2 single domain, JONSWAP wave-maker, sponges, Manning 0.02"
    if cfg == "c1":
        return [cases.config1()], "C1 512x64 flume, dx=0.5 m, sine wave-maker, 1:20 beach"
    return [cases.config3(4096, 4096)], "C3 4096^2 single domain, solitary wave on a truncated cone"


STAT_FIELDS = ("mass_full", "total_time", "max_depth", "cfl_rate", "health")


def gather_member_stats(stats: list, dist=None, device: str = "cuda") -> np.ndarray:
    """Every rank's per-member FP64 totals (one row of STAT_FIELDS per member, ranks in order),
    gathered once at the end of a run: about 40 B per member, no collective inside a step."""
    import torch
    local = torch.tensor([[float(s[k]) for k in STAT_FIELDS] for s in stats], dtype=torch.float64, device=device)
    if dist is None:
        return local.cpu().numpy()
    parts = [torch.empty_like(local) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, local)
    return torch.cat(parts).cpu().numpy()


def job_rate(ms: float, cells: int, steps: int, dist=None, device: str = "cuda"):
    """Whole-job throughput: every rank's cells over the slowest rank's time (max over ranks)."""
    import torch
    ms_t = torch.tensor([ms], dtype=torch.float64, device=device)
    cells_t = torch.tensor([float(cells)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        dist.all_reduce(cells_t, op=dist.ReduceOp.SUM)
    ms_max, total = float(ms_t.item()), float(cells_t.item())
    return total * steps / (ms_max / 1e3) / 1e9, ms_max, total


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.path = tempfile.mktemp(suffix=".csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.index, self.q = index, q
        self.f = open(self.path, "w")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def once(self):
        """One sample now.  Called right after the timed work is queued (the GPU is busy with it),
        so that even a timed region shorter than the sampling period has a sample under load."""
        try:
            r = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.q}", "--format=csv,noheader,nounits"],
                               capture_output=True, text=True, timeout=20)
            self.f.write(r.stdout)
            self.f.flush()
        except Exception:
            pass

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(seconds: float, members):
    """FP32 transcription (OpenMP) on one representative member: cell-steps per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    # the member closest to the ensemble's mean size
    sizes = [p.nx * p.ny for p, *_ in members]
    mean = sum(sizes) / len(sizes)
    k = min(range(len(sizes)), key=lambda i: abs(sizes[i] - mean))
    p, z, bnx, bny = members[k]
    o = O.Oracle(p, z, bnx, bny, "f32")
    o.physical_steps(3)
    t = o.time_physical_steps(2)
    n = max(2, int(seconds / max(t / 2, 1e-6)))
    t = o.time_physical_steps(n)
    rate = p.nx * p.ny * n / t
    return rate, O.threads("f32"), f"{n} physical steps of one {p.nx}x{p.ny} member (FP32 transcription, OpenMP)"


def sampled_member_accuracy(batch, members, steps_cap: int):
    """The smallest member of the benchmarked batch, as it stands after every step the run took,
    against the FP64 oracle stepped as many times from the same initial condition: eta RMS over the
    interior (m) and the relative difference of the FP64 water volume.  The member's FP64 clock
    gives its step count exactly (it sums the float time step once per step).  Eta is compared on
    the free surface max(w, B), the bed standing for the surface of a dry cell.  Skipped when the
    oracle would need more than about a minute (steps_cap < 0) or more than steps_cap steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    k = min(range(len(members)), key=lambda i: members[i][0].nx * members[i][0].ny)
    p, z, bnx, bny = members[k]
    st = batch.stats_current()[k]
    dt = float(np.float32(p.timestep))
    nsteps = int(round(st["total_time"] / dt))
    o = O.Oracle(p, z, bnx, bny, "f64")
    t_probe = o.time_physical_steps(4)
    limit = steps_cap if steps_cap > 0 else int(60.0 / max(t_probe / 4, 1e-6))
    if nsteps > limit:
        return {"member": k, "steps": nsteps, "skipped": f"the FP64 oracle would need {nsteps} steps (cap {limit})"}
    o.physical_steps(nsteps - 4)
    ref = o.state()
    got = batch.state(k)
    # eta on the free surface max(w, B): the water level where there is water, the bed where dry
    bed = o.bottom()[2:-2, 2:-2, 2]
    d = np.maximum(got[2:-2, 2:-2, 0].astype(np.float64), bed) - np.maximum(ref[2:-2, 2:-2, 0], bed)
    m_ref = o.reset_timestep()["mass_full"]
    return {"member": k, "size": [int(p.nx), int(p.ny)], "steps": nsteps,
            "eta_rms_m": float(np.sqrt(np.mean(d * d))), "eta_max_abs_m": float(np.max(np.abs(d))),
            "mass_rel_diff": float(abs(st["mass_full"] - m_ref) / m_ref), "health": int(st["health"])}


def member_k(cfg: str, k: int):
    """Member k of a workload alone (without building the others)."""
    from celeris_b200 import cases
    if cfg == "c4":
        return cases.config4(1, 1, first_member=k)[0]
    if cfg == "c5":
        return cases.config5(1, 1, first_member=k)[0]
    return members_for(cfg, 0, 1)[0][0]


def _ref_worker(cfg, ks, seconds, barrier, out):
    """One process of the reference arm: the reference-shader build stepping members `ks` in turn,
    each for an equal share of `seconds` (one domain at a time per process)."""
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    import oracle as O
    barrier.wait(timeout=600)
    work, t = 0, 0.0
    for k in ks:
        p, z, bnx, bny = member_k(cfg, k)
        o = O.Oracle(p, z, bnx, bny, "ref")
        o.physical_steps(1)
        tk, steps = 0.0, 0
        while tk < seconds / len(ks) or steps == 0:
            tk += o.time_physical_steps(1)
            steps += 1
        work += p.nx * p.ny * steps
        t += tk
        del o
    out.put((ks, work, t))


def reference_pool(cfg: str, count: int, seconds: float):
    """The reference-shader build on every host core at once: one spawned process per core, the
    workload's members dealt out to them in turn (member k to process k mod cores), each process
    stepping its members one after another (the build's texture bindings are process-wide, as a D3D
    context's are, so one process runs one domain at a time).  Rate = all cell-steps / the longest
    process time."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    cores = max(1, min(len(os.sched_getaffinity(0)), count))
    barrier, out = ctx.Barrier(cores), ctx.Queue()
    shares = [list(range(c, count, cores)) for c in range(cores)]
    procs = [ctx.Process(target=_ref_worker, args=(cfg, ks, seconds, barrier, out)) for ks in shares]
    for q in procs:
        q.start()
    res = [out.get(timeout=3600) for _ in procs]
    for q in procs:
        q.join(timeout=60)
    work = sum(r[1] for r in res)
    t = max(r[2] for r in res)
    sample = (f"all {count} members, about {seconds / max(len(s) for s in shares):.1f} s of stepping each "
              f"({cores} processes at once, members dealt out in turn; the reference's compute.hlsl compiled "
              f"for the CPU)")
    return work / t, cores, sample


def reference_arm(args):
    """CPU implementation of the path on the host cores, same metric and config."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    members, workload = members_for(args.config, 0, args.members)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    kind = "port"
    # the reference's own compute.hlsl compiled for the CPU (oracle/_ref, built from the reference
    # sources), when that build is present, on all host cores
    if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref_shader.so")):
        # about 4 s of stepping per member on each process, whatever the member count
        cores = max(1, min(len(os.sched_getaffinity(0)), len(members)))
        per_proc = -(-len(members) // cores)
        rate, cores, sample = reference_pool(args.config, len(members), max(1.0, args.cpu_seconds / 3.0) * per_proc)
        kind = "reference"
    else:   # the FP32 restatement with OpenMP
        rate, cores, sample = cpu_sample(max(1.0, args.cpu_seconds), members)
    val = rate / 1e9
    out = {"metric": "Gcell-steps/s", "value": val, "unit": "Gcell-steps/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "higher_is_better": True, "dtype": "f32", "data": "synthetic",
           "config": {"workload": workload},
           "cpu_baseline": {"value": val, "unit": "Gcell-steps/s", "cores": cores, "kind": kind, "sample": sample},
           "e2e": {"value": val, "unit": "Gcell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.cuda.current_device()
    import celeris_b200 as cb

    members, workload = members_for(args.config, rank, args.members, world, args.scaling)
    for m in members:
        if args.correction_steps >= 0:
            m[0].correction_steps = args.correction_steps
        if args.adaptive:
            m[0].adaptive = 1
    batch = cb.Batch([(m[0], m[1]) for m in members], args.form, lanes=args.lanes)
    stream = torch.cuda.Stream()
    batch.set_stream(stream.cuda_stream)
    cells = batch.cells
    N = members[0][0].correction_steps
    with torch.cuda.stream(stream):
        # the autotuner times each (band width, strip height, stencil rows, stencil width) candidate
        # for a few steps; those
        # steps are warm-up too and lie outside the timed region
        batch.use_graph(not args.no_graph)
        tuned = batch.autotune(args.tune_steps) if args.tune_steps > 0 else None
        if args.stencil_rows:
            batch.set_stencil_rows(args.stencil_rows)
        if args.stencil_width:
            batch.set_stencil_width(args.stencil_width)
        if args.band_width or args.strip_height or args.col_chunks:
            batch.set_tuning(args.band_width, args.strip_height, args.col_chunks)
        batch.step(max(3, args.warmup))
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident throughput --------------------------------------------------------
    barrier()
    clk = Clocks(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    batch.step(args.steps)
    e1.record(stream)
    clk.once()   # the steps are queued and running
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    barrier()
    value, ms_max, total_cells = job_rate(ms, cells, args.steps, dist)

    # ---- end to end through the C ABI: pinned dt upload + stats readback every step -------
    n = batch.n
    dt_pinned = torch.tensor([float(np.float32(m[0].timestep)) for m in members], dtype=torch.float32).pin_memory()
    e2e_steps = args.steps
    barrier()
    t0 = time.perf_counter()
    e0.record(stream)
    # straight through the C ABI (the library's public interface), results into a caller-owned array
    lib = cb.lib()
    dt_ptr = C.cast(C.c_void_p(dt_pinned.data_ptr()), C.POINTER(C.c_float))
    stats_out = (cb.Stats * n)()
    for _ in range(e2e_steps):
        if not args.adaptive:   # an adaptive batch chooses its steps on the device
            cb.check(lib.cel_batch_set_timestep(batch.h, dt_ptr))
        cb.check(lib.cel_batch_step(batch.h, 1))
        cb.check(lib.cel_batch_stats(batch.h, stats_out))
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3)
    e2e_t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    if dist is not None:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_value = total_cells * e2e_steps / (float(e2e_t.item()) / 1e3) / 1e9
    # the whole ensemble's totals on every rank (members are sharded; each rank holds `count`)
    ens = gather_member_stats(batch.stats(), dist)
    ensemble = {"members": int(ens.shape[0]), "mass_full_sum_m3": float(ens[:, 0].sum()),
                "unhealthy_members": int((ens[:, 4] != 0).sum())}
    h2d = 0 if args.adaptive else n * 4
    # the read-back block of each lane: error flag, its members' FP64 clocks and 12 FP64 totals each
    lanes = batch.lanes
    d2h = (lanes + n + 12 * n) * 8

    # ---- roofline of the dominant kernel: per-launch CUDA events, direct launches ----------
    # (with timing on, the lanes run one after another, so each launch's span is its own; a
    # stencil launch covers one lane's cells, cells / lanes on average)
    batch.use_graph(False)
    batch.kernel_timing(True)
    kt_steps = 10
    batch.step(kt_steps)
    torch.cuda.synchronize()
    kt = batch.kernel_times()
    batch.kernel_timing(False)
    batch.use_graph(not args.no_graph)
    st_ms, st_n = kt.get("fused_stencil", (0.0, 0))
    comp = 8.0 if args.form == "mixed" else 0.0
    # the paired-row stencil rebuilds the bottom from the corner grid (4 B); the one-row stencil
    # reads BA, BX and BY (12 B)
    bottom = 0.0 if batch.stencil_rows == 2 else 8.0
    stencil_bytes_cell = ((104 + bottom + comp) + N * (128 + bottom + comp)) / (1 + N)  # average over pass kinds
    avg_launch_s = st_ms / max(st_n, 1) / 1e3
    cells_launch = cells / lanes
    achieved = stencil_bytes_cell * cells_launch / avg_launch_s / 1e9 if avg_launch_s > 0 else 0.0
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    # DRAM bytes per cell of one stencil launch measured by ncu (dram__bytes_read.sum +
    # dram__bytes_write.sum / cells) on the first 8 members of this ensemble in one lane, mixed form,
    # paired-row stencil at 96 threads per strip (corner-grid bottom): predictor 106.9, corrector
    # 132.9; scaled here to this launch's cells.
    ncu_bytes_cell = {"mixed": (106.9, 132.9)}
    traffic = None
    if args.form in ncu_bytes_cell:
        pb, cbytes = ncu_bytes_cell[args.form]
        traffic = (pb + N * cbytes) / (1 + N) * cells_launch
    total_kernel_ms = sum(v[0] for v in kt.values())
    shares = {k: round(v[0] / total_kernel_ms, 4) for k, v in kt.items()} if total_kernel_ms > 0 else {}
    step_bytes = cb.byte_model(args.form, N)[1]

    # ---- per-domain forms (the comparison): each member its own engine, launched one after another
    def per_domain(form: str, psteps: int = 30):
        engines = [cb.Engine(m[0], m[1], form) for m in members]
        for e in engines:
            e.set_stream(stream.cuda_stream)
        for e in engines:
            e.physical_steps(3)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(psteps):
            for e in engines:
                e.physical_steps(1)
        e1.record(stream)
        torch.cuda.synchronize()
        rate = cells * psteps / (e0.elapsed_time(e1) / 1e3) / 1e9
        for e in engines:
            e.close()
        return rate

    plain = fused_pd = None
    if not args.no_plain and rank == 0 and args.config in ("c4", "c5"):
        plain = per_domain("plain")          # the reference's pass structure, FP32
        fused_pd = per_domain("fused")       # this design's kernels, FP32, but one domain per launch set

    # ---- CPU leg (rank 0, N=1): the FP32 transcription timed, and the FP64 oracle as the checker
    # of one sampled member of the benchmarked batch ------------------------------------------------
    cpu = accuracy = None
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        rate, cores, sample = cpu_sample(args.cpu_seconds, members)
        cpu = {"value": rate / 1e9, "unit": "Gcell-steps/s", "cores": cores, "kind": "port", "sample": sample}
        if args.accuracy_steps != 0 and not args.adaptive:
            accuracy = sampled_member_accuracy(batch, members, args.accuracy_steps)

    if rank == 0:
        out = {
            "metric": "Gcell-steps/s", "value": value, "unit": "Gcell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": args.scaling, "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload, "form": args.form, "members_per_gpu": len(members),
                       "cells_per_gpu": cells, "correction_steps": N, "adaptive": bool(args.adaptive), "cuda_graph": not args.no_graph,
                       "l2": "working set (%.1f GB) larger than L2 (126 MB); no flush" % (
                           cells * 4 * (46 + (9 if args.form == "mixed" else 0)) / 1e9),
                       "parallelism": f"ensemble sharded by domain over {world} GPU(s)",
                       "lanes": lanes,
                       "tuning": {"column_band_width": batch.tuning[0], "strip_height": batch.tuning[1],
                                  "stencil_rows_per_step": batch.stencil_rows,
                                  "stencil_threads_per_strip": batch.stencil_width,
                                  "autotuned": tuned is not None,
                                  "pcr_switch": {
                                      "column_chunks": batch.col_chunks,
                                      "rows_per_chunk_tallest_member": -(-max(m[0].ny for m in members) // batch.col_chunks),
                                      "cluster_ctas": (batch.col_chunks // 8
                                                       if batch.tuning[0] == 32 and batch.col_chunks >= 32 else 0),
                                      "tile_transposed": batch.tuning[0] == 16 and batch.col_chunks == 1,
                                      "meaning": "column solver: L and U sweeps split into this many chunks per "
                                                 "column, each swept serially (Thomas) and joined by a scan of "
                                                 "their transfer maps (warp shuffles; with cluster_ctas > 0 "
                                                 "through the distributed shared memory of a CTA cluster, every "
                                                 "chunk held in registers)"}}},
            "e2e": {"value": e2e_value, "unit": "Gcell-steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "kernel": "fused_stencil", "peak_source": peak_src,
                         "algorithmic_bytes_per_cell": stencil_bytes_cell, "cells_per_launch": cells_launch,
                         "avg_launch_ms": avg_launch_s * 1e3},
            "step_roofline": {"bytes_per_cell_step": step_bytes,
                              "achieved_gbs": value * 1e9 * step_bytes / world / 1e9,
                              "frac": value * 1e9 * step_bytes / world / 1e9 / peak if peak else None},
            "kernel_shares": shares,
            "gpu_launches": batch.launches_per_step * args.steps,
            "ensemble": ensemble,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "plain_per_domain": plain,
            "vs_plain_per_domain": (value / world / plain) if plain else None,
            "fused_per_domain": fused_pd,
            "vs_fused_per_domain": (value / world / fused_pd) if fused_pd else None,
            "accuracy": accuracy,
        }
        print(json.dumps(out), flush=True)
    batch.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
