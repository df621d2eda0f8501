"""The multi-GPU path's host logic on CPU ranks (gloo, world size 2).

bench.py shards ensembles by domain, with no collective inside a step.  Weak scaling: rank r runs
members r*count .. r*count+count-1 of the seeded list.  Strong scaling: one fixed ensemble is split
over the ranks by cost (interior cells, largest member first to the least-loaded rank).  The job's
rate is every rank's cells over the slowest rank's time.  Here two CPU processes check the weak
shards (the right, disjoint slices of one ensemble), the strong shards (disjoint, complete and
balanced to within 5 % of the cells) and the max/sum reductions that give the job rate.
"""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    from celeris_b200 import cases
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        count = 3
        members, _ = bench.members_for("c4", rank, count)
        whole = cases.config4(count * world)
        mine = [(int(p.nx), int(p.ny), float(np.asarray(z, np.float64).sum())) for p, z, _, _ in members]
        expect = [(int(p.nx), int(p.ny), float(np.asarray(z, np.float64).sum()))
                  for p, z, _, _ in whole[rank * count:(rank + 1) * count]]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        cells = sum(p.nx * p.ny for p, _, _, _ in members)
        rate, ms_max, total = bench.job_rate(10.0 + rank, cells, 100, dist, device="cpu")
        # per-member totals of this rank's members, gathered at the end of a run
        fake = [{"mass_full": 100.0 * rank + k, "total_time": 1.5, "max_depth": 2.0, "cfl_rate": 3.0,
                 "health": 5 if (rank, k) == (1, 2) else 0} for k in range(count)]
        ens = bench.gather_member_stats(fake, dist, device="cpu")
        out.put((rank, mine == expect, gathered, cells, rate, ms_max, total, ens))
    finally:
        dist.destroy_process_group()


def test_ensemble_shards_and_job_rate():
    world, port = 2, _port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert all(r[1] for r in res)                              # each shard is its slice of the ensemble
    shards = res[0][2]
    flat = [m for shard in shards for m in shard]
    assert len(set(flat)) == len(flat)                         # disjoint members
    total = sum(r[3] for r in res)
    for r in res:                                              # every rank holds the whole ensemble's rows
        ens = r[7]
        assert ens.shape == (world * 3, 5)
        np.testing.assert_array_equal(ens[:, 0], [0, 1, 2, 100, 101, 102])
        assert int((ens[:, 4] != 0).sum()) == 1
    for _, _, _, _, rate, ms_max, tot, _ in res:
        assert ms_max == 11.0                                  # the slowest rank's time
        assert tot == total                                    # every rank's cells
        assert abs(rate - total * 100 / (11.0 / 1e3) / 1e9) < 1e-9


def _rank_strong(rank: int, world: int, port: int, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        members, _ = bench.members_for("c4", rank, 16, world, "strong")
        mine = [(int(p.nx), int(p.ny), float(np.asarray(z, np.float64).sum())) for p, z, _, _ in members]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_strong_scaling_splits_one_ensemble_by_cost():
    from celeris_b200 import cases
    from celeris_b200.shards import partition_by_cost
    world, port = 2, _port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_strong, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = res[0][1]
    assert gathered == res[1][1]                               # both ranks see the same shards
    whole = [(int(p.nx), int(p.ny), float(np.asarray(z, np.float64).sum())) for p, z, _, _ in cases.config4(16)]
    flat = [m for shard in gathered for m in shard]
    assert sorted(flat) == sorted(whole)                       # disjoint and complete
    cells = [sum(nx * ny for nx, ny, _ in shard) for shard in gathered]
    assert max(cells) <= 1.05 * sum(cells) / world             # balanced
    # the full 64-member ensemble over 2, 4 and 8 ranks
    sizes = [nx * ny for nx, ny in cases.c4_sizes(64)]
    for w in (2, 4, 8):
        shards = partition_by_cost(sizes, w)
        assert sorted(i for s in shards for i in s) == list(range(64))
        load = [sum(sizes[i] for i in s) for s in shards]
        assert max(load) <= 1.05 * sum(sizes) / w, (w, load)
