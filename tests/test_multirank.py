"""The multi-GPU path's host logic on CPU ranks (gloo, world size 2).

bench.py shards the ensemble by domain: rank r runs members r*count .. r*count+count-1 of the
seeded list (weak scaling, no collective inside a step), and the job's rate is every rank's
cells over the slowest rank's time.  Here two CPU processes check both: the shards are the
right, disjoint slices of one ensemble, and the max/sum reductions give the job rate.
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
