"""The multi-GPU host logic of bench.py on two CPU ranks (gloo).

Cells shard across ranks with no exchange: each rank draws its own seeded
cells, and the job's time is the max over ranks of each rank's local time
(the only collective). Run here as two processes over gloo on 127.0.0.1,
the same helpers `bench.py --gpus N` calls under torchrun with NCCL.
"""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

import sys
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, w, local = bench.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w)
    try:
        # each rank its own shard of cells
        _, n, T, dt, par = bench.inputs(16, seed=bench.rank_seed(r))
        mine = torch.tensor([float(n.sum()), float(T.sum())], dtype=torch.float64)
        allv = [torch.zeros(2, dtype=torch.float64) for _ in range(w)]
        dist.all_gather(allv, mine)
        # the job's times: the max over ranks, per entry
        local = [1.0 + r, 10.0 - r, 0.25 * (r + 1)]
        job = bench.job_times(local, torch.device("cpu"), w)
        out.put((r, local, [v.tolist() for v in allv], job,
                 bench.job_rate(100, w, job[0])))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_cells_and_take_the_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, l0, g0, j0, v0), (r1, l1, g1, j1, v1) = res
    assert (r0, r1) == (0, 1)
    # the shards differ (distinct seeds) and every rank sees the same set
    assert g0 == g1 and g0[0] != g0[1]
    want = list(np.maximum(l0, l1))
    assert j0 == want and j1 == want
    assert v0 == v1 == 100 * world / want[0]


def test_one_rank_needs_no_collective():
    assert bench.job_times([2.5, 1.0], torch.device("cpu"), 1) == [2.5, 1.0]
    assert bench.job_rate(262144, 1, 2.0) == 131072.0
    assert bench.rank_seed(0) != bench.rank_seed(1)
