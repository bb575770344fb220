"""Multi-rank host logic on CPU (gloo, world size 2): the batch partition and the
max-over-ranks job time.  No GPU is involved."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from pyto_b200.batch import max_over_ranks, partition_by_dof
        lo, hi = partition_by_dof(sizes, world)[rank]
        mine = torch.tensor([lo, hi], dtype=torch.int64)
        allr = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(allr, mine)
        t = max_over_ranks(0.5 + rank)  # rank r "took" 0.5 + r seconds
        q.put((rank, [tuple(x.tolist()) for x in allr], t))
    finally:
        dist.destroy_process_group()


def test_partition_covers_each_problem_once_and_balances():
    from pyto_b200.batch import batch_shapes, partition_by_dof
    shapes = batch_shapes(64, 32, 96, seed=0)
    sizes = [3 * (a + 1) * (b + 1) * (c + 1) for a, b, c in shapes] + [8 * 3 * 129 * 65 * 65]
    for world in (1, 2, 3, 4, 8):
        parts = partition_by_dof(sizes, world)
        assert len(parts) == world
        covered = [i for lo, hi in parts for i in range(lo, hi)]
        assert covered == list(range(len(sizes)))
        loads = [sum(sizes[lo:hi]) for lo, hi in parts]
        assert max(loads) <= sum(sizes) / world + max(sizes)


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_partition_and_job_time():
    sizes = list(np.random.default_rng(0).integers(1000, 100000, 20))
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=90) for _ in range(2)]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (r0, parts0, t0), (r1, parts1, t1) = sorted(res)
    assert parts0 == parts1
    assert parts0[0][0] == 0 and parts0[0][1] == parts0[1][0] and parts0[1][1] == len(sizes)
    assert t0 == t1 == 1.5
