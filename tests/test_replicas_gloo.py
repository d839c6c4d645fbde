"""The multi-GPU form is replicas only: each rank solves its own problems
(disjoint seeded phases) with no collective on the data path, and the job
time is the maximum over ranks.  Checked here with two gloo ranks on CPU."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    t = bench.max_over_ranks(10.0 + 3.0 * rank)
    ph = bench.phases(rank, 4, 64)
    dist.destroy_process_group()
    q.put((rank, t, ph))


def test_max_over_ranks_and_disjoint_replica_inputs():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(2):
        r, t, ph = q.get(timeout=120)
        out[r] = (t, ph)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 13.0
    assert not np.allclose(out[0][1], out[1][1])


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(4.5) == 4.5
