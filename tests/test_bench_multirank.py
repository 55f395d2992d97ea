"""The multi-rank host logic of bench.py on CPU with two gloo ranks: every rank builds its own
k-grid (shifted by rank/N of a grid spacing, so the ranks' k-points are disjoint), the ranks meet
at the barriers, and the timing that is reported is the maximum over ranks."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    W = bench.build_workload("config1-small", rank, world)
    kvals = np.array([float(np.real(W.H[p, 0, 0, 0])) for p in range(W.nprob)])
    bench.barrier(world)
    t = bench.allmax(10.0 + rank, world)
    out[rank] = (kvals.tolist(), t, W.kpt_steps())
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_the_k_grid():
    world, port = 2, 29511 + os.getpid() % 1000
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    k0, t0, n0 = out[0]
    k1, t1, n1 = out[1]
    assert t0 == t1 == 11.0          # max over ranks
    assert n0 == n1 > 0              # same work per rank: weak scaling
    # diagonal of H_k(-1) is -2 cos(k): the two shifted grids share no k-point
    assert len(set(np.round(k0, 12)) & set(np.round(k1, 12))) == 0
