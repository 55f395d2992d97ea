"""ShardedLattice (nessi_b200/lattice.py) on one GPU against the native lattice step
(nessi_gpu_lattice_2b_start / _timestep): the Python composition of k-average, exchange, Sigma_2B
and Dyson step must reproduce the library's own bit for bit.  The exchange runs through a real
one-rank NCCL process group on the library's G_loc memory (the weight is 1, so the all-reduce is
exact): the path a multi-GPU run takes, minus the other ranks (cntr_distributed_array_impl.hpp:
370-399 is what it replaces)."""
import socket

import numpy as np
import pytest

from nessi_b200 import herm_matrix, workloads

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_lattice_one_rank_matches_native(monkeypatch):
    import torch
    import torch.distributed as dist
    from nessi_b200 import gpu
    from nessi_b200.lattice import ShardedLattice
    monkeypatch.setenv("NESSI_VOLTERRA_PP", "100")  # the same Volterra kernels in both batches
    W = workloads.config4(nkx=4, nky=4, nt=70, ntau=30)
    d = W.descs[0]
    nt = d["nt"]
    native = gpu.Batch(W.descs)
    workloads.upload(native, W)
    native.lattice_2b_start(max_iter=5, tol=0.0)
    for n in range(W.k + 1, nt + 1):
        native.lattice_2b_timestep(n, W.ncorr)
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % _free_port(), rank=0, world_size=1)
    try:
        sharded = gpu.Batch(W.descs)
        workloads.upload(sharded, W)
        sl = ShardedLattice(sharded)
        sl.world = 2  # run the weighted all-reduce even though the group has one rank
        it, _ = sl.start(max_iter=5, tol=0.0)
        assert it == 6
        for n in range(W.k + 1, nt + 1):
            sl.timestep(n, W.ncorr)
        torch.cuda.synchronize()
        assert sl.exchanges == (W.k + 1) * 7 + (nt - W.k) * (W.ncorr + 1)
        for which in ("gloc", 0, W.nprob - 1):
            a = herm_matrix(nt, d["ntau"], 1, -1)
            c = herm_matrix(nt, d["ntau"], 1, -1)
            if which == "gloc":
                native.get_gloc(0, a)
                sharded.get_gloc(0, c)
            else:
                native.get_G(which, a)
                sharded.get_G(which, c)
            for comp in ("ret", "les", "tv", "mat"):
                assert np.array_equal(getattr(a, comp), getattr(c, comp)), (which, comp)
        sharded.close()
    finally:
        dist.destroy_process_group()
        native.close()
