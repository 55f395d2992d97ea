"""The sharded lattice (nessi_b200.lattice) on CPU: the time-step slice extents of the libcntr
layout, the reference's block distribution of k-points, and the whole self-consistent lattice
(bootstrap + predictor/corrector steps) with its k-points split over two gloo processes against
the single-process oracle lattice.  The batch under the driver is a stand-in whose pieces are the
oracle's own routines, so these tests check the composition and the exchange, not the kernels."""
import os
import sys

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from nessi_b200 import herm_matrix
from nessi_b200.lattice import ShardedLattice, prefix_extents, shard_bounds, slice_extents
from builders import make_lattice, rel_err, u_matrices

HERE = os.path.dirname(os.path.abspath(__file__))
BETA, H, K, NCORR, NT, NTAU = 5.0, 0.02, 5, 3, 24, 16


class OracleLatticeBatch:
    """Stand-in for gpu.Batch holding the k-points [first, last) of a lattice: every method is
    the oracle routine the device batch replaces, on host herm_matrix objects."""

    def __init__(self, O, Gs, Hs, U):
        self.O, self.Gs, self.Hs, self.U = O, Gs, Hs, u_matrices(U)
        G0 = Gs[0]
        self.Gloc = herm_matrix(G0.nt, G0.ntau, G0.size1, G0.sig)
        self.Sig = herm_matrix(G0.nt, G0.ntau, G0.size1, G0.sig)

    def group_shape(self, g):
        G0 = self.Gs[0]
        return G0.nt, G0.ntau, G0.size1, K, len(self.Gs)

    def gloc_views(self, g):
        return {c: torch.from_numpy(getattr(self.Gloc, c).reshape(-1).view(np.float64)) for c in ("ret", "les", "tv", "mat")}

    def extrapolate_timestep(self, n):
        for G in self.Gs:
            self.O.extrapolate_timestep(n, G, K)

    def gloc_timestep(self, g, t):
        self.O.gloc_timestep(t, self.Gs, self.Gloc)

    def sigma_2b_timestep(self, g, t):
        self.O.sigma_2b_timestep(t, self.Sig, self.Gloc, self.U)

    def dyson_start(self):
        for G, Hk in zip(self.Gs, self.Hs):
            self.O.dyson_start(G, 0.0, Hk, self.Sig, BETA, H, K)

    def dyson_timestep(self, n):
        for G, Hk in zip(self.Gs, self.Hs):
            self.O.dyson_timestep(n, G, 0.0, Hk, self.Sig, BETA, H, K)


def _lattice(O, nkx, nky):
    return make_lattice(O, nkx, nky, NT, NTAU, BETA, H, u_max=2.0, t_ramp=0.2, u_mat=0.7)


def _oracle_reference(O, nkx, nky):
    Gs, Hs, U = _lattice(O, nkx, nky)
    Gloc, Sig = herm_matrix(NT, NTAU, 1, -1), herm_matrix(NT, NTAU, 1, -1)
    Um = u_matrices(U)
    it, err = O.lattice2b_start(Gs, Gloc, Sig, Um, 0.0, Hs, BETA, H, K, max_iter=6, tol=0.0)
    for n in range(K + 1, NT + 1):
        O.lattice2b_timestep(n, Gs, Gloc, Sig, Um, 0.0, Hs, BETA, H, K, ncorr=NCORR)
    return Gs, Gloc, it, err


def _run_shard(O, nkx, nky, first, last):
    Gs, Hs, U = _lattice(O, nkx, nky)
    b = OracleLatticeBatch(O, Gs[first:last], Hs[first:last], U)
    L = ShardedLattice(b)
    it, err = L.start(max_iter=6, tol=0.0)
    for n in range(K + 1, NT + 1):
        L.timestep(n, NCORR)
    return b, L, it, err


def test_slice_extents_follow_the_layout():
    rng = np.random.default_rng(1)
    nt, ntau, s = 7, 5, 3
    G = herm_matrix(nt, ntau, s, -1)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(G, c)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    flat = {c: getattr(G, c).reshape(-1) for c in ("ret", "les", "tv", "mat")}
    for t in range(-1, nt + 1):
        got = [flat[c][a:a + n] for c, a, n in slice_extents(t, ntau, s)]
        want = [G.mat] if t < 0 else [G.ret_row(t), G.tv[t], G.les_col(t)]
        assert len(got) == len(want)
        for x, y in zip(got, want):
            assert np.array_equal(x, y.reshape(-1))
    for k in (0, 3, nt):  # the prefix of time steps 0..k ends where slice k ends
        ends = {c: a + n for c, a, n in slice_extents(k, ntau, s)}
        assert {c: n for c, a, n in prefix_extents(k, ntau, s) if a == 0} == ends


@pytest.mark.parametrize("nk,world", [(9, 2), (1024, 8), (10, 4), (3, 3), (5, 1)])
def test_shard_bounds_cover_every_k_point(nk, world):
    b = [shard_bounds(nk, r, world) for r in range(world)]
    assert b[0][0] == 0 and b[-1][1] == nk
    assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
    sizes = [hi - lo for lo, hi in b]
    assert max(sizes) - min(sizes) <= 1
    assert sizes == sorted(sizes)  # the reference's rule: the last ranks hold the remainder


def test_single_process_driver_is_the_oracle_lattice(oracle):
    """One process: the driver's sequence of pieces is the oracle's lattice, bit for bit."""
    Gs, Gloc, it_o, err_o = _oracle_reference(oracle, 3, 3)
    b, L, it, err = _run_shard(oracle, 3, 3, 0, 9)
    assert L.world == 1 and L.exchanges == 0
    assert it == it_o == 7
    assert abs(err - err_o) <= 1e-12 * err_o + 1e-14
    for G, R in zip(b.Gs, Gs):
        for c in ("ret", "les", "tv", "mat"):
            assert np.array_equal(getattr(G, c), getattr(R, c)), c
    for c in ("ret", "les", "tv"):
        assert np.array_equal(getattr(b.Gloc, c), getattr(Gloc, c)), c


def _rank(rank, world, port, nkx, nky, out):
    import torch.distributed as dist
    for p in (HERE, os.path.join(os.path.dirname(HERE), "oracle"), os.path.dirname(HERE)):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        import oracle as O
        first, last = shard_bounds(nkx * nky, rank, world)
        b, L, it, err = _run_shard(O, nkx, nky, first, last)
        out[rank] = dict(first=first, last=last, it=it, err=err, exchanges=L.exchanges, nk_total=L.nk_total[0],
                         G=[{c: getattr(G, c).copy() for c in ("ret", "les", "tv")} for G in b.Gs],
                         Gloc={c: getattr(b.Gloc, c).copy() for c in ("ret", "les", "tv")})
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nkx,nky,world,blocks", [(3, 3, 2, [(0, 4), (4, 9)]),
                                                  (5, 2, 3, [(0, 3), (3, 6), (6, 10)])])
def test_gloo_ranks_match_the_single_process_lattice(oracle, nkx, nky, world, blocks):
    """3x3 k-points split 4 + 5 over two processes and 5x2 split 3 + 3 + 4 over three (unequal
    weights): G_loc after every exchange is the full k-average, so every G_k and G_loc equal the
    one-process oracle lattice to rounding (the partial sums are added in another order)."""
    Gs, Gloc, it_o, err_o = _oracle_reference(oracle, nkx, nky)
    port = 29611 + 7 * world + os.getpid() % 1000
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, nkx, nky, out), nprocs=world, join=True, start_method="spawn")
    res = [out[r] for r in range(world)]
    assert [(r["first"], r["last"]) for r in res] == blocks
    steps = NT - K
    for r in res:
        assert r["nk_total"] == nkx * nky
        assert r["it"] == it_o == 7
        assert abs(r["err"] - err_o) <= 1e-9 * err_o + 1e-14  # converged to rounding: ~1e-19
        # bootstrap: (k+1) slices before and after each of 7 iterations; steps: ncorr + 1 each
        assert r["exchanges"] == (K + 1) * (1 + 7) + steps * (NCORR + 1)
        for c in ("ret", "les", "tv"):
            assert rel_err(r["Gloc"][c], getattr(Gloc, c)) < 1e-13, c
        for j, G in enumerate(r["G"]):
            R = Gs[r["first"] + j]
            for c in ("ret", "les", "tv"):
                assert rel_err(G[c], getattr(R, c)) < 1e-13, c
    for c in ("ret", "les", "tv"):  # every process holds the same G_loc
        for r in res[1:]:
            assert np.array_equal(res[0]["Gloc"][c], r["Gloc"][c])


def _rank_with_failure(rank, world, port, out):
    """Rank 1 raises in the middle of the time stepping (a host-side failure); rank 0 must see its
    next exchange fail within the process group's timeout instead of waiting for ever."""
    import time
    import torch.distributed as dist
    for p in (HERE, os.path.join(os.path.dirname(HERE), "oracle"), os.path.dirname(HERE)):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    import oracle as O
    first, last = shard_bounds(9, rank, world)
    Gs, Hs, U = _lattice(O, 3, 3)
    b = OracleLatticeBatch(O, Gs[first:last], Hs[first:last], U)
    if rank == 1:
        real = b.dyson_timestep

        def failing(n):
            if n == K + 3:
                raise RuntimeError("injected failure on rank 1 at step %d" % n)
            real(n)
        b.dyson_timestep = failing
    L = ShardedLattice(b)
    L.start(max_iter=6, tol=0.0)
    t0 = time.time()
    try:
        for n in range(K + 1, NT + 1):
            L.timestep(n, NCORR)
        out[rank] = ("finished", time.time() - t0)
    except Exception as e:  # rank 1: the injected error; rank 0: the failed collective
        out[rank] = (type(e).__name__ + ": " + str(e)[:200], time.time() - t0)
        if rank == 1:
            os._exit(3)   # leave without tearing down the group, as a crashed process would
    os._exit(0)


def test_a_failing_rank_does_not_hang_the_others():
    world, port = 2, 29711 + os.getpid() % 1000
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.start_processes(_rank_with_failure, args=(world, port, out), nprocs=world, join=False,
                             start_method="spawn")
    for p in ctx.processes:
        p.join(timeout=120)
    assert all(not p.is_alive() for p in ctx.processes), "a rank is still waiting"
    for p in ctx.processes:
        if p.is_alive():
            p.kill()
    assert "injected failure" in out[1][0]
    msg, waited = out[0]
    assert msg != "finished" and waited < 60, out[0]   # rank 0's collective failed, it did not hang
    assert [p.exitcode for p in ctx.processes] == [0, 3]


def test_sharded_lattice_rejects_bad_arguments(oracle):
    """The checks nessi_gpu_lattice_2b_start / _timestep make, and the exchange sizes."""
    Gs, Hs, U = _lattice(oracle, 2, 2)
    b = OracleLatticeBatch(oracle, Gs, Hs, U)
    L = ShardedLattice(b)
    with pytest.raises(ValueError):
        L.start(max_iter=-1)
    with pytest.raises(ValueError):
        L.timestep(K, NCORR)          # n must exceed the solve order
    with pytest.raises(ValueError):
        L.timestep(K + 1, 0)          # at least one corrector
    # one time step's all-reduce: ret row, tv row and les column of G_loc
    assert L.exchange_bytes(NT) == 16 * (2 * (NT + 1) + NTAU + 1)
    assert L.exchange_bytes(-1) == 16 * (NTAU + 1)
    assert L.weight == {0: 1.0} and L.nk_total == {0: 4}
