"""Self-consistent lattice (Sigma_2B of the k-averaged G_loc) with its k-points sharded over
processes, one per GPU.

libcntr's lattice programs block-distribute the k-points over MPI ranks
(cntr_distributed_array_impl.hpp:95-125) and, before every self-energy evaluation, gather the
current time-step slice of all k-points on every rank with MPI_Allgatherv
(cntr_distributed_array_impl.hpp:370-399, driven from gw_selfene_impl.cpp:18-28).  The
second-order local self-energy reads only the k-average G_loc (hubbard_chain_selfen_impl.cpp:
63-75), so here each process averages its own k-points on its GPU (``nessi_gpu_gloc_timestep``)
and the processes add the slices weighted by their share of the k-points with ONE all-reduce of
2(n+1)+ntau+1 elements of s^2 complex numbers (NCCL over NVLink, gloo on CPU), instead of
gathering Nk slices.  Every process then forms the same Sigma_2B and advances its own k-points.

The step sequence is the one of ``nessi_gpu_lattice_2b_start`` / ``nessi_gpu_lattice_2b_timestep``
(hubbard_chain_2b.cpp:245-290 and 306-324 with G -> G_loc), with an exchange after every G_loc
evaluation; the bootstrap's convergence distance is maximised over the processes, like the
MPI_Allreduce of the errors in gw.cpp:416-417, so that every process takes the same branch and
all collectives match.

The batch object needs: ``group_shape(g)``, ``gloc_views(g)`` (tensors aliasing G_loc in the
libcntr layout), ``extrapolate_timestep``, ``gloc_timestep``, ``sigma_2b_timestep``,
``dyson_start``, ``dyson_timestep`` and, for a device batch, ``set_stream``.
"""
from __future__ import annotations


def slice_extents(tstp: int, ntau: int, size1: int):
    """[(component, first, count)] in complex numbers of time step tstp of a herm_matrix stored in
    libcntr's layout (cntr_herm_matrix_impl.hpp:457-477): ret(tstp, 0..tstp), tv(tstp, 0..ntau),
    les(0..tstp, tstp) -- each contiguous -- or the whole mat for tstp = -1."""
    s2 = size1 * size1
    if tstp < 0:
        return [("mat", 0, (ntau + 1) * s2)]
    tri = tstp * (tstp + 1) // 2
    return [("ret", tri * s2, (tstp + 1) * s2), ("tv", tstp * (ntau + 1) * s2, (ntau + 1) * s2),
            ("les", tri * s2, (tstp + 1) * s2)]


def prefix_extents(k: int, ntau: int, size1: int):
    """Time steps 0..k of ret, les and tv: the prefixes [(component, 0, count)] in complex numbers."""
    s2 = size1 * size1
    tri = (k + 1) * (k + 2) // 2
    return [("ret", 0, tri * s2), ("les", 0, tri * s2), ("tv", 0, (k + 1) * (ntau + 1) * s2)]


def _cut(views, extents):
    return [views[c][2 * a:2 * (a + n)] for c, a, n in extents]


class ShardedLattice:
    """The lattice start and time step of one batch, its G_loc summed over the processes of
    ``process_group`` (None: the default group; a single process needs no exchange)."""

    def __init__(self, batch, groups=(0,), process_group=None, stream=None):
        import torch
        import torch.distributed as dist
        self.b, self.groups, self.pg = batch, tuple(groups), process_group
        self.world = dist.get_world_size(process_group) if dist.is_available() and dist.is_initialized() else 1
        self.shape = {g: batch.group_shape(g) for g in self.groups}
        ks = {self.shape[g][3] for g in self.groups}
        if len(ks) != 1:
            raise ValueError("sharded lattice: the groups must share one solve order")
        self.k = ks.pop()
        self.views = {g: batch.gloc_views(g) for g in self.groups}
        self.device = next(iter(self.views[self.groups[0]].values())).device
        self.stream = None
        if self.device.type == "cuda":
            # the library and the exchange share one (non-default) stream, so the all-reduce is
            # ordered after the k-average and before Sigma_2B without a host synchronisation
            self.stream = stream if stream is not None else torch.cuda.Stream(device=self.device)
            batch.set_stream(self.stream.cuda_stream)
        local = torch.tensor([float(self.shape[g][4]) for g in self.groups], dtype=torch.float64, device=self.device)
        total = local.clone()
        if self.world > 1:
            with self._on_stream():
                dist.all_reduce(total, group=self.pg)
        self.weight = {g: float(local[i] / total[i]) for i, g in enumerate(self.groups)}
        self.nk_total = {g: int(round(float(total[i]))) for i, g in enumerate(self.groups)}
        longest = max(2 * (2 * (s[0] + 1) + s[1] + 1) * s[2] * s[2] for s in self.shape.values())
        self._buf = torch.empty(longest, dtype=torch.float64, device=self.device)
        self.exchanges = 0

    def _on_stream(self):
        import contextlib
        import torch
        return torch.cuda.stream(self.stream) if self.stream is not None else contextlib.nullcontext()

    # ---- the exchange --------------------------------------------------------------------
    def exchange(self, g, tstp):
        """G_loc(tstp) of group g <- sum over processes of (P_rank / P_total) G_loc_rank(tstp)."""
        if self.world == 1:
            return
        import torch
        import torch.distributed as dist
        _, ntau, s, _, _ = self.shape[g]
        parts = _cut(self.views[g], slice_extents(tstp, ntau, s))
        n = sum(p.numel() for p in parts)
        buf = self._buf[:n]
        with self._on_stream():
            o = 0
            for p in parts:
                torch.mul(p, self.weight[g], out=buf[o:o + p.numel()])
                o += p.numel()
            dist.all_reduce(buf, group=self.pg)
            o = 0
            for p in parts:
                p.copy_(buf[o:o + p.numel()])
                o += p.numel()
        self.exchanges += 1

    def _gloc(self, g, tstp):
        self.b.gloc_timestep(g, tstp)
        self.exchange(g, tstp)

    # ---- bootstrap and time step -----------------------------------------------------------
    def _snapshot(self):
        import torch
        with self._on_stream():
            return [torch.cat(_cut(self.views[g], prefix_extents(self.k, self.shape[g][1], self.shape[g][2])))
                    for g in self.groups]

    def _distance(self, cur, prev):
        """sum over t = 0..k of distance_norm2(t) (cntr_utilities_impl.hpp:607-650): every
        element's Frobenius norm of the difference, summed, maximised over the processes."""
        import torch
        import torch.distributed as dist
        with self._on_stream():
            err = torch.zeros((), dtype=torch.float64, device=self.device)
            for g, c, p in zip(self.groups, cur, prev):
                s2 = self.shape[g][2] ** 2
                d = (c - p).view(-1, 2 * s2)
                err = err + torch.sqrt((d * d).sum(dim=1)).sum()
            if self.world > 1:
                dist.all_reduce(err, op=dist.ReduceOp.MAX, group=self.pg)
            return float(err)

    def start(self, max_iter=20, tol=1e-12):
        """Bootstrap of time steps 0..k; returns (iterations, last distance), as
        nessi_gpu_lattice_2b_start."""
        if max_iter < 0:
            raise ValueError("lattice start: max_iter < 0")
        k = self.k
        for g in self.groups:
            for t in range(k + 1):
                self._gloc(g, t)
        prev = self._snapshot()
        err = 0.0
        for it in range(max_iter + 1):
            for g in self.groups:
                for t in range(k + 1):
                    self.b.sigma_2b_timestep(g, t)
            self.b.dyson_start()
            for g in self.groups:
                for t in range(k + 1):
                    self._gloc(g, t)
            cur = self._snapshot()
            err = self._distance(cur, prev)
            if err < tol and it > 2:
                return it + 1, err
            prev = cur
        return max_iter + 1, err

    def timestep(self, n, corrector_steps=3):
        """Predictor (extrapolation of step n from n-1-k..n-1) and corrector_steps x [G_loc(n),
        exchange, Sigma_2B(n), dyson_timestep(n)], then the final G_loc(n), as
        nessi_gpu_lattice_2b_timestep."""
        if corrector_steps < 1:
            raise ValueError("lattice timestep: corrector_steps must be >= 1")
        if n <= self.k:
            raise ValueError("lattice timestep: n = %d must exceed the solve order %d" % (n, self.k))
        self.b.extrapolate_timestep(n - 1)
        for _ in range(corrector_steps):
            for g in self.groups:
                self._gloc(g, n)
                self.b.sigma_2b_timestep(g, n)
            self.b.dyson_timestep(n)
        for g in self.groups:
            self._gloc(g, n)

    def exchange_bytes(self, tstp):
        """Bytes one process contributes to the all-reduces of time step tstp (all groups)."""
        return sum(16 * sum(c for _, _, c in slice_extents(tstp, s[1], s[2])) for s in self.shape.values())


def shard_bounds(nk: int, rank: int, world: int):
    """Block distribution of nk k-points over world processes, [first, last): process i takes
    floor(remaining / (world - i)) of the k-points left, so the last nk % world processes hold
    one more (the tid_map of cntr_distributed_array_impl.hpp:114-128)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("shard_bounds: rank %d of %d" % (rank, world))
    first = 0
    for i in range(world):
        size = (nk - first) // (world - i)
        if i == rank:
            return first, first + size
        first += size
    raise AssertionError("unreachable")


__all__ = ["ShardedLattice", "slice_extents", "prefix_extents", "shard_bounds"]
