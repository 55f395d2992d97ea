"""Synthetic inputs with the shapes of the benchmark configurations.

Each builder returns a ``Workload``: one shared self-energy Sigma, per-problem Hamiltonians
H_k(t) (cntr::function layout, t = -1 first), the bootstrap time steps (mat and 0..k) of every
G_k, and the batch descriptors.  All values are generated from formulas and seeds; no dataset
is involved.

chain2 (2-band chain, size1 = 2, Nk k-points in [-pi, pi)):
    h_k(t) = [[-2cos(k - A(t)), 0.5], [0.5, 1 - 2cos(k - A(t))]],
    A(t) = exp(-(t-5)^2/2) sin(3t),  H(-1) at A = 0,
    Sigma = V^2 G_bath (x) 1_2 with V = 0.5, G_bath a semicircular bath (half-bandwidth 2,
    201 levels), shared by all k.
chain4 (4-band chain, size1 = 4): diagonal -2cos(k - A) + eps_a, eps = (-1.5, -0.5, 0.5, 1.5),
    nearest-band hoppings 0.3, same Sigma (x) 1_4.
uneven (independent problems of mixed orbital size and length): size1 drawn from {1,2,3,5,8} and
    nt from U[500, 3000] with a seed; h = (X + X^H)/2, X complex N(0, 0.5^2); a rank-1 quench
    u u^H (u complex N(0, 0.3^2)) switched on at t = 0; Sigma = 0.49 G_bath (x) 1_s shared by the
    problems of one size (sigma_group = size1).  Every problem is a Dyson problem: VIE2 problems
    would each carry a source term Q as large as G, which does not fit next to ~150 GB of G.
impurity (config 0): one size1 = 1 level quenched from 0 to 1 at t = 0 in the semicircular bath
    with V = 1, beta = 10, nt = 200, ntau = 400, h = 0.02.
lattice2b (square lattice, size1 = 1, nkx x nky k-points in [-pi, pi)^2):
    eps_k = -2(cos kx + cos ky), mu = 0 (half filling), free equilibrium (U = 0 on the Matsubara
    branch), U(t) = min(t, 2) switched on at t = 0; Sigma = Sigma_2B[G_loc, U] recomputed from the
    k-average every corrector iteration.
"""
import numpy as np

from . import equilibrium as eq
from .herm_matrix import herm_matrix


class Workload:
    lattice = False  # True: Sigma_2B of G_loc, recomputed each step (U, ncorr set)
    U = None
    ncorr = 0

    def __init__(self, name, descs, sigma, H, boot, k, info):
        self.name = name
        self.descs = descs          # list of batch descriptors
        self.sigma = sigma          # herm_matrix of sigma_group 0, or {sigma_group: herm_matrix}
        self.H = H                  # (nprob, nt+2, s, s)
        self.boot = boot            # list of herm_matrix(nt=k) with mat and steps 0..k per problem
        self.k = k
        self.info = info

    @property
    def nprob(self):
        return len(self.descs)

    def kpt_steps(self):
        return sum(d["nt"] - self.k for d in self.descs)


def peierls(t):
    return np.exp(-(t - 5.0) ** 2 / 2.0) * np.sin(3.0 * t)


def chain_H(kvals, nt, h, eps_band, hop):
    """H_k(t) for a chain with band offsets eps_band and inter-band hopping matrix hop."""
    s = len(eps_band)
    nk = len(kvals)
    H = np.zeros((nk, nt + 2, s, s), np.complex128)
    times = np.concatenate([[None], np.arange(nt + 1) * h])
    for it, t in enumerate(times):
        A = 0.0 if t is None else peierls(t)
        for a in range(s):
            H[:, it, a, a] = -2.0 * np.cos(kvals - A) + eps_band[a]
        H[:, it] += hop
    return H


def bootstrap_free(H0, mu, beta, h, k, ntau, sig=-1):
    """Time steps -1..k of the free propagator of H0 (the interim bootstrap of the benchmark)."""
    s = H0.shape[0]
    G = herm_matrix(k, ntau, s, sig)
    eq.green_from_H(G, mu, H0, beta, h)
    return G


def chain(nk, nt, ntau, beta, h, size1, k=5, V=0.5, mu=0.0, kshift=0.0, kslice=None):
    if size1 == 2:
        eps_band = np.array([0.0, 1.0])
        hop = np.array([[0, 0.5], [0.5, 0]], np.complex128)
    elif size1 == 4:
        eps_band = np.array([-1.5, -0.5, 0.5, 1.5])
        hop = np.zeros((4, 4), np.complex128)
        for a in range(3):
            hop[a, a + 1] = hop[a + 1, a] = 0.3
    else:
        raise ValueError("chain workloads have size1 2 or 4")
    kvals = -np.pi + 2 * np.pi * np.arange(nk) / nk + kshift
    if kslice is not None:  # one chunk of the k-grid (the grid is propagated chunk by chunk)
        kvals = kvals[kslice]
    H = chain_H(kvals, nt, h, eps_band, hop)
    Gb = eq.semicircle_bath(nt, ntau, beta, h)
    sigma = eq.kron_identity(Gb, size1, V * V)
    boot = []
    cache = {}
    for i in range(len(kvals)):
        key = H[i, 0].tobytes()
        if key not in cache:
            cache[key] = bootstrap_free(H[i, 0], mu, beta, h, k, ntau)
        boot.append(cache[key])
    descs = [dict(nt=nt, ntau=ntau, size1=size1, sig=-1, solve_order=k, sigma_group=0, beta=beta, h=h, mu=mu)
             for _ in range(len(kvals))]
    info = dict(model="%d-band chain" % size1, size1=size1, nk=nk, nt=nt, ntau=ntau, beta=beta, h=h,
                solve_order=k, sigma="V^2 G_bath (x) 1, V=%g, shared" % V)
    if kslice is not None:
        info["k_chunk"] = "k-points %d..%d of %d (one chunk; G of the whole grid is 2.5 TB)" % (
            kslice.start, kslice.stop - 1, nk)
    return Workload("chain%d" % size1, descs, sigma, H, boot, k, info)


def config0(nt=200, ntau=400, beta=10.0, h=0.02, k=5, V=1.0, eps0=1.0):
    """Impurity quench, the CPU-sized case: one size1 = 1 level quenched from 0 to eps0 at t = 0
    (H(-1) = 0, H(t >= 0) = eps0), coupled with V = 1 to the semicircular bath (half-bandwidth 2,
    201 levels): Sigma = V^2 G_bath; beta = 10, nt = 200, ntau = 400, h = 0.02.  The bootstrap
    given here is the free propagator of H(-1); the parity test solves dyson_mat and dyson_start
    on the device instead."""
    H = np.zeros((1, nt + 2, 1, 1), np.complex128)
    H[0, 1:, 0, 0] = eps0
    sigma = eq.kron_identity(eq.semicircle_bath(nt, ntau, beta, h), 1, V * V)
    boot = [bootstrap_free(H[0, 0], 0.0, beta, h, k, ntau)]
    descs = [dict(nt=nt, ntau=ntau, size1=1, sig=-1, solve_order=k, sigma_group=0, beta=beta, h=h, mu=0.0)]
    info = dict(model="impurity level quenched 0 -> %g in a semicircular bath" % eps0, size1=1, nk=1, nt=nt,
                ntau=ntau, beta=beta, h=h, solve_order=k, sigma="V^2 G_bath, V=%g" % V)
    return Workload("impurity", descs, sigma, H, boot, k, info)


def config1(nk=256, nt=1000, ntau=600, kshift=0.0):
    """Plain method batched over k, FP64: 2-band chain, Nk=256, nt=1000, ntau=600, beta=20, h=0.01."""
    return chain(nk, nt, ntau, 20.0, 0.01, 2, kshift=kshift)


def config2(nk=512, nt=4000, ntau=800, kshift=0.0, chunk=32, chunk_index=0):
    """4-band chain, Nk=512, nt=4000, ntau=800, beta=20, h=0.01, propagated in chunks of `chunk`
    k-points (one chunk: 32 x 4.1 GB of G)."""
    sl = slice(chunk_index * chunk, min(nk, (chunk_index + 1) * chunk))
    return chain(nk, nt, ntau, 20.0, 0.01, 4, kshift=kshift, kslice=sl)


def lattice2b(nkx, nky, nt, ntau, beta, h, u_max=2.0, t_ramp=2.0, ncorr=3, k=5, kshift=0.0):
    """Self-consistent square lattice with the local second-order self-energy."""
    kx = -np.pi + 2 * np.pi * np.arange(nkx) / nkx + kshift
    ky = -np.pi + 2 * np.pi * np.arange(nky) / nky
    eps = np.array([-2.0 * (np.cos(a) + np.cos(b)) for a in kx for b in ky])
    nk = len(eps)
    H = np.zeros((nk, nt + 2, 1, 1), np.complex128)
    H[:, :, 0, 0] = eps[:, None]
    sigma = herm_matrix(nt, ntau, 1, -1)
    boot, cache = [], {}
    for i in range(nk):
        key = round(float(eps[i]), 14)
        if key not in cache:
            cache[key] = bootstrap_free(H[i, 0], 0.0, beta, h, k, ntau)
        boot.append(cache[key])
    descs = [dict(nt=nt, ntau=ntau, size1=1, sig=-1, solve_order=k, sigma_group=0, beta=beta, h=h, mu=0.0)
             for _ in range(nk)]
    info = dict(model="square lattice, local Sigma_2B[G_loc]", size1=1, nk=nk, nkx=nkx, nky=nky, nt=nt, ntau=ntau,
                beta=beta, h=h, solve_order=k, correctors=ncorr,
                sigma="U(t)U(t') G_loc(t,t')^2 G_loc(t',t), U(t) = %g min(t/%g, 1), U = 0 on the Matsubara branch"
                      % (u_max, t_ramp))
    W = Workload("lattice2b", descs, sigma, H, boot, k, info)
    W.lattice = True
    W.ncorr = ncorr
    U = np.zeros((nt + 2, 1), np.complex128)
    U[1:, 0] = u_max * np.minimum(np.arange(nt + 1) * h / t_ramp, 1.0)
    W.U = U
    return W


def config4(nkx=32, nky=32, nt=2000, ntau=800, kshift=0.0):
    """32x32 square lattice, size1 = 1, nt = 2000, ntau = 800, beta = 20, h = 0.01, 3 correctors."""
    return lattice2b(nkx, nky, nt, ntau, 20.0, 0.01, kshift=kshift)


def uneven(nprob=96, sizes=(1, 2, 3, 5, 8), nt_range=(500, 3000), ntau=400, beta=10.0, h=0.01, k=5, V=0.7,
           seed=20261203):
    """Config 3: independent problems of uneven size and length in one batch (groups by size)."""
    rng = np.random.default_rng(seed)
    s_list = [int(rng.choice(sizes)) for _ in range(nprob)]
    nt_list = [int(rng.integers(nt_range[0], nt_range[1] + 1)) for _ in range(nprob)]
    H, boot, descs = [], [], []
    for s, nt in zip(s_list, nt_list):
        x = rng.normal(0, 0.5, (s, s)) + 1j * rng.normal(0, 0.5, (s, s))
        h0 = (x + x.conj().T) / 2
        u = rng.normal(0, 0.3, s) + 1j * rng.normal(0, 0.3, s)
        Hp = np.zeros((nt + 2, s, s), np.complex128)
        Hp[0] = h0
        Hp[1:] = h0 + np.outer(u, u.conj())
        H.append(Hp)
        boot.append(bootstrap_free(h0, 0.0, beta, h, k, ntau))
        descs.append(dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, sigma_group=s, beta=beta, h=h, mu=0.0))
    Gb = eq.semicircle_bath(max(nt_list), ntau, beta, h)
    sigma = {}
    for s in sorted(set(s_list)):
        ntg = max(nt for ss, nt in zip(s_list, nt_list) if ss == s)
        Gs = herm_matrix(ntg, ntau, 1, -1)
        Gs.ret[...] = Gb.ret[:Gs.ret.shape[0]]
        Gs.les[...] = Gb.les[:Gs.les.shape[0]]
        Gs.tv[...] = Gb.tv[:ntg + 1]
        Gs.mat[...] = Gb.mat
        sigma[s] = eq.kron_identity(Gs, s, V * V)
    info = dict(model="uneven batch of independent Dyson problems", nprob=nprob, sizes=list(sizes),
                nt_range=list(nt_range), ntau=ntau, beta=beta, h=h, solve_order=k, seed=seed,
                size1_counts={str(s): s_list.count(s) for s in sorted(set(s_list))},
                sigma="V^2 G_bath (x) 1_s, V=%g, shared per size1" % V)
    W = Workload("uneven", descs, sigma, H, boot, k, info)
    return W


def config3(**kw):
    """96 problems, size1 in {1,2,3,5,8}, nt in [500, 3000], ntau = 400, beta = 10, h = 0.01."""
    return uneven(**kw)


def upload(batch, W):
    """Copy Sigma, H and the bootstrap steps of a workload into a gpu.Batch."""
    if isinstance(W.sigma, dict):
        for grp, S in W.sigma.items():
            batch.set_sigma(grp, S)
    else:
        batch.set_sigma(0, W.sigma)
    for p in range(W.nprob):
        batch.set_H(p, W.H[p])
        B = W.boot[p]
        batch.set_timestep(p, -1, B.mat)
        for t in range(W.k + 1):
            batch.set_timestep(p, t, B.get_timestep(t))
    if W.lattice:
        batch.set_U(0, W.U)
