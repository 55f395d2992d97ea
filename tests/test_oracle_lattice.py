"""Oracle checks of the lattice pieces (CPU): Sigma_2B against the scalar bubble routines, its
orbital structure, and particle-number conservation of the self-consistent lattice (the second-
order local self-energy of G_loc is conserving, so sum_k n_k(t) must stay constant)."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import make_lattice, make_sigma, rel_err, u_matrices


def _scalar_sigma_2b(O, tstp, G, U):
    """Sigma_2B from the scalar Bubble1/Bubble2 routines (hubbard_chain_selfen_impl.cpp:25-75)."""
    nt, ntau = G.nt, G.ntau
    P = herm_matrix(nt, ntau, 1, 1)
    S = herm_matrix(nt, ntau, 1, -1)
    O.bubble1(tstp, P, G, G, G, G)
    P.smul(tstp, -1.0)
    u = U[:, 0]
    if tstp == -1:
        P.mat[:, 0, 0] *= u[0] * u[0]
    else:
        P.ret_row(tstp)[:, 0, 0] *= u[tstp + 1] * u[1:tstp + 2]
        P.tv[tstp, :, 0, 0] *= u[tstp + 1] * u[0]
        P.les_col(tstp)[:, 0, 0] *= u[1:tstp + 2] * u[tstp + 1]
    O.bubble2(tstp, S, G, G, P, P)
    return S


def test_sigma_2b_matches_scalar_bubbles(oracle):
    rng = np.random.default_rng(7)
    nt, ntau, beta, h = 12, 16, 4.0, 0.05
    G = make_sigma(oracle, rng, nt, ntau, 1, -1, beta, h, lam=1.0)
    U = (rng.normal(0, 1, (nt + 2, 1)) + 1j * rng.normal(0, 0.3, (nt + 2, 1)))
    S = herm_matrix(nt, ntau, 1, -1)
    for t in range(-1, nt + 1):
        oracle.sigma_2b_timestep(t, S, G, u_matrices(U))
        R = _scalar_sigma_2b(oracle, t, G, U)
        if t == -1:
            assert rel_err(S.mat, R.mat) < 1e-14
        else:
            assert rel_err(S.get_timestep(t), R.get_timestep(t)) < 1e-14


def test_sigma_2b_block_diagonal(oracle):
    """A block-diagonal G with diagonal U gives a block-diagonal Sigma whose blocks are the
    scalar Sigma_2B of each orbital."""
    rng = np.random.default_rng(8)
    nt, ntau, beta, h = 10, 12, 3.0, 0.05
    Gs = [make_sigma(oracle, rng, nt, ntau, 1, -1, beta, h, lam=1.0) for _ in range(2)]
    G = herm_matrix(nt, ntau, 2, -1)
    for i in range(2):
        G.ret[:, i, i] = Gs[i].ret[:, 0, 0]
        G.les[:, i, i] = Gs[i].les[:, 0, 0]
        G.tv[:, :, i, i] = Gs[i].tv[:, :, 0, 0]
        G.mat[:, i, i] = Gs[i].mat[:, 0, 0]
    U = rng.normal(0, 1, (nt + 2, 2)) + 0j
    S = herm_matrix(nt, ntau, 2, -1)
    for t in range(-1, nt + 1):
        oracle.sigma_2b_timestep(t, S, G, u_matrices(U))
        for i in range(2):
            R = _scalar_sigma_2b(oracle, t, Gs[i], U[:, i:i + 1])
            got = S.mat[:, i, i] if t == -1 else S.get_timestep(t)[:, i, i]
            ref = R.mat[:, 0, 0] if t == -1 else R.get_timestep(t)[:, 0, 0]
            assert rel_err(got, ref) < 1e-14
        off = S.mat[:, 0, 1] if t == -1 else S.get_timestep(t)[:, 0, 1]
        assert np.max(np.abs(off)) == 0.0


def _density_drift(O, h, nt):
    ntau, beta, k = 40, 5.0, 5
    Gs, Hs, U = make_lattice(O, 3, 3, nt, ntau, beta, h, u_max=2.0, t_ramp=0.3)
    Gloc = herm_matrix(nt, ntau, 1, -1)
    Sig = herm_matrix(nt, ntau, 1, -1)
    Um = u_matrices(U)
    it, err = O.lattice2b_start(Gs, Gloc, Sig, Um, 0.0, Hs, beta, h, k, max_iter=30, tol=1e-12)
    assert err < 1e-12
    for n in range(k + 1, nt + 1):
        O.lattice2b_timestep(n, Gs, Gloc, Sig, Um, 0.0, Hs, beta, h, k, ncorr=3)
    assert np.max(np.abs(Sig.ret_row(nt))) > 1e-3  # the interaction did something
    dens = np.array([np.imag(Gloc.les[Gloc.les_index(t, t), 0, 0]) for t in range(nt + 1)])
    return np.max(np.abs(dens - dens[0]))


def test_lattice_conserves_particle_number(oracle):
    """The drift of n(t) is a discretization error that vanishes with h (second order here,
    limited by the kink of the linear U ramp)."""
    d1 = _density_drift(oracle, 0.02, 40)
    d2 = _density_drift(oracle, 0.01, 80)
    assert d1 < 3e-5 and d2 < d1 / 3, (d1, d2)
