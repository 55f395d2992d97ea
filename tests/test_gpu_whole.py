"""The whole-propagation entry points with libcntr's signatures against the oracle:
cntr::convolution (gpu.convolution: every time step from one upload, nessi_gpu_convolution_host),
cntr::dyson (gpu.dyson) and cntr::vie2 (gpu.vie2): Matsubara fixpoint, start and every time step
on the device."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import component_errors, make_H, make_sigma, rel_err, solve_oracle
from test_gpu_conv import _pair
from test_gpu_vie2 import _kernel_pair, _oracle_vie2, _source

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_whole_convolution(oracle):
    """A non-hermitian A with its partner Acc, all components of C at n = -1..nt."""
    from nessi_b200 import gpu
    rng = np.random.default_rng(11)
    nt, ntau, beta, h, k, s = 12, 10, 2.0, 0.05, 5, 2
    A, Acc = _pair(oracle, rng, nt, ntau, s, -1, beta, h, k)
    B = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.8)
    C, R = herm_matrix(nt, ntau, s, -1), herm_matrix(nt, ntau, s, -1)
    gpu.convolution(C, A, Acc, B, B, beta, h, k)
    for n in range(-1, nt + 1):
        oracle.convolution_timestep(n, R, A, Acc, B, B, beta, h, k)
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(C, comp), getattr(R, comp)) < TOL, comp


@pytest.mark.parametrize("s", [1, 2])
def test_whole_dyson(oracle, s):
    from nessi_b200 import gpu
    rng = np.random.default_rng(21 + s)
    nt, ntau, beta, h, k, mu = 20, 16, 3.0, 0.05, 5, 0.1
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    H = make_H(rng, nt, s, h)
    ref, _ = solve_oracle(oracle, herm_matrix(nt, ntau, s, -1), H, Sig, mu, beta, h, k)
    G = herm_matrix(nt, ntau, s, -1)
    gpu.dyson(G, mu, H, Sig, beta, h, k)
    assert rel_err(G.mat, ref.mat) < TOL
    e = component_errors(G, ref, 0, nt)
    assert max(e.values()) < TOL, e


def test_whole_vie2(oracle):
    from nessi_b200 import gpu
    rng = np.random.default_rng(31)
    nt, ntau, beta, h, k, s = 20, 16, 4.0, 0.05, 5, 2
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    ref, _ = _oracle_vie2(oracle, F, Fcc, Q, beta, h, k)
    G = herm_matrix(nt, ntau, s, -1)
    gpu.vie2(G, F, Fcc, Q, beta, h, k)
    assert rel_err(G.mat, ref.mat) < TOL
    e = component_errors(G, ref, 0, nt)
    assert max(e.values()) < TOL, e
