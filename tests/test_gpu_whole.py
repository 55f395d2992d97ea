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


def _mat_problem(oracle, seed, s, ntau, beta):
    from builders import rand_herm
    from nessi_b200 import function
    rng = np.random.default_rng(seed)
    Sig = herm_matrix(-1, ntau, s, -1)
    oracle.green_from_H(Sig, 0.0, rand_herm(rng, s, 0.7), beta, 1.0)
    Sig.smul(-1, 0.3)
    h0, mf = rand_herm(rng, s, 0.8), rand_herm(rng, s, 0.3)
    H = function(-1, s)
    H.set_value(-1, h0)
    return Sig, H, h0, mf


@pytest.mark.parametrize("s", [1, 2])
def test_dyson_mat_drop_in(oracle, s):
    """gpu.dyson_mat (cntr::dyson_mat, fixpoint) on a Matsubara-only herm_matrix (nt = -1)."""
    from nessi_b200 import gpu
    ntau, beta, k, mu = 200, 5.0, 5, 0.1
    Sig, H, _, _ = _mat_problem(oracle, 60 + s, s, ntau, beta)
    ref = herm_matrix(-1, ntau, s, -1)
    oracle.dyson_mat(ref, Sig, mu, H, beta, k)
    G = herm_matrix(-1, ntau, s, -1)
    gpu.dyson_mat(G, mu, H, Sig, beta, k)
    assert rel_err(G.mat, ref.mat) < TOL


@pytest.mark.parametrize("s", [1, 2])
def test_dyson_mat_mean_field_overload(oracle, s):
    """dyson_mat(G, mu, H, SigmaMF, Sigma, ...) (cntr_dyson_impl.hpp:472-492): against the same
    steps done by the oracle (G0 = green_from_H, F = -(G0 * Sigma + G0 SigmaMF), vie2_mat
    fixpoint, force_matsubara_hermitian), and against dyson_mat with H(-1) + SigmaMF."""
    from nessi_b200 import function, gpu
    ntau, beta, k, mu = 200, 5.0, 5, 0.1
    Sig, H, h0, mf = _mat_problem(oracle, 70 + s, s, ntau, beta)
    G0 = herm_matrix(-1, ntau, s, -1)
    oracle.green_from_H(G0, mu, h0, beta, 1.0)
    C = herm_matrix(-1, ntau, s, -1)
    oracle.convolution_matsubara(C, G0, Sig, beta, k)
    F = herm_matrix(-1, ntau, s, -1)
    F.mat[...] = -(C.mat + G0.mat @ mf)
    ref = herm_matrix(-1, ntau, s, -1)
    oracle.vie2_mat(ref, F, F, G0, beta, k)
    oracle.force_matsubara_hermitian(ref)
    G = herm_matrix(-1, ntau, s, -1)
    gpu.dyson_mat(G, mu, H, Sig, beta, k, SigmaMF=mf)
    assert rel_err(G.mat, ref.mat) < TOL
    Hmf = function(-1, s)
    Hmf.set_value(-1, h0 + mf)
    alt = herm_matrix(-1, ntau, s, -1)
    oracle.dyson_mat(alt, Sig, mu, Hmf, beta, k)
    assert rel_err(G.mat, alt.mat) < 1e-9    # the two formulations agree to the fixpoint's convergence


@pytest.mark.parametrize("s", [1, 2])
def test_dyson_mat_mean_field_steepest_descent(oracle, s):
    """dyson_mat(G, mu, H, SigmaMF, Sigma, ..., CNTR_MAT_CG) (dyson_mat_steep_dispatch with SigmaMF,
    cntr_dyson_impl.hpp:545-572): against the same steps on the oracle (F = -(G0 * Sigma + G0 SigmaMF),
    Fcc = -(Sigma * G0 + SigmaMF G0), vie2_mat steepest descent, force_matsubara_hermitian)."""
    from nessi_b200 import gpu
    ntau, beta, k, mu = 200, 5.0, 5, 0.1
    Sig, H, h0, mf = _mat_problem(oracle, 90 + s, s, ntau, beta)
    G0 = herm_matrix(-1, ntau, s, -1)
    oracle.green_from_H(G0, mu, h0, beta, 1.0)
    C, Cc = herm_matrix(-1, ntau, s, -1), herm_matrix(-1, ntau, s, -1)
    oracle.convolution_matsubara(C, G0, Sig, beta, k)
    oracle.convolution_matsubara(Cc, Sig, G0, beta, k)
    F, Fcc = herm_matrix(-1, ntau, s, -1), herm_matrix(-1, ntau, s, -1)
    F.mat[...] = -(C.mat + G0.mat @ mf)
    Fcc.mat[...] = -(Cc.mat + mf @ G0.mat)
    ref = herm_matrix(-1, ntau, s, -1)
    oracle.vie2_mat(ref, F, Fcc, G0, beta, k, method=1)
    oracle.force_matsubara_hermitian(ref)
    G = herm_matrix(-1, ntau, s, -1)
    gpu.dyson_mat(G, mu, H, Sig, beta, k, SigmaMF=mf, method=1)
    assert rel_err(G.mat, ref.mat) < TOL


def test_vie2_timestep_sin(oracle):
    """gpu.vie2_timestep_sin through a propagation (n = -1, the start at n = k, then every step)
    against the oracle's restatement of cntr_vie2_impl.hpp:1779-1838, regular part and Gsin."""
    from nessi_b200 import function, gpu
    rng = np.random.default_rng(81)
    nt, ntau, beta, h, k, s = 14, 12, 3.0, 0.05, 5, 2
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    Fsin, Qsin = function(nt, s), function(nt, s)
    for t in range(-1, nt + 1):
        Fsin.set_value(t, 0.3 * (rng.normal(size=(s, s)) + 1j * rng.normal(size=(s, s))))
        Qsin.set_value(t, rng.normal(size=(s, s)) + 1j * rng.normal(size=(s, s)))
    runs = []
    for f in (gpu.vie2_timestep_sin, oracle.vie2_timestep_sin):
        G, Gsin = herm_matrix(nt, ntau, s, -1), function(nt, s)
        for n in [-1, k] + list(range(k + 1, nt + 1)):
            f(n, G, Gsin, F, Fcc, Fsin, Q, Qsin, beta, h, k)
        runs.append((G, Gsin))
    (G, Gs), (R, Rs) = runs
    assert rel_err(Gs.data, Rs.data) < 1e-13
    for c in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(G, c), getattr(R, c)) < TOL, c
