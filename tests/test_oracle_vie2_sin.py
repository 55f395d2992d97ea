"""The oracle's vie2_timestep_sin (cntr_vie2_impl.hpp:1779-1838: [1 + F] G = Q where F and Q carry
instantaneous parts Fsin, Qsin) and the host herm_matrix left/right multiplications it is built
from (cntr_herm_matrix_impl.hpp:2955-2995, 3206-3246).  Two limits have exact answers: without
instantaneous parts it is vie2 itself, and without the regular part of F the solution is the
time-local G = (1 + Fsin)^-1 Q, Gsin = (1 + Fsin)^-1 Qsin."""
import numpy as np

from nessi_b200 import function, herm_matrix
from builders import make_sigma, rand_herm, rel_err
from test_gpu_vie2 import _kernel_pair, _oracle_vie2, _source

NT, NTAU, BETA, H, K, S = 14, 12, 3.0, 0.05, 5, 2


def _rand_fn(rng, scale):
    f = function(NT, S)
    for t in range(-1, NT + 1):
        f.set_value(t, scale * (rng.normal(size=(S, S)) + 1j * rng.normal(size=(S, S))))
    return f


def test_left_right_multiply_follow_the_time_arguments():
    rng = np.random.default_rng(1)
    G = herm_matrix(NT, NTAU, S, -1)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(G, c)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    f = _rand_fn(rng, 1.0)
    t = 6
    L, R = G.copy(), G.copy()
    L.left_multiply(t, f, 0.5)
    R.right_multiply(t, f, 2.0)
    for m in range(t + 1):
        assert np.allclose(L.get_ret(t, m), 0.5 * f.get_value(t) @ G.get_ret(t, m))
        assert np.allclose(L.get_les(m, t), 0.5 * f.get_value(m) @ G.get_les(m, t))
        assert np.allclose(R.get_ret(t, m), 2.0 * G.get_ret(t, m) @ f.get_value(m))
        assert np.allclose(R.get_les(m, t), 2.0 * G.get_les(m, t) @ f.get_value(t))
    for m in range(NTAU + 1):
        assert np.allclose(L.get_tv(t, m), 0.5 * f.get_value(t) @ G.get_tv(t, m))
        assert np.allclose(R.get_tv(t, m), 2.0 * G.get_tv(t, m) @ f.get_value(-1))
    L.left_multiply(-1, f)
    assert np.allclose(L.mat, np.einsum("ab,mbc->mac", f.get_value(-1), G.mat))
    assert np.array_equal(L.tv[t + 1], G.tv[t + 1])   # other time steps untouched


def _propagate_sin(O, F, Fcc, Fsin, Q, Qsin):
    G, Gsin = herm_matrix(NT, NTAU, S, -1), function(NT, S)
    O.vie2_timestep_sin(-1, G, Gsin, F, Fcc, Fsin, Q, Qsin, BETA, H, K)
    O.vie2_timestep_sin(K, G, Gsin, F, Fcc, Fsin, Q, Qsin, BETA, H, K)
    for n in range(K + 1, NT + 1):
        O.vie2_timestep_sin(n, G, Gsin, F, Fcc, Fsin, Q, Qsin, BETA, H, K)
    return G, Gsin


def test_without_instantaneous_parts_it_is_vie2(oracle):
    rng = np.random.default_rng(2)
    F, Fcc = _kernel_pair(oracle, rng, NT, NTAU, S, BETA, H, K)
    Q = _source(oracle, rng, NT, NTAU, S, BETA, H)
    zero = function(NT, S)
    G, Gsin = _propagate_sin(oracle, F, Fcc, zero, Q, zero)
    ref, _ = _oracle_vie2(oracle, F, Fcc, Q, BETA, H, K)
    for c in ("ret", "les", "tv", "mat"):
        assert np.array_equal(getattr(G, c), getattr(ref, c)), c
    assert not np.any(Gsin.data)


def test_time_local_limit(oracle):
    """F = Fsin delta only: G(t,t') = (1 + Fsin(t))^-1 Q(t,t') component by component (Fsin(-1) on
    the Matsubara branch) and Gsin = (1 + Fsin)^-1 Qsin."""
    rng = np.random.default_rng(3)
    F0, Fcc0 = herm_matrix(NT, NTAU, S, -1), herm_matrix(NT, NTAU, S, -1)
    Q = _source(oracle, rng, NT, NTAU, S, BETA, H)
    Fsin, Qsin = _rand_fn(rng, 0.3), _rand_fn(rng, 1.0)
    G, Gsin = _propagate_sin(oracle, F0, Fcc0, Fsin, Q, Qsin)
    finv = np.linalg.inv(np.eye(S) + Fsin.data)
    assert rel_err(Gsin.data, np.einsum("tab,tbc->tac", finv, Qsin.data)) < 1e-13
    ref = Q.copy()
    for t in range(-1, NT + 1):
        ref.left_multiply(t, finv)
    for c in ("ret", "les", "tv"):
        assert rel_err(getattr(G, c), getattr(ref, c)) < 1e-12, c
    # the Matsubara branch goes through vie2_mat's Fourier-based start and fixpoint: rounding 1e-11
    assert rel_err(G.mat, ref.mat) < 1e-10
