"""The Matsubara solvers' method argument on the GPU against the oracle: dyson_mat with
CNTR_MAT_FOURIER (dyson_mat_fourier_dispatch, cntr_dyson_impl.hpp:356-446), CNTR_MAT_CG
(dyson_mat_steep_dispatch, :519-540) and the fixpoint, force_hermitian on and off (:1393-1450),
and vie2_mat with the Fourier and steepest-descent methods (cntr_vie2_impl.hpp:1229-1250).  Bar: 1e-10 relative; and
libcntr's own known answer for all three dyson_mat methods with its bounds."""
import numpy as np
import pytest

from builders import make_H, make_sigma, rand_herm, rel_err
from nessi_b200 import herm_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-10
FOURIER, CG, FIXPOINT = 0, 1, 2


def _dyson_mat_pair(oracle, s, sig, method, force_herm, ntau=24, seed=0):
    from nessi_b200 import gpu
    rng = np.random.default_rng(seed)
    nt, beta, h, mu, k = 6, 5.0, 0.05, 0.1, 5
    Sig = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h)
    H = make_H(rng, nt, s, h)
    if sig == 1:  # bosonic levels above zero
        for t in range(-1, nt + 1):
            H.data[t + 1] += 3.0 * np.eye(s)
    Go = herm_matrix(nt, ntau, s, sig)
    oracle.dyson_mat(Go, Sig, mu, H, beta, k, method=method, force_hermitian=force_herm)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=sig, solve_order=k, beta=beta, h=h, mu=mu)])
    b.set_sigma(0, Sig)
    b.set_H(0, H)
    b.dyson_mat(method, force_herm)
    Gg = herm_matrix(nt, ntau, s, sig)
    b.get_G(0, Gg)
    b.close()
    return Gg.mat, Go.mat


@pytest.mark.parametrize("s,sig", [(1, -1), (2, -1), (3, -1), (1, 1), (2, 1), (5, -1)])
def test_dyson_mat_fourier(oracle, s, sig):
    g, o = _dyson_mat_pair(oracle, s, sig, FOURIER, True, seed=11 * s + sig)
    assert rel_err(g, o) < TOL


@pytest.mark.parametrize("method", [FOURIER, FIXPOINT])
def test_dyson_mat_without_force_hermitian(oracle, method):
    g, o = _dyson_mat_pair(oracle, 2, -1, method, False, seed=5)
    assert rel_err(g, o) < TOL


def test_dyson_mat_fourier_and_fixpoint_agree(oracle):
    """Two discretisations of the same equation: close, not equal (the Fourier tail is first order)."""
    g0, _ = _dyson_mat_pair(oracle, 2, -1, FOURIER, True, ntau=200, seed=3)
    g2, _ = _dyson_mat_pair(oracle, 2, -1, FIXPOINT, True, ntau=200, seed=3)
    assert rel_err(g0, g2) < 1e-3


@pytest.mark.parametrize("s,sig", [(1, -1), (2, -1), (3, -1), (2, 1)])
def test_dyson_mat_steepest_descent(oracle, s, sig):
    g, o = _dyson_mat_pair(oracle, s, sig, CG, True, seed=17 * s + sig)
    assert rel_err(g, o) < TOL


@pytest.mark.parametrize("method,tol", [(FOURIER, 1e-3), (FIXPOINT, 1e-7), (CG, 1e-7)])
def test_dyson_mat_methods_known_answer(oracle, method, tol):
    """libcntr's own known answer (libcntr/test/matsubara.cpp:33-106) with its bounds, on the GPU."""
    from test_oracle_mat_methods import embedding_case
    from nessi_b200 import distance_norm2, gpu
    exact, Sig, h1, beta = embedding_case(oracle)
    ntau = exact.ntau
    b = gpu.Batch([dict(nt=5, ntau=ntau, size1=1, sig=-1, solve_order=5, beta=beta, h=1.0, mu=0.0)])
    b.set_sigma(0, _padded(Sig, 5))
    b.set_H(0, np.broadcast_to(h1, (7, 1, 1)).copy())
    b.dyson_mat(method)
    m = np.zeros((ntau + 1, 1, 1), np.complex128)
    b.get_timestep(0, -1, m)
    b.close()
    G = herm_matrix(-1, ntau, 1, -1)
    G.mat[...] = m
    assert distance_norm2(-1, exact, G) < tol


def _padded(S, nt):
    """A Matsubara-only herm_matrix as one with nt time steps (zero real-time components)."""
    P = herm_matrix(nt, S.ntau, S.size1, S.sig)
    P.mat[...] = S.mat
    return P


@pytest.mark.parametrize("s", [1, 2, 3])
def test_vie2_mat_steepest_descent(oracle, s):
    """vie2_mat by steepest descent (vie2_mat_steep, cntr_vie2_impl.hpp:486-600, 1241-1244) with a
    non-hermitian kernel F = -A*B and its partner Fcc = -B*A, against the oracle; without
    Fcc^mat the method is refused."""
    from nessi_b200 import gpu
    rng = np.random.default_rng(950 + s)
    nt, ntau, beta, h, k = 6, 16, 4.0, 0.05, 5
    A = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.6)
    B = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.5)
    F, Fcc = herm_matrix(nt, ntau, s, -1), herm_matrix(nt, ntau, s, -1)
    oracle.convolution_matsubara(F, A, B, beta, k)
    oracle.convolution_matsubara(Fcc, B, A, beta, k)
    F.mat[...] *= -1.0
    Fcc.mat[...] *= -1.0
    Q = herm_matrix(nt, ntau, s, -1)
    oracle.green_from_H(Q, 0.1, rand_herm(rng, s, 0.8), beta, h)
    Go = herm_matrix(nt, ntau, s, -1)
    oracle.vie2_mat(Go, F, Fcc, Q, beta, k, method=CG)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)])
    b.set_F(0, F, Fcc)
    b.set_Q(0, Q)
    b.vie2_mat(CG)
    m = np.zeros((ntau + 1, s, s), np.complex128)
    b.get_timestep(0, -1, m)
    b.close()
    assert rel_err(m, Go.mat) < TOL
    # a group given Fcc's ret and les only (no Fcc^mat) cannot run it
    L = gpu.load_library()
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)])
    gpu._check(L.nessi_gpu_set_F(b._h, 0, gpu._ptr(F.ret), gpu._ptr(F.les), gpu._ptr(F.tv), gpu._ptr(F.mat),
                                 gpu._ptr(Fcc.ret), gpu._ptr(Fcc.les)))
    b.set_Q(0, Q)
    with pytest.raises(gpu.NessiGpuError) as ei:
        b.vie2_mat(CG)
    assert ei.value.code == 1
    b.close()


@pytest.mark.parametrize("s", [1, 2, 3])
def test_vie2_mat_fourier(oracle, s):
    from nessi_b200 import gpu
    rng = np.random.default_rng(900 + s)
    nt, ntau, beta, h, k = 6, 16, 4.0, 0.05, 5
    A = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.6)
    B = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.5)
    F = herm_matrix(nt, ntau, s, -1)
    oracle.convolution_matsubara(F, A, B, beta, k)
    F.mat[...] *= -1.0
    Q = herm_matrix(nt, ntau, s, -1)
    oracle.green_from_H(Q, 0.1, rand_herm(rng, s, 0.8), beta, h)
    Go = herm_matrix(nt, ntau, s, -1)
    oracle.vie2_mat(Go, F, F, Q, beta, k, method=FOURIER)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)])
    b.set_F(0, F, F)
    b.set_Q(0, Q)
    b.vie2_mat(FOURIER)
    m = np.zeros((ntau + 1, s, s), np.complex128)
    b.get_timestep(0, -1, m)
    b.close()
    assert rel_err(m, Go.mat) < TOL
