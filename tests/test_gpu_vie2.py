"""GPU parity of vie2_start / vie2_timestep ([1 + F] G = Q, cntr_vie2_impl.hpp) through the C ABI.

F = -(A * B) and Fcc = -(B * A) are convolutions of two different contour functions, so F is not
hermitian and every place where the reference switches between F and Fcc is exercised; the
problems of a group share F and have their own Q.  FP64 bar 1e-10 relative, mixed <= 1e-8.
The known-answer test is the integral form of libcntr/test/dyson.cpp:100-160 (embedding of a
two-level system), run on the GPU."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix, function
from builders import component_errors, make_sigma, rand_herm, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _kernel_pair(O, rng, nt, ntau, s, beta, h, k):
    A = make_sigma(O, rng, nt, ntau, s, -1, beta, h, lam=0.6)
    B = make_sigma(O, rng, nt, ntau, s, -1, beta, h, lam=0.5)
    F, Fcc = herm_matrix(nt, ntau, s, -1), herm_matrix(nt, ntau, s, -1)
    O.convolution_matsubara(F, A, B, beta, k)
    O.convolution_matsubara(Fcc, B, A, beta, k)
    for t in range(0, nt + 1):
        O.convolution_timestep(t, F, A, A, B, B, beta, h, k)
        O.convolution_timestep(t, Fcc, B, B, A, A, beta, h, k)
    for t in range(-1, nt + 1):
        F.smul(t, -1.0)
        Fcc.smul(t, -1.0)
    return F, Fcc


def _source(O, rng, nt, ntau, s, beta, h):
    Q = herm_matrix(nt, ntau, s, -1)
    O.green_from_H(Q, 0.1, rand_herm(rng, s, 0.8), beta, h)
    return Q


def _oracle_vie2(O, F, Fcc, Q, beta, h, k):
    G = herm_matrix(Q.nt, Q.ntau, Q.size1, -1)
    O.vie2_mat(G, F, Fcc, Q, beta, k)
    G0 = G.copy()
    O.vie2_start(G, F, Fcc, Q, beta, h, k)
    for n in range(k + 1, Q.nt + 1):
        O.vie2_timestep(n, G, F, Fcc, Q, beta, h, k)
    return G, G0


def _check(Gg, Go, k, nt, tol):
    e = component_errors(Gg, Go, 0, nt)
    worst = max(e.values())
    assert worst < tol, e
    return worst


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_vie2_matches_oracle(oracle, s):
    from nessi_b200 import gpu
    rng = np.random.default_rng(100 + s)
    nt, ntau, beta, h, k = 24, 16, 4.0, 0.05, 5
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Qs = [_source(oracle, rng, nt, ntau, s, beta, h) for _ in range(3)]
    ref = [_oracle_vie2(oracle, F, Fcc, Q, beta, h, k) for Q in Qs]
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)] * 3)
    b.set_F(0, F, Fcc)
    for p, Q in enumerate(Qs):
        b.set_Q(p, Q)
        b.set_timestep(p, -1, ref[p][1].mat)
    b.vie2_start()
    for n in range(k + 1, nt + 1):
        b.vie2_timestep(n)
    for p in range(3):
        Gg = herm_matrix(nt, ntau, s, -1)
        b.get_G(p, Gg)
        _check(Gg, ref[p][0], k, nt, TOL)
    b.close()


def test_vie2_embedding_known_answer(oracle):
    """libcntr/test/dyson.cpp integral form: G = G0 - G0*Sigma*G with Sigma = lam^2 G_2 reproduces
    the (0,0) element of the exact two-level propagator; the reference requires err/Nt < 1e-6."""
    from nessi_b200 import gpu
    O = oracle
    Nt, Ntau, dt, beta, k = 200, 400, 0.05, 10.0, 5
    eps1, eps2, lam, mu = -1.0, 1.0, 0.2, -0.1
    G2 = herm_matrix(Nt, Ntau, 2, -1)
    O.green_from_H(G2, mu, np.array([[eps1, 1j * lam], [-1j * lam, eps2]]), beta, dt)
    Gx = herm_matrix(Nt, Ntau, 1, -1)
    for t in range(-1, Nt + 1):
        Gx.set_matrixelement(t, 0, 0, G2, 0, 0)
    Sig = herm_matrix(Nt, Ntau, 1, -1)
    O.green_from_H(Sig, mu, np.array([[eps2]]), beta, dt)
    for t in range(-1, Nt + 1):
        Sig.smul(t, lam * lam)
    G0 = herm_matrix(Nt, Ntau, 1, -1)
    O.green_from_H(G0, mu, np.array([[eps1]]), beta, dt)
    F, Fcc = herm_matrix(Nt, Ntau, 1, -1), herm_matrix(Nt, Ntau, 1, -1)
    for t in range(0, Nt + 1):
        O.convolution_timestep(t, F, G0, G0, Sig, Sig, beta, dt, k)
        O.convolution_timestep(t, Fcc, Sig, Sig, G0, G0, beta, dt, k)
        F.smul(t, -1)
        Fcc.smul(t, -1)
    hf = function(Nt, 1)
    hf.set_constant(np.array([[eps1]]))
    Gm = herm_matrix(Nt, Ntau, 1, -1)
    O.dyson_mat(Gm, Sig, mu, hf, beta, k)
    b = gpu.Batch([dict(nt=Nt, ntau=Ntau, size1=1, sig=-1, solve_order=k, beta=beta, h=dt)])
    b.set_F(0, F, Fcc)
    b.set_Q(0, G0)
    b.set_timestep(0, -1, Gm.mat)
    b.vie2_start()
    for n in range(k + 1, Nt + 1):
        b.vie2_timestep(n)
    Gg = herm_matrix(Nt, Ntau, 1, -1)
    b.get_G(0, Gg)
    b.close()
    err = sum(O.distance_norm2(t, Gx, Gg) for t in range(Nt + 1))
    assert err / Nt < 1.0e-6, err / Nt
    # and the same numbers as the oracle's integral form
    Go = Gm.copy()
    O.vie2_start(Go, F, Fcc, G0, beta, dt, k)
    for n in range(k + 1, Nt + 1):
        O.vie2_timestep(n, Go, F, Fcc, G0, beta, dt, k)
    _check(Gg, Go, k, Nt, TOL)


def test_dyson_and_vie2_groups_in_one_batch(oracle):
    """One batch, a Dyson group (size 2) and a VIE2 group (size 3): each call advances its kind."""
    from nessi_b200 import gpu
    from builders import make_H, solve_oracle
    rng = np.random.default_rng(77)
    nt, ntau, beta, h, k = 20, 12, 3.0, 0.05, 5
    Sig = make_sigma(oracle, rng, nt, ntau, 2, -1, beta, h)
    H = make_H(rng, nt, 2, h)
    Gd, Gd0 = solve_oracle(oracle, herm_matrix(nt, ntau, 2, -1), H, Sig, 0.1, beta, h, k)
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, 3, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, 3, beta, h)
    Gv, Gv0 = _oracle_vie2(oracle, F, Fcc, Q, beta, h, k)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=2, sig=-1, solve_order=k, beta=beta, h=h, mu=0.1, sigma_group=0),
                   dict(nt=nt, ntau=ntau, size1=3, sig=-1, solve_order=k, beta=beta, h=h, sigma_group=1)])
    b.set_sigma(0, Sig)
    b.set_H(0, H)
    b.set_G(0, Gd0)
    b.set_F(1, F, Fcc)
    b.set_Q(1, Q)
    b.set_timestep(1, -1, Gv0.mat)
    b.vie2_start()
    for n in range(k + 1, nt + 1):
        b.dyson_timestep(n)
        b.vie2_timestep(n)
    out_d, out_v = herm_matrix(nt, ntau, 2, -1), herm_matrix(nt, ntau, 3, -1)
    b.get_G(0, out_d)
    b.get_G(1, out_v)
    b.close()
    _check(out_d, Gd, k, nt, TOL)
    _check(out_v, Gv, k, nt, TOL)


def test_vie2_mixed_precision(oracle):
    from nessi_b200 import gpu
    rng = np.random.default_rng(5)
    nt, ntau, beta, h, k, s = 80, 40, 4.0, 0.02, 5, 2
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    Go, G0 = _oracle_vie2(oracle, F, Fcc, Q, beta, h, k)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)], gpu.PREC_MIXED)
    b.set_F(0, F, Fcc)
    b.set_Q(0, Q)
    b.set_timestep(0, -1, G0.mat)
    b.vie2_start()
    for n in range(k + 1, nt + 1):
        b.vie2_timestep(n)
    Gg = herm_matrix(nt, ntau, s, -1)
    b.get_G(0, Gg)
    b.close()
    _check(Gg, Go, k, nt, 1e-8)


def test_vie2_errors():
    from nessi_b200 import gpu
    b = gpu.Batch([dict(nt=10, ntau=8, size1=1, sig=-1, solve_order=5, beta=3.0, h=0.05)])
    with pytest.raises(gpu.NessiGpuError):
        b.vie2_timestep(7)          # no VIE2 group
    F = herm_matrix(10, 8, 1, -1)
    b.set_F(0, F, F)
    with pytest.raises(gpu.NessiGpuError):
        b.vie2_start()              # Q not set
    with pytest.raises(gpu.NessiGpuError):
        b.dyson_timestep(7)         # no Dyson group left
    b.close()


@pytest.mark.parametrize("pp", [-1, 1, 4, 8, 100])
def test_vie2_problems_per_cta(oracle, monkeypatch, pp):
    """The VIE2 path of the size1 <= 2 Volterra kernels with every problems-per-CTA grouping."""
    from nessi_b200 import gpu
    monkeypatch.setenv("NESSI_VOLTERRA_PP", str(pp))
    rng = np.random.default_rng(300 + pp)
    nt, ntau, beta, h, k, s = 80, 10, 4.0, 0.05, 5, 2
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Qs = [_source(oracle, rng, nt, ntau, s, beta, h) for _ in range(5)]
    ref = [_oracle_vie2(oracle, F, Fcc, Q, beta, h, k) for Q in Qs]
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)] * 5)
    b.set_F(0, F, Fcc)
    for p, Q in enumerate(Qs):
        b.set_Q(p, Q)
        b.set_timestep(p, -1, ref[p][1].mat)
    b.vie2_start()
    for n in range(k + 1, nt + 1):
        b.vie2_timestep(n)
    for p in range(5):
        Gg = herm_matrix(nt, ntau, s, -1)
        b.get_G(p, Gg)
        _check(Gg, ref[p][0], k, nt, TOL)
    b.close()


@pytest.mark.parametrize("s", [1, 2, 3])
def test_vie2_mat_and_whole_pipeline(oracle, s):
    """vie2_mat on the GPU (fixpoint method) against the oracle, then vie2_start and vie2_timestep
    from that G^mat: the whole VIE2 propagation on the device."""
    from nessi_b200 import gpu
    rng = np.random.default_rng(500 + s)
    nt, ntau, beta, h, k = 20, 16, 4.0, 0.05, 5
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Qs = [_source(oracle, rng, nt, ntau, s, beta, h) for _ in range(2)]
    ref = [_oracle_vie2(oracle, F, Fcc, Q, beta, h, k) for Q in Qs]
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)] * 2)
    b.set_F(0, F, Fcc)
    for p, Q in enumerate(Qs):
        b.set_Q(p, Q)
    b.vie2_mat()
    for p in range(2):
        m = np.zeros((ntau + 1, s, s), np.complex128)
        b.get_timestep(p, -1, m)
        assert rel_err(m, ref[p][1].mat) < TOL
    b.vie2_start()
    for n in range(k + 1, nt + 1):
        b.vie2_timestep(n)
    for p in range(2):
        Gg = herm_matrix(nt, ntau, s, -1)
        b.get_G(p, Gg)
        _check(Gg, ref[p][0], k, nt, TOL)
    b.close()


@pytest.mark.parametrize("s", [3, 5])
@pytest.mark.parametrize("pp", [100, 101])
def test_vie2_cluster_recursion_large_orbitals(oracle, monkeypatch, s, pp):
    """The VIE2 form of the cluster and whole-GPU recursions for size1 >= 3 (element-parallel
    chains)."""
    from nessi_b200 import gpu
    monkeypatch.setenv("NESSI_VOLTERRA_PP", str(pp))
    rng = np.random.default_rng(700 + s)
    nt, ntau, beta, h, k = 30, 8, 4.0, 0.05, 5
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Qs = [_source(oracle, rng, nt, ntau, s, beta, h) for _ in range(3)]
    ref = [_oracle_vie2(oracle, F, Fcc, Q, beta, h, k) for Q in Qs]
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h)] * 3)
    b.set_F(0, F, Fcc)
    for p, Q in enumerate(Qs):
        b.set_Q(p, Q)
        b.set_timestep(p, -1, ref[p][1].mat)
    b.vie2_start()
    for n in range(k + 1, nt + 1):
        b.vie2_timestep(n)
    for p in range(3):
        Gg = herm_matrix(nt, ntau, s, -1)
        b.get_G(p, Gg)
        _check(Gg, ref[p][0], k, nt, TOL)
    b.close()
