"""GPU dyson_mat (fixpoint) and dyson_start against the oracle's restatement of libcntr
(cntr_dyson_impl.hpp:1393-1535), and the whole mat -> start -> timestep pipeline on the GPU.
Bar: 1e-10 relative per component."""
import numpy as np
import pytest

from builders import make_H, make_sigma, rel_err, component_errors
from nessi_b200 import herm_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _setup(oracle, s, nt, ntau, sig, seed, beta=5.0, h=0.05, mu=0.1):
    rng = np.random.default_rng(seed)
    Sig = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h)
    H = make_H(rng, nt, s, h)
    if sig == 1:  # keep bosonic levels positive
        for t in range(-1, nt + 1):
            H.data[t + 1] += 3.0 * np.eye(s)
    return Sig, H, beta, h, mu


@pytest.mark.parametrize("s,sig", [(1, -1), (2, -1), (3, -1), (2, 1), (5, -1)])
def test_dyson_mat_and_start(oracle, s, sig):
    from nessi_b200 import gpu
    nt, ntau, k = 10, 20, 5
    Sig, H, beta, h, mu = _setup(oracle, s, nt, ntau, sig, seed=7 * s + sig)
    Go = herm_matrix(nt, ntau, s, sig)
    oracle.dyson_mat(Go, Sig, mu, H, beta, k)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=sig, solve_order=k, beta=beta, h=h, mu=mu)])
    b.set_sigma(0, Sig)
    b.set_H(0, H)
    b.dyson_mat()
    Gg = herm_matrix(nt, ntau, s, sig)
    b.get_G(0, Gg)
    e_mat = rel_err(Gg.mat, Go.mat)
    # dyson_start from the same (oracle) Matsubara function
    oracle.dyson_start(Go, mu, H, Sig, beta, h, k)
    Gs = herm_matrix(nt, ntau, s, sig)
    Gs.mat[...] = Go.mat
    b.set_G(0, Gs)
    b.dyson_start()
    b.get_G(0, Gs)
    e = component_errors(Gs, Go, 0, k)
    print("s=%d sig=%d mat %.2e start %s" % (s, sig, e_mat, e))
    b.close()
    assert e_mat < TOL
    for c, v in e.items():
        assert v < TOL, (c, v)


def test_full_pipeline_on_gpu(oracle):
    from nessi_b200 import gpu
    s, nt, ntau, k, sig = 2, 30, 20, 5, -1
    Sig, H, beta, h, mu = _setup(oracle, s, nt, ntau, sig, seed=99)
    Go = herm_matrix(nt, ntau, s, sig)
    oracle.dyson_mat(Go, Sig, mu, H, beta, k)
    oracle.dyson_start(Go, mu, H, Sig, beta, h, k)
    for n in range(k + 1, nt + 1):
        oracle.dyson_timestep(n, Go, mu, H, Sig, beta, h, k)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=sig, solve_order=k, beta=beta, h=h, mu=mu)] * 2)
    b.set_sigma(0, Sig)
    for p in range(2):
        b.set_H(p, H)
    b.dyson_mat()
    b.dyson_start()
    for n in range(k + 1, nt + 1):
        b.dyson_timestep(n)
    for p in range(2):
        Gg = herm_matrix(nt, ntau, s, sig)
        b.get_G(p, Gg)
        assert rel_err(Gg.mat, Go.mat) < TOL
        for c, v in component_errors(Gg, Go, 0, nt).items():
            assert v < TOL, (c, v)
    b.close()
