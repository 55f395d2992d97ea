"""Parity of the CUDA dyson_timestep (through the C ABI) with the oracle's restatement of
libcntr's serial dyson_timestep (cntr_dyson_impl.hpp:1618-1648).  Bar: FP64 path within
1e-10 relative (max |x - x_ref| / max |x_ref| per component) on every time step."""
import numpy as np
import pytest

from builders import make_H, make_sigma, solve_oracle, component_errors
from nessi_b200 import herm_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _run(oracle, s, nt_list, ntau, sig=-1, beta=5.0, h=0.05, k=5, mu=0.1, seed=0):
    from nessi_b200 import gpu
    rng = np.random.default_rng(seed)
    ntmax = max(nt_list)
    Sig = make_sigma(oracle, rng, ntmax, ntau, s, sig, beta, h)
    Hs, Go, G0 = [], [], []
    for nt in nt_list:
        H = make_H(rng, nt, s, h)
        S_p = herm_matrix(nt, ntau, s, sig)   # Sigma restricted to this problem's nt
        S_p.mat[...] = Sig.mat
        S_p.ret[...] = Sig.ret[:S_p.ret.shape[0]]
        S_p.les[...] = Sig.les[:S_p.les.shape[0]]
        S_p.tv[...] = Sig.tv[:nt + 1]
        G = herm_matrix(nt, ntau, s, sig)
        Gf, Gb = solve_oracle(oracle, G, H, S_p, mu, beta, h, k)
        Hs.append(H); Go.append(Gf); G0.append(Gb)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=sig, solve_order=k, beta=beta, h=h, mu=mu)
                   for nt in nt_list])
    b.set_sigma(0, Sig)
    for p in range(len(nt_list)):
        b.set_G(p, G0[p])
        b.set_H(p, Hs[p])
    for n in range(k + 1, ntmax + 1):
        b.dyson_timestep(n)
    b.synchronize()
    errs = []
    for p, nt in enumerate(nt_list):
        Gg = herm_matrix(nt, ntau, s, sig)
        b.get_G(p, Gg)
        errs.append(component_errors(Gg, Go[p], k + 1, nt))
    b.close()
    return errs


@pytest.mark.parametrize("s,nt,ntau,npb", [(1, 40, 30, 3), (2, 30, 20, 2), (3, 22, 14, 2), (4, 18, 12, 2),
                                           (5, 14, 10, 1), (8, 13, 10, 1)])
def test_dyson_timestep_parity(oracle, s, nt, ntau, npb):
    errs = _run(oracle, s, [nt] * npb, ntau, seed=s)
    for e in errs:
        for comp, v in e.items():
            assert v < TOL, (comp, v, e)


@pytest.mark.parametrize("ntau", [6, 8, 10, 12])
def test_dyson_timestep_short_tau_grid(oracle, ntau):
    """ntau < 2k+2 exercises the tabulated Gregory rows and the rcorr boundary terms."""
    errs = _run(oracle, 1, [16, 16], ntau, seed=100 + ntau)
    for e in errs:
        for comp, v in e.items():
            assert v < TOL, (comp, v)


def test_dyson_timestep_bosonic(oracle):
    errs = _run(oracle, 2, [16], 16, sig=1, mu=-1.5, seed=7)
    for comp, v in errs[0].items():
        assert v < TOL, (comp, v)


def test_dyson_timestep_uneven_batch(oracle):
    """Problems of one Sigma group with different nt: only problems with nt >= n step."""
    errs = _run(oracle, 2, [26, 19, 12, 26], 12, seed=11)
    for e in errs:
        for comp, v in e.items():
            assert v < TOL, (comp, v)


def test_single_problem_cntr_signature(oracle):
    """gpu.dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder) mirrors cntr::dyson_timestep."""
    from nessi_b200 import gpu
    rng = np.random.default_rng(3)
    nt, ntau, s, beta, h, k, mu = 12, 10, 2, 4.0, 0.05, 5, 0.0
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    H = make_H(rng, nt, s, h)
    G = herm_matrix(nt, ntau, s, -1)
    Gf, G0 = solve_oracle(oracle, G, H, Sig, mu, beta, h, k, nt_stop=k + 1)
    Gg = G0.copy()
    gpu.dyson_timestep(k + 1, Gg, mu, H, Sig, beta, h, k)
    e = component_errors(Gg, Gf, k + 1, k + 1)
    for comp, v in e.items():
        assert v < TOL, (comp, v)


@pytest.fixture
def volterra_pp(monkeypatch):
    """Force the problems-per-CTA setting of the size1 <= 2 Volterra kernels for new batches."""
    def set_pp(pp):
        monkeypatch.setenv("NESSI_VOLTERRA_PP", str(pp))
    return set_pp


@pytest.mark.parametrize("s", [1, 2])
@pytest.mark.parametrize("pp", [-1, 1, 2, 4, 8, 100, 101])
def test_volterra_problems_per_cta(oracle, volterra_pp, s, pp):
    """Every grouping of problems per CTA (and the one-problem kernels, -1, the group-wide
    cluster recursion, 100, and the whole-GPU recursion, 101) gives the oracle's numbers on an uneven batch whose histories span
    several 32-row blocks; the batch size is not a multiple of the grouping, so partly filled CTAs
    are exercised too."""
    volterra_pp(pp)
    errs = _run(oracle, s, [90, 75, 90, 40, 90, 66, 90, 90, 12], 10, seed=40 + s)
    for e in errs:
        for comp, v in e.items():
            assert v < TOL, (comp, v)


@pytest.mark.parametrize("s,nt", [(3, 40), (4, 36), (5, 30), (8, 28)])
@pytest.mark.parametrize("pp", [-1, 100, 101])
def test_volterra_large_orbitals(oracle, volterra_pp, s, nt, pp):
    """size1 >= 3: the one-problem kernels, the cluster recursion and the whole-GPU recursion
    (blocks of 16 rows for size1 3-4, 8 above; several blocks per step, an uneven batch) against
    the oracle."""
    volterra_pp(pp)
    errs = _run(oracle, s, [nt, nt - 9, nt, 12], 8, seed=60 + s)
    for e in errs:
        for comp, v in e.items():
            assert v < TOL, (comp, v)


@pytest.mark.parametrize("pp", [100, 101])
def test_cluster_recursion_many_problems(oracle, volterra_pp, pp):
    """More problems than one cluster holds (several clusters, the last one partly filled), each
    history spanning several blocks; the same batch through the whole-GPU recursion."""
    volterra_pp(pp)
    errs = _run(oracle, 1, [70] * 40 + [33, 51], 10, seed=77)
    for e in errs:
        for comp, v in e.items():
            assert v < TOL, (comp, v)
