"""GPU parity of the lattice pieces through the C ABI: extrapolate_timestep, the k-average G_loc,
Sigma_2B, and whole self-consistent lattice propagations (bootstrap + predictor/corrector steps)
against the oracle.  FP64 bar 1e-10 relative; mixed precision <= 1e-8."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import make_H, make_lattice, make_sigma, rel_err, solve_oracle, component_errors, u_matrices

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _solved(O, seed, nt, ntau, s, beta=3.0, h=0.05, k=5):
    rng = np.random.default_rng(seed)
    Sig = make_sigma(O, rng, nt, ntau, s, -1, beta, h)
    H = make_H(rng, nt, s, h)
    G = herm_matrix(nt, ntau, s, -1)
    G, _ = solve_oracle(O, G, H, Sig, 0.1, beta, h, k)
    return G


@pytest.mark.parametrize("s", [1, 2, 3])
def test_extrapolate_timestep(oracle, s):
    from nessi_b200 import gpu
    nt, ntau, k = 16, 10, 5
    G = _solved(oracle, 30 + s, nt, ntau, s)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=3.0, h=0.05)])
    for n in (k, k + 3, nt - 1):
        b.set_G(0, G)
        b.extrapolate_timestep(n)
        out = herm_matrix(nt, ntau, s, -1)
        b.get_G(0, out)
        R = G.copy()
        oracle.extrapolate_timestep(n, R, k)
        assert rel_err(out.get_timestep(n + 1), R.get_timestep(n + 1)) < 1e-13
        # nothing else changed
        assert rel_err(out.get_timestep(n), G.get_timestep(n)) == 0.0
    b.close()


@pytest.mark.parametrize("s", [1, 2])
def test_gloc_and_sigma_2b(oracle, s):
    """G_loc of three problems and Sigma_2B of it at every time step (including mat), for a
    non-diagonal G (s = 2 exercises the orbital indices) and a complex diagonal U."""
    from nessi_b200 import gpu
    nt, ntau, k = 12, 10, 5
    Gs = [_solved(oracle, 40 + 10 * s + i, nt, ntau, s) for i in range(3)]
    rng = np.random.default_rng(5)
    U = rng.normal(0, 1, (nt + 2, s)) + 1j * rng.normal(0, 0.3, (nt + 2, s))
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=3.0, h=0.05)] * 3)
    for i, G in enumerate(Gs):
        b.set_G(i, G)
    b.set_U(0, U)
    Lref = herm_matrix(nt, ntau, s, -1)
    Sref = herm_matrix(nt, ntau, s, -1)
    for t in range(-1, nt + 1):
        b.gloc_timestep(0, t)
        b.sigma_2b_timestep(0, t)
        oracle.gloc_timestep(t, Gs, Lref)
        oracle.sigma_2b_timestep(t, Sref, Lref, u_matrices(U))
    L = herm_matrix(nt, ntau, s, -1)
    S = herm_matrix(nt, ntau, s, -1)
    b.get_gloc(0, L)
    b.get_sigma(0, S)
    b.close()
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(L, comp), getattr(Lref, comp)) < 1e-14, comp
        assert rel_err(getattr(S, comp), getattr(Sref, comp)) < 1e-13, comp


def _lattice_run(O, precision, nkx, nky, nt, ntau, u_mat):
    from nessi_b200 import gpu
    beta, h, k, ncorr = 5.0, 0.02, 5, 3
    Gs, Hs, U = make_lattice(O, nkx, nky, nt, ntau, beta, h, u_max=2.0, t_ramp=0.2, u_mat=u_mat)
    nk = len(Gs)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=1, sig=-1, solve_order=k, beta=beta, h=h)] * nk, precision)
    for p in range(nk):
        b.set_G(p, Gs[p])
        b.set_H(p, Hs[p])
    b.set_sigma(0, herm_matrix(nt, ntau, 1, -1))
    b.set_U(0, U)
    it_g, err_g = b.lattice_2b_start(max_iter=6, tol=0.0)
    for n in range(k + 1, nt + 1):
        b.lattice_2b_timestep(n, ncorr)
    out = [herm_matrix(nt, ntau, 1, -1) for _ in range(nk)]
    for p in range(nk):
        b.get_G(p, out[p])
    L = herm_matrix(nt, ntau, 1, -1)
    b.get_gloc(0, L)
    b.close()
    # oracle
    Gloc = herm_matrix(nt, ntau, 1, -1)
    Sig = herm_matrix(nt, ntau, 1, -1)
    Um = u_matrices(U)
    it_o, err_o = O.lattice2b_start(Gs, Gloc, Sig, Um, 0.0, Hs, beta, h, k, max_iter=6, tol=0.0)
    assert it_g == it_o == 7
    assert abs(err_g - err_o) <= 1e-9 * max(err_o, 1e-300) + 1e-14
    for n in range(k + 1, nt + 1):
        O.lattice2b_timestep(n, Gs, Gloc, Sig, Um, 0.0, Hs, beta, h, k, ncorr=ncorr)
    worst = {}
    for p in range(nk):
        e = component_errors(out[p], Gs[p], 0, nt)
        for c, v in e.items():
            worst[c] = max(worst.get(c, 0.0), v)
    e = component_errors(L, Gloc, 0, nt)
    worst["gloc"] = max(e.values())
    return worst


@pytest.mark.parametrize("u_mat", [0.0, 0.7])
def test_lattice_2b_fp64(oracle, u_mat):
    """Config-4 type lattice (square lattice, size1 = 1, U ramp, 3 correctors) at 1e-10.  A
    nonzero U on the Matsubara branch makes Sigma^tv nonzero and exercises the tv path."""
    from nessi_b200 import gpu
    worst = _lattice_run(oracle, gpu.PREC_FP64, 3, 3, 30, 20, u_mat)
    assert max(worst.values()) < TOL, worst


def test_lattice_2b_cluster_recursion(oracle, monkeypatch):
    """The lattice step with the group-wide cluster recursion for both Volterra components."""
    from nessi_b200 import gpu
    monkeypatch.setenv("NESSI_VOLTERRA_PP", "100")
    worst = _lattice_run(oracle, gpu.PREC_FP64, 3, 3, 70, 20, 0.7)
    assert max(worst.values()) < TOL, worst


def test_lattice_2b_mixed(oracle):
    from nessi_b200 import gpu
    worst = _lattice_run(oracle, gpu.PREC_MIXED, 4, 2, 60, 30, 0.0)
    assert max(worst.values()) < 1e-8, worst


def test_lattice_requires_interaction():
    from nessi_b200 import gpu
    b = gpu.Batch([dict(nt=10, ntau=8, size1=1, sig=-1, solve_order=5, beta=3.0, h=0.05)])
    with pytest.raises(gpu.NessiGpuError):
        b.lattice_2b_timestep(7, 3)
    with pytest.raises(gpu.NessiGpuError):
        b.sigma_2b_timestep(0, 3)
    with pytest.raises(gpu.NessiGpuError):
        b.extrapolate_timestep(2)   # below the solve order
    b.close()
