"""GPU parity of the element-parallel path through the C ABI against the oracle: incr_convolution
(every component, masks, a function ft, alpha), convolution_timestep_new, dyson_timestep_omp (both
lesser branches: n < 2k+1 and the conjugate equation for n >= 2k+1) and vie2_timestep_omp
(cntr_convolution_impl.hpp:4164-4976, cntr_dyson_omp_impl.hpp:37-605, cntr_vie2_impl.hpp:1851-2190),
at 1e-10 per component; and the reference's own omp known answer (libcntr/test/dyson.cpp:138-165)
computed on the GPU at its tolerance."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix, function
from builders import make_H, rel_err
from test_gpu_conv import DevHM, _pair, make_sigma

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _func(rng, nt, s):
    """function data (F(-1) first) of a smooth, non-hermitian matrix function"""
    F = np.zeros((nt + 2, s, s), np.complex128)
    x = rng.normal(0, 0.5, (s, s)) + 1j * rng.normal(0, 0.5, (s, s))
    for t in range(-1, nt + 1):
        F[t + 1] = np.eye(s) + np.cos(0.3 * t) * x
    return F


@pytest.mark.parametrize("s,sig,k,ntau,with_ft", [(1, -1, 5, 9, False), (2, -1, 5, 14, True), (3, 1, 3, 10, True),
                                                  (2, 1, 4, 16, False)])
def test_incr_convolution_matches_oracle(oracle, s, sig, k, ntau, with_ft):
    """C += alpha A * ft * B at every time step -1..nt (n < k, n <= 2k+2 and the omega-split range;
    ntau = 9 < 2k+1 exercises the overlapping end loops of the tau integral) for 2 problems."""
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(500 + 7 * s + k)
    nt, beta, h, alpha = 16, 3.0, 0.05, 0.8 - 0.3j
    probs, dev = [], []
    for _ in range(2):
        A, Acc = _pair(oracle, rng, nt, ntau, s, sig, beta, h, k)
        B = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.9)
        C = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.5)
        ft = _func(rng, nt, s) if with_ft else None
        probs.append((A, Acc, B, C, ft))
        dev.append((DevHM(C), DevHM(A), DevHM(Acc), DevHM(B),
                    torch.from_numpy(ft).cuda() if with_ft else None))
    fts = [d[4].data_ptr() for d in dev] if with_ft else None
    for n in range(-1, nt + 1):
        gpu.incr_convolution_dev(n, alpha, [d[0].ptrs() for d in dev], [d[1].ptrs() for d in dev],
                                 [d[2].ptrs() for d in dev], [d[3].ptrs() for d in dev], [d[3].ptrs() for d in dev],
                                 nt, ntau, s, sig, sig, k, beta, h, ft=fts)
    torch.cuda.synchronize()
    for (A, Acc, B, C, ft), d in zip(probs, dev):
        R = C.copy()
        for n in range(-1, nt + 1):
            oracle.incr_convolution(n, alpha, R, A, Acc, B, B, beta, h, k, ft=ft)
        G = d[0].host()
        for comp in ("ret", "les", "tv", "mat"):
            assert rel_err(getattr(G, comp), getattr(R, comp)) < TOL, comp


def test_incr_convolution_component_masks(oracle):
    """Each component restricted to the indices of one of three OpenMP threads (device mask), the
    three masks summing to the whole time step, and convolution_timestep_new at the end."""
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(77)
    s, sig, k, nt, ntau, beta, h = 2, -1, 5, 15, 13, 2.5, 0.04
    A, Acc = _pair(oracle, rng, nt, ntau, s, sig, beta, h, k)
    B = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.8)
    C0 = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.4)
    dC, dA, dAcc, dB = DevHM(C0), DevHM(A), DevHM(Acc), DevHM(B)
    R = C0.copy()
    tstp, nth = 13, 3
    for which, size in ((1, tstp + 1), (2, ntau + 1), (3, tstp + 1)):
        for tid in range(nth):
            mask = np.array([i % nth == tid for i in range(size)], np.uint8)
            dm = torch.from_numpy(mask).cuda()
            gpu.incr_convolution_component_dev(which, tstp, dm.data_ptr(), 0.5 + 0.5j, [dC.ptrs()], [dA.ptrs()],
                                               [dAcc.ptrs()], [dB.ptrs()], [dB.ptrs()], nt, ntau, s, sig, sig, k,
                                               beta, h)
            torch.cuda.synchronize()
            oracle.incr_convolution_part(which, tstp, mask.astype(bool), 0.5 + 0.5j, R, A, Acc, B, B, beta, h, k)
    G = dC.host()
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(G, comp), getattr(R, comp)) < TOL, comp
    # convolution_timestep_new overwrites the step
    gpu.convolution_timestep_new_dev(tstp, [dC.ptrs()], [dA.ptrs()], [dAcc.ptrs()], [dB.ptrs()], [dB.ptrs()], nt,
                                     ntau, s, sig, sig, k, beta, h)
    torch.cuda.synchronize()
    oracle.convolution_timestep_new(tstp, R, A, Acc, B, B, beta, h, k)
    G = dC.host()
    for comp in ("ret", "les", "tv"):
        assert rel_err(getattr(G, comp), getattr(R, comp)) < TOL, comp


@pytest.mark.parametrize("s,sig,k", [(1, -1, 5), (2, -1, 5), (4, 1, 3), (8, -1, 2)])
def test_dyson_timestep_omp_matches_oracle(oracle, s, sig, k):
    """dyson_timestep_omp for n = k+1..nt for 2 problems (different H and mu) from the same
    bootstrap, every component of every step against the oracle's restatement; nt covers the
    serial lesser branch (n < 2k+1) and the conjugate-equation branch."""
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(900 + 10 * s + k)
    nt, ntau, beta, h = 3 * k + 12, 3 * k + 6, 4.0, 0.04
    Sig = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.6)
    probs = []
    for i in range(2):
        H = make_H(rng, nt, s, h)
        if sig == 1:
            for t in range(-1, nt + 1):
                H.set_value(t, H.get_value(t) + 4.0 * np.eye(s))
        mu = 0.1 * (i + 1)
        G = herm_matrix(nt, ntau, s, sig)
        oracle.dyson_mat(G, Sig, mu, H, beta, k)
        oracle.dyson_start(G, mu, H, Sig, beta, h, k)
        probs.append((G, H, mu))
    dG = [DevHM(G) for G, _, _ in probs]
    dS = DevHM(Sig)
    dH = [torch.from_numpy(np.ascontiguousarray(H.data)).cuda() for _, H, _ in probs]
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for n in range(k + 1, nt + 1):
        gpu.dyson_timestep_omp_dev(n, [d.ptrs() for d in dG], [dS.ptrs()] * 2, [x.data_ptr() for x in dH],
                                   [mu for _, _, mu in probs], nt, ntau, s, sig, k, beta, h, status.data_ptr())
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    for (G, H, mu), d in zip(probs, dG):
        for n in range(k + 1, nt + 1):
            oracle.dyson_timestep_omp(n, G, mu, H, Sig, beta, h, k)
        Gg = d.host()
        for comp in ("ret", "les", "tv"):
            assert rel_err(getattr(Gg, comp), getattr(G, comp)) < TOL, comp


@pytest.mark.parametrize("s,sig", [(1, -1), (2, 1), (3, -1)])
def test_vie2_timestep_omp_matches_oracle(oracle, s, sig):
    """vie2_timestep_omp for n = k+1..nt with F = -G0 * Sigma, Fcc = -Sigma * G0, Q = G0 (the
    reference's integral form of the Dyson equation), G bootstrapped by the oracle's vie2_mat and
    vie2_start; Q must come back unchanged."""
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(1300 + 10 * s)
    k, nt, ntau, beta, h = 5, 24, 18, 3.0, 0.05
    G0 = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=1.0)
    Sig = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.5)
    F, Fcc = herm_matrix(nt, ntau, s, sig), herm_matrix(nt, ntau, s, sig)
    for t in range(-1, nt + 1):
        oracle.convolution_timestep(t, F, G0, G0, Sig, Sig, beta, h, k)
        oracle.convolution_timestep(t, Fcc, Sig, Sig, G0, G0, beta, h, k)
        F.smul(t, -1)
        Fcc.smul(t, -1)
    G = herm_matrix(nt, ntau, s, sig)
    oracle.vie2_mat(G, F, Fcc, G0, beta, k)
    oracle.vie2_start(G, F, Fcc, G0, beta, h, k)
    dG, dF, dFcc, dQ = DevHM(G), DevHM(F), DevHM(Fcc), DevHM(G0)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for n in range(k + 1, nt + 1):
        gpu.vie2_timestep_omp_dev(n, [dG.ptrs()], [dF.ptrs()], [dFcc.ptrs()], [dQ.ptrs()], nt, ntau, s, sig, k, beta, h,
                                  status.data_ptr())
        oracle.vie2_timestep_omp(n, G, F, Fcc, G0, beta, h, k)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    Gg, Qg = dG.host(), dQ.host()
    for comp in ("ret", "les", "tv"):
        assert rel_err(getattr(Gg, comp), getattr(G, comp)) < TOL, comp
        assert np.array_equal(getattr(Qg, comp), getattr(G0, comp)), comp


def test_vie2_omp_embedding_known_answer_on_gpu(oracle):
    """libcntr/test/dyson.cpp:138-165 on the GPU: F and Fcc by convolution_timestep_new (the
    reference's convolution_timestep_omp), vie2_timestep_omp for t > k (t <= k by the start,
    as the reference dispatches), err / Nt < 1e-6 against the exact embedding solution."""
    import torch
    from nessi_b200 import gpu
    from test_oracle_fixtures import _embedding
    O = oracle
    c = _embedding(O)
    Nt, Ntau, k, beta, dt = c["Nt"], c["Ntau"], c["k"], c["beta"], c["dt"]
    Ga = herm_matrix(Nt, Ntau, 1, -1)
    O.dyson_mat(Ga, c["Sig"], c["mu"], c["hf"], beta, k)
    G0 = herm_matrix(Nt, Ntau, 1, -1)
    O.green_from_H(G0, c["mu"], np.array([[c["eps1"]]]), beta, dt)
    F, Fcc = herm_matrix(Nt, Ntau, 1, -1), herm_matrix(Nt, Ntau, 1, -1)
    dF, dFcc, dG0, dS = DevHM(F), DevHM(Fcc), DevHM(G0), DevHM(c["Sig"])
    for t in range(0, Nt + 1):
        gpu.convolution_timestep_new_dev(t, [dF.ptrs()], [dG0.ptrs()], [dG0.ptrs()], [dS.ptrs()], [dS.ptrs()], Nt,
                                         Ntau, 1, -1, -1, k, beta, dt)
        gpu.convolution_timestep_new_dev(t, [dFcc.ptrs()], [dS.ptrs()], [dS.ptrs()], [dG0.ptrs()], [dG0.ptrs()], Nt,
                                         Ntau, 1, -1, -1, k, beta, dt)
    torch.cuda.synchronize()
    F, Fcc = dF.host(), dFcc.host()
    for t in range(0, Nt + 1):
        F.smul(t, -1)
        Fcc.smul(t, -1)
    for t in range(0, k + 1):
        O.vie2_timestep_omp(t, Ga, F, Fcc, G0, beta, dt, k)
    dG, dF, dFcc = DevHM(Ga), DevHM(F), DevHM(Fcc)
    for t in range(k + 1, Nt + 1):
        gpu.vie2_timestep_omp_dev(t, [dG.ptrs()], [dF.ptrs()], [dFcc.ptrs()], [dG0.ptrs()], Nt, Ntau, 1, -1, k, beta,
                                  dt)
    torch.cuda.synchronize()
    Ga = dG.host()
    err = sum(O.distance_norm2(t, c["Gx"], Ga) for t in range(Nt + 1))
    assert err / Nt < 1.0e-6


def test_python_dropins_on_host_data(oracle):
    """The host-data drop-ins with libcntr's signatures: gpu.dyson_timestep_omp (n = k+1..nt),
    gpu.vie2_timestep_omp (n = -1, 1..nt: vie2_mat, the starts of order n as the reference
    dispatches them, then the element-parallel step), gpu.incr_convolution with a function F and
    gpu.convolution_timestep_omp, each against the oracle."""
    from nessi_b200 import gpu
    from test_gpu_vie2 import _kernel_pair, _source
    rng = np.random.default_rng(2024)
    s, sig, k, nt, ntau, beta, h, mu = 2, -1, 4, 18, 12, 3.0, 0.05, 0.2
    Sig = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.6)
    H = make_H(rng, nt, s, h)
    G = herm_matrix(nt, ntau, s, sig)
    oracle.dyson_mat(G, Sig, mu, H, beta, k)
    oracle.dyson_start(G, mu, H, Sig, beta, h, k)
    R = G.copy()
    for n in range(k + 1, nt + 1):
        gpu.dyson_timestep_omp(4, n, G, mu, H, Sig, beta, h, k)
        oracle.dyson_timestep_omp(n, R, mu, H, Sig, beta, h, k)
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(G, comp), getattr(R, comp)) < TOL, ("dyson", comp)
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    V, RV = herm_matrix(nt, ntau, s, sig), herm_matrix(nt, ntau, s, sig)
    for n in [-1] + list(range(1, nt + 1)):
        gpu.vie2_timestep_omp(4, n, V, F, Fcc, Q, beta, h, k)
        oracle.vie2_timestep_omp(n, RV, F, Fcc, Q, beta, h, k)
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(V, comp), getattr(RV, comp)) < TOL, ("vie2", comp)
    A, Acc = _pair(oracle, rng, nt, ntau, s, sig, beta, h, k)
    ft = _func(rng, nt, s)
    C = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.3)
    RC = C.copy()
    for n in (-1, 2, 9, nt):
        gpu.incr_convolution(n, 0.6 + 0.2j, C, A, Acc, Sig, Sig, beta, h, k, ft=ft)
        oracle.incr_convolution(n, 0.6 + 0.2j, RC, A, Acc, Sig, Sig, beta, h, k, ft=ft)
    gpu.convolution_timestep_omp(4, 11, C, A, Acc, Sig, Sig, beta, h, k)
    oracle.convolution_timestep_new(11, RC, A, Acc, Sig, Sig, beta, h, k)
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(C, comp), getattr(RC, comp)) < TOL, ("incr", comp)
