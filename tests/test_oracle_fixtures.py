"""The oracle against the known-answer tests of libcntr's own suite (libcntr/test/*.cpp):
the embedding fixture of dyson.cpp:23-160 and the free-propagator convolution identity
A*B = (A-B)/(wa-wb) of convolution.cpp:30-185.  Tolerances are the reference's."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix, function


def _embedding(O, Nt=200, Ntau=400, dt=0.05, beta=10.0):
    eps1, eps2, lam, mu, k = -1.0, 1.0, 0.2, -0.1, 5
    h2 = np.array([[eps1, 1j * lam], [-1j * lam, eps2]])
    hf = function(Nt, 1)
    hf.set_constant(np.array([[eps1]]))
    G2 = herm_matrix(Nt, Ntau, 2, -1)
    O.green_from_H(G2, mu, h2, beta, dt)
    Gx = herm_matrix(Nt, Ntau, 1, -1)
    for t in range(-1, Nt + 1):
        Gx.set_matrixelement(t, 0, 0, G2, 0, 0)
    Sig = herm_matrix(Nt, Ntau, 1, -1)
    O.green_from_H(Sig, mu, np.array([[eps2]]), beta, dt)
    for t in range(-1, Nt + 1):
        Sig.smul(t, lam * lam)
    return dict(Nt=Nt, Ntau=Ntau, dt=dt, beta=beta, mu=mu, k=k, hf=hf, Gx=Gx, Sig=Sig, eps1=eps1)


def test_dyson_embedding_integro_differential(oracle):
    O = oracle
    c = _embedding(O)
    Ga = herm_matrix(c["Nt"], c["Ntau"], 1, -1)
    O.dyson_mat(Ga, c["Sig"], c["mu"], c["hf"], c["beta"], c["k"])
    O.dyson_start(Ga, c["mu"], c["hf"], c["Sig"], c["beta"], c["dt"], c["k"])
    for n in range(c["k"] + 1, c["Nt"] + 1):
        O.dyson_timestep(n, Ga, c["mu"], c["hf"], c["Sig"], c["beta"], c["dt"], c["k"])
    err = sum(O.distance_norm2(t, c["Gx"], Ga) for t in range(c["Nt"] + 1))
    assert err / c["Nt"] < 1.0e-3          # dyson.cpp:95 (tol_coarse)
    assert err / c["Nt"] < 1.0e-5          # what the restatement actually reaches (2.1e-6)


def test_dyson_embedding_integral_form(oracle):
    O = oracle
    c = _embedding(O)
    Nt, Ntau, k, beta, dt = c["Nt"], c["Ntau"], c["k"], c["beta"], c["dt"]
    Ga = herm_matrix(Nt, Ntau, 1, -1)
    O.dyson_mat(Ga, c["Sig"], c["mu"], c["hf"], beta, k)
    G0 = herm_matrix(Nt, Ntau, 1, -1)
    O.green_from_H(G0, c["mu"], np.array([[c["eps1"]]]), beta, dt)
    F, Fcc = herm_matrix(Nt, Ntau, 1, -1), herm_matrix(Nt, Ntau, 1, -1)
    for t in range(0, Nt + 1):
        O.convolution_timestep(t, F, G0, G0, c["Sig"], c["Sig"], beta, dt, k)
        O.convolution_timestep(t, Fcc, c["Sig"], c["Sig"], G0, G0, beta, dt, k)
        F.smul(t, -1)
        Fcc.smul(t, -1)
        if t == k:
            O.vie2_start(Ga, F, Fcc, G0, beta, dt, k)
        elif t > k:
            O.vie2_timestep(t, Ga, F, Fcc, G0, beta, dt, k)
    err = sum(O.distance_norm2(t, c["Gx"], Ga) for t in range(Nt + 1))
    assert err / Nt < 1.0e-6               # dyson.cpp:133 (tol_tight)


@pytest.mark.parametrize("sig", [-1, 1])
def test_convolution_free_propagators(oracle, sig):
    O = oracle
    nt, ntau, beta, h, wa, wb, k = 7, 500, 5.0, 0.01, 1.123, 0.345, 5
    A, B, C, AB = (herm_matrix(nt, ntau, 1, sig) for _ in range(4))
    O.green_from_H(A, 0.0, np.array([[wa]]), beta, h)
    O.green_from_H(B, 0.0, np.array([[wb]]), beta, h)
    C = A.copy()
    for t in range(-1, nt + 1):
        C.incr_timestep(t, B, -1.0)
        C.smul(t, 1.0 / (wa - wb))
    for t in range(-1, nt + 1):
        O.convolution_timestep(t, AB, A, A, B, B, beta, h, k)
    err = sum(O.distance_norm2(t, C, AB) for t in range(-1, nt + 1))
    assert err < 1e-6 * 4                  # convolution.cpp:28 (eps, four norms summed there)


def test_extrapolation_is_exact_for_polynomials(oracle):
    """extrapolate_timestep reproduces a degree-k polynomial in t exactly
    (the property libcntr/test/utilities.cpp:213-300 checks)."""
    O = oracle
    nt, ntau, k = 12, 6, 5
    G = herm_matrix(nt, ntau, 1, -1)
    f = lambda t, tp: (0.3 + 0.1j) * t ** 3 - 0.2 * t * tp + 0.05j * tp ** 2 + 1.0
    for t in range(nt + 1):
        for tp in range(t + 1):
            G.ret[G.ret_index(t, tp)] = f(t, tp)
        for tp in range(t + 1):
            G.les[G.les_index(tp, t)] = f(tp, t)
        G.tv[t, :, 0, 0] = [f(t, m) for m in range(ntau + 1)]
    n = 9
    O.extrapolate_timestep(n, G, k)
    assert np.allclose(G.tv[n + 1, :, 0, 0], [f(n + 1, m) for m in range(ntau + 1)], rtol=1e-10, atol=1e-9)
    assert np.allclose(G.ret_row(n + 1)[k + 1:, 0, 0], [f(n + 1, tp) for tp in range(k + 1, n + 2)],
                       rtol=1e-10, atol=1e-9)


def test_dyson_mat_fixpoint_embedding(oracle):
    """libcntr/test/matsubara.cpp:34-94: the Matsubara Dyson equation of the level eps1 = -1
    embedded by lam = 0.2 into eps2 = 1 (beta = 20, ntau = 400, order 5), solved by the fixpoint
    method, reproduces the (0,0) element of the free 2 x 2 propagator within 1e-7."""
    O = oracle
    eps1, eps2, lam, mu, beta, ntau, k = -1.0, 1.0, 0.2, 0.0, 20.0, 400, 5
    G2 = herm_matrix(-1, ntau, 2, -1)
    O.green_from_H(G2, mu, np.array([[eps1, 1j * lam], [-1j * lam, eps2]]), beta, 1.0)
    exact = herm_matrix(-1, ntau, 1, -1)
    exact.mat[:, 0, 0] = G2.mat[:, 0, 0]
    Sig = herm_matrix(-1, ntau, 1, -1)
    O.green_from_H(Sig, mu, np.array([[eps2]]), beta, 1.0)
    Sig.smul(-1, lam * lam)
    H = function(-1, 1)
    H.set_value(-1, np.array([[eps1]]))
    G = herm_matrix(-1, ntau, 1, -1)
    O.dyson_mat(G, Sig, mu, H, beta, k, method=O.CNTR_MAT_FIXPOINT)
    err = O.distance_norm2(-1, exact, G)
    assert err < 1.0e-7, err               # matsubara.cpp:47 (tol_tight)


@pytest.mark.parametrize("sig,shift", [(-1, 0.0), (1, 3.0)])
def test_green_from_H_is_the_free_propagator(oracle, sig, shift):
    """libcntr/test/equilibrium.cpp:240-290: green_from_H of the 2 x 2 H = sqrt(2) [[1, -i], [i, -1]]
    (nt = 100, ntau = 500, beta = 5, h = 0.01) against the closed form V g(w) V^dagger of its
    eigenlevels, summed distance over t = -1..nt-1 below 1e-6.  The bosonic variant shifts the
    levels above the chemical potential (w + 3 > 0) so that the occupations stay finite."""
    from test_oracle_bubble import FreeLevels
    O = oracle
    nt, ntau, beta, h = 100, 500, 5.0, 0.01
    a = np.sqrt(2.0) * np.array([[1.0, -1j], [1j, -1.0]]) + shift * np.eye(2)
    w, V = np.linalg.eigh(a)
    exact = FreeLevels(w, sig, beta, V.conj().T).herm_matrix(nt, ntau, h)
    G = herm_matrix(nt, ntau, 2, sig)
    O.green_from_H(G, 0.0, a, beta, h)
    err = sum(O.distance_norm2(t, G, exact) for t in range(-1, nt))
    assert err < 1e-6, err                 # equilibrium.cpp:244 (eps)


def test_convolution_bosonic_boundary_signs(oracle):
    """libcntr/test/convolution.cpp:98-143: the free-boson identity A*B = (A - B)/(wa - wb) at
    beta = 0.1, ntau = 500, t_max = 2 on refined grids h = 2/nt, nt = 10..640; the reference
    checks the last time step of the finest grid at 1e-6 (its last assignment is the lesser
    distance); here every component of that step is checked, and the error falls with h."""
    O = oracle
    wa, wb, k, beta, ntau, tmax = 1.123, 0.345, 5, 0.1, 500, 2.0
    errs = []
    for fac2 in (1, 4, 16, 64):
        nt = 10 * fac2
        h = tmax / nt
        A, B, AB = (herm_matrix(nt, ntau, 1, 1) for _ in range(3))
        O.green_from_H(A, 0.0, np.array([[wa]]), beta, h)
        O.green_from_H(B, 0.0, np.array([[wb]]), beta, h)
        C = A.copy()
        C.incr_timestep(nt, B, -1.0)
        C.smul(nt, 1.0 / (wa - wb))
        for n in (-1, nt):  # convolution_timestep reads only A and B: the last step suffices
            O.convolution_timestep(n, AB, A, A, B, B, beta, h, k)
        errs.append(O.distance_norm2(nt, C, AB))
    assert errs[-1] < 1e-6, errs            # convolution.cpp:142 (eps)
    assert errs[-1] < errs[0]


def test_downfolding_of_a_three_level_system(oracle):
    """libcntr/test/downfold.cpp:367-427 (time-independent): the (0,0) element of the free 3 x 3
    propagator of a = [[1, -1, -1], [-1, 2, -1], [-1, -1, 3]] (the e^{+-i pi} couplings), from the
    embedded 1 x 1 problem: G0 the zero-level propagator, eta = a_{0R} G_RR a_{R0} with G_RR the
    free propagator of the 2 x 2 rest, F = -(G0 * eta) - G0 a_00, Fcc = -(eta * G0) - a_00 G0,
    [1 + F] G = G0 by vie2 (nt = 20, ntau = 300, beta = 1, h = 0.01, order 5); the reference
    accepts a summed distance below 1e-6."""
    O = oracle
    nt, ntau, beta, h, k = 20, 300, 1.0, 0.01, 5
    a = np.array([[1.0, np.exp(1j * np.pi), np.exp(1j * np.pi)],
                  [np.exp(-1j * np.pi), 2.0, np.exp(1j * np.pi)],
                  [np.exp(-1j * np.pi), np.exp(-1j * np.pi), 3.0]])
    A = herm_matrix(nt, ntau, 3, -1)
    O.green_from_H(A, 0.0, a, beta, h)
    R = herm_matrix(nt, ntau, 2, -1)
    O.green_from_H(R, 0.0, a[1:, 1:], beta, h)
    G0 = herm_matrix(nt, ntau, 1, -1)
    O.green_from_H(G0, 0.0, np.zeros((1, 1)), beta, h)
    eta = herm_matrix(nt, ntau, 1, -1)
    v, w = a[0:1, 1:], a[1:, 0:1]   # a_{0R}, a_{R0}: time-independent couplings
    for c in ("ret", "les", "tv", "mat"):
        getattr(eta, c)[...] = np.einsum("ab,nbc,cd->nad", v, getattr(R, c).reshape(-1, 2, 2), w).reshape(
            getattr(eta, c).shape)
    F, Fcc = herm_matrix(nt, ntau, 1, -1), herm_matrix(nt, ntau, 1, -1)
    for n in range(-1, nt + 1):
        O.convolution_timestep(n, F, G0, G0, eta, eta, beta, h, k)
        O.convolution_timestep(n, Fcc, eta, eta, G0, G0, beta, h, k)
    e00 = a[0, 0].real
    for c in ("ret", "les", "tv", "mat"):
        getattr(F, c)[...] = -getattr(F, c) - e00 * getattr(G0, c)
        getattr(Fcc, c)[...] = -getattr(Fcc, c) - e00 * getattr(G0, c)
    G = herm_matrix(nt, ntau, 1, -1)
    O.vie2_mat(G, F, Fcc, G0, beta, k)
    O.vie2_start(G, F, Fcc, G0, beta, h, k)
    for n in range(k + 1, nt + 1):
        O.vie2_timestep(n, G, F, Fcc, G0, beta, h, k)
    A00 = herm_matrix(nt, ntau, 1, -1)
    for t in range(-1, nt + 1):
        A00.set_matrixelement(t, 0, 0, A, 0, 0)
    err = sum(O.distance_norm2(t, G, A00) for t in range(-1, nt))
    assert err < 1e-6, err                 # downfold.cpp:371 (eps)
