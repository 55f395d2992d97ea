"""The oracle's restatement of libcntr's OpenMP-path routines (incr_convolution, the
convolution_*_new / convolution_*_omp drivers, dyson_timestep_omp, vie2_timestep_omp), pinned by
the reference's own known-answer tests for them: the "Integral form (omp)" embedding case of
libcntr/test/dyson.cpp:138-165 and the free-propagator identities of
libcntr/test/convolution.cpp:285-355 (convolution_new, convolution_omp).  The restatement runs in
one thread's order; the thread split of the reference only changes which thread computes an
element."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from test_oracle_fixtures import _embedding


def _rel(a, b):
    d = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / (d if d > 0 else 1.0))


def test_vie2_omp_embedding(oracle):
    """dyson.cpp:138-165: convolution_timestep_omp for F = -G0*Sigma, Fcc = -Sigma*G0 and
    vie2_timestep_omp for every step t = 0..Nt (t <= k dispatches to vie2_start of order t),
    err / Nt < tol_tight = 1e-6 against the exact embedding solution."""
    O = oracle
    c = _embedding(O)
    Nt, Ntau, k, beta, dt = c["Nt"], c["Ntau"], c["k"], c["beta"], c["dt"]
    Ga = herm_matrix(Nt, Ntau, 1, -1)
    O.dyson_mat(Ga, c["Sig"], c["mu"], c["hf"], beta, k)
    G0 = herm_matrix(Nt, Ntau, 1, -1)
    O.green_from_H(G0, c["mu"], np.array([[c["eps1"]]]), beta, dt)
    F, Fcc = herm_matrix(Nt, Ntau, 1, -1), herm_matrix(Nt, Ntau, 1, -1)
    for t in range(0, Nt + 1):
        O.convolution_timestep_new(t, F, G0, G0, c["Sig"], c["Sig"], beta, dt, k)
        O.convolution_timestep_new(t, Fcc, c["Sig"], c["Sig"], G0, G0, beta, dt, k)
        F.smul(t, -1)
        Fcc.smul(t, -1)
        O.vie2_timestep_omp(t, Ga, F, Fcc, G0, beta, dt, k)
    err = sum(O.distance_norm2(t, c["Gx"], Ga) for t in range(Nt + 1))
    assert err / Nt < 1.0e-6               # dyson.cpp:164 (tol_tight)


def test_dyson_omp_embedding(oracle):
    """dyson_timestep_omp on the same embedding fixture, as the Dyson-form section of dyson.cpp
    (:67-96) runs the serial step: err / Nt < tol_coarse = 1e-3 against the exact solution."""
    O = oracle
    c = _embedding(O)
    Nt, Ntau, k, beta, dt, mu = c["Nt"], c["Ntau"], c["k"], c["beta"], c["dt"], c["mu"]
    Ga = herm_matrix(Nt, Ntau, 1, -1)
    O.dyson_mat(Ga, c["Sig"], mu, c["hf"], beta, k)
    O.dyson_start(Ga, mu, c["hf"], c["Sig"], beta, dt, k)
    for n in range(k + 1, Nt + 1):
        O.dyson_timestep_omp(n, Ga, mu, c["hf"], c["Sig"], beta, dt, k)
    err = sum(O.distance_norm2(t, c["Gx"], Ga) for t in range(Nt + 1))
    assert err / Nt < 1.0e-3               # dyson.cpp:95 (tol_coarse)


@pytest.mark.parametrize("sig,driver", [(-1, "new"), (1, "omp")])
def test_convolution_new_and_omp_free_propagators(oracle, sig, driver):
    """convolution.cpp:285-355: C = A * B = (A - B) / (wa - wb) for free propagators through
    convolution_new (fermions) and convolution_omp (bosons), nt = 7, ntau = 500, the four
    distances summed below eps = 1e-6 (the reference sums distance_norm2 and its ret/tv/les
    parts, at most twice the full distance)."""
    O = oracle
    nt, ntau, beta, h, wa, wb, k = 7, 500, 5.0, 0.01, 1.123, 0.345, 5
    A, B, AB = (herm_matrix(nt, ntau, 1, sig) for _ in range(3))
    O.green_from_H(A, 0.0, np.array([[wa]]), beta, h)
    O.green_from_H(B, 0.0, np.array([[wb]]), beta, h)
    C = A.copy()
    for t in range(-1, nt + 1):
        C.incr_timestep(t, B, -1.0)
        C.smul(t, 1.0 / (wa - wb))
    for t in range(-1, nt + 1):
        if driver == "new":
            O.convolution_timestep_new(t, AB, A, A, B, B, beta, h, k)
        else:  # convolution_omp: the masks of 4 threads, one component call per thread
            if t == -1:
                AB.mat[...] = 0
            else:
                AB.ret_row(t)[...] = 0
                AB.tv[t] = 0
                AB.les_col(t)[...] = 0
            nth = 4
            for tid in range(nth):
                if t == -1:
                    O.incr_convolution_part(0, t, [i % nth == tid for i in range(ntau + 1)], 1.0, AB, A, A, B, B,
                                            beta, h, k)
                    continue
                mret = [i % nth == tid for i in range(t + 1)]
                mles = [mret[t - i] for i in range(t + 1)]
                O.incr_convolution_part(1, t, mret, 1.0, AB, A, A, B, B, beta, h, k)
                O.incr_convolution_part(2, t, [i % nth == tid for i in range(ntau + 1)], 1.0, AB, A, A, B, B,
                                        beta, h, k)
                O.incr_convolution_part(3, t, mles, 1.0, AB, A, A, B, B, beta, h, k)
    err = sum(O.distance_norm2(t, C, AB) for t in range(-1, nt + 1))
    assert 2 * err < 1e-6


def _rand_hm(rng, nt, ntau, s, sig, scale=1.0):
    """random herm_matrix data with the one property a hermitian function's lesser part needs
    for its two continuations to agree: G^<(t,t) = -G^<(t,t)^dagger"""
    G = herm_matrix(nt, ntau, s, sig)
    for a in (G.ret, G.les, G.tv, G.mat):
        a[...] = scale * (rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape))
    for t in range(nt + 1):
        x = G.les[G.les_index(t, t)]
        x[...] = 0.5 * (x - x.conj().T)
    return G


@pytest.mark.parametrize("s", [1, 2])
def test_incr_convolution_is_the_same_quadrature(oracle, s):
    """incr_convolution reorganises convolution_timestep's integrals per output element: for
    hermitian A and B and ntau >= 2k+2 (where the tau weights coincide) C + alpha A*B equals the serial
    convolution_timestep scaled by alpha and added, to round-off, at every time step including
    those below k; a function ft = 1 changes nothing."""
    O = oracle
    rng = np.random.default_rng(7 + s)
    nt, ntau, k, beta, h = 16, 14, 5, 2.0, 0.05
    A, B = (_rand_hm(rng, nt, ntau, s, -1, 0.3) for _ in range(2))
    Acc, Bcc = A, B
    alpha = 0.7 - 0.4j
    ones = np.zeros((nt + 2, s, s), np.complex128)
    ones[:] = np.eye(s)
    for t in range(-1, nt + 1):
        C0 = _rand_hm(rng, nt, ntau, s, -1)
        C1, C2 = C0.copy(), C0.copy()
        O.incr_convolution(t, alpha, C1, A, Acc, B, Bcc, beta, h, k)
        O.incr_convolution(t, alpha, C2, A, Acc, B, Bcc, beta, h, k, ft=ones)
        R = _rand_hm(rng, nt, ntau, s, -1)
        O.convolution_timestep(t, R, A, Acc, B, Bcc, beta, h, k)
        comps = [("mat", C1.mat, C0.mat + alpha * R.mat, C2.mat)] if t == -1 else [
            ("ret", C1.ret_row(t), C0.ret_row(t) + alpha * R.ret_row(t), C2.ret_row(t)),
            ("tv", C1.tv[t], C0.tv[t] + alpha * R.tv[t], C2.tv[t]),
            ("les", C1.les_col(t), C0.les_col(t) + alpha * R.les_col(t), C2.les_col(t))]
        for name, got, want, with_ft in comps:
            assert _rel(got, want) < 1e-12, (t, name, _rel(got, want))
            assert _rel(with_ft, got) < 1e-14, (t, name)


def test_omp_discretization_gap_on_impurity_shape(oracle):
    """The OpenMP solver is a different discretization (the equation in the other time argument
    for j < n-k): on the single-orbital impurity problem with the config-0 parameters
    (semicircular bath, beta 10, ntau 400, h 0.02; here nt 120) its result differs from the
    serial dyson_timestep by the discretization error in the retarded and lesser components
    (measured 7.8e-10 and 1.3e-10 relative, above the 1e-10 parity bar, far below the physics),
    while the left-mixing step is the serial one up to round-off (1e-14)."""
    from nessi_b200 import function, workloads
    O = oracle
    W = workloads.config0(nt=120)
    d = W.descs[0]
    nt, ntau, k = d["nt"], d["ntau"], W.k
    H = function(nt, 1)
    for t in range(-1, nt + 1):
        H.set_value(t, W.H[0, t + 1])
    G1 = herm_matrix(nt, ntau, 1, -1)
    O.dyson_mat(G1, W.sigma, d["mu"], H, d["beta"], k)
    O.dyson_start(G1, d["mu"], H, W.sigma, d["beta"], d["h"], k)
    G2 = G1.copy()
    for n in range(k + 1, nt + 1):
        O.dyson_timestep(n, G1, d["mu"], H, W.sigma, d["beta"], d["h"], k)
        O.dyson_timestep_omp(n, G2, d["mu"], H, W.sigma, d["beta"], d["h"], k)
    gaps = {c: _rel(getattr(G2, c), getattr(G1, c)) for c in ("ret", "les", "tv")}
    assert 1e-11 < gaps["ret"] < 1e-6 and 1e-11 < gaps["les"] < 1e-6, gaps
    assert gaps["tv"] < 1e-12, gaps
