"""The oracle against libcntr's own output: the golden densities of the Falicov-Kimball Bethe-lattice
quench of libcntr/test/fkm_bethe_quench.cpp ("Reference calculation for fkm - commit cae14da"),
stored by the reference in fkm_bethe_quench.h5 and extracted to tests/golden/fkm_bethe_quench.json
by tests/golden/make_fkm_golden.py.

The test restates the reference test's driver with the oracle's routines:
    G0 = [i d/dt + mu - f0 - Delta]^-1,  G1 = [i d/dt + mu - f1 - Delta]^-1,  G = (G0 + G1)/2,  Delta = G
with f0 = -U/2, f1 = +U/2 (U0 = 1 on the Matsubara branch, U1 = 2 for t >= 0), nt = 50, ntau = 200,
beta = 5, h = 0.01, order 5: the Matsubara fixpoint by dyson_mat (Fourier method), the bootstrap
by dyson_start iterated to convergence, then per step extrapolate_timestep of Delta and three
dyson_timestep sweeps.  The densities rho(t) of G0 and G1 (herm_matrix::density_matrix,
cntr_herm_matrix_impl.hpp:984-995) must match libcntr's within the reference's bound
(sum_t |rho - rho_ref|^2 < 1e-7); the restatement reaches 9e-24, max |rho - rho_ref| = 4.8e-13."""
import json
import os

import numpy as np

from nessi_b200 import function, herm_matrix
from nessi_b200.herm_matrix import distance_norm2

HERE = os.path.dirname(os.path.abspath(__file__))
NT, NTAU, KT, BETA, H, U0, U1 = 50, 200, 5, 5.0, 0.01, 1.0, 2.0
ERRMAX, ITERMAX, ITER_RTIME = 1e-7, 100, 3


def bethe_mat(G, beta, npts=400):
    """G^M(tau) of the semicircular density of states A(w) = sqrt(4 - w^2) / (2 pi) (the Bethe
    lattice of bandwidth 4 that green_equilibrium_mat_bethe uses as the initial Delta):
    G^M(tau) = -int dw A(w) e^{-tau w} / (1 + e^{-beta w}), by Gauss-Chebyshev quadrature of the
    second kind (w = 2 cos theta).  Only the starting point of the Matsubara iteration; the
    converged result does not depend on it."""
    j = np.arange(1, npts + 1)
    theta = j * np.pi / (npts + 1)
    w = 2.0 * np.cos(theta)
    weight = (2.0 / (npts + 1)) * np.sin(theta) ** 2  # int A(w) dw = 1
    taus = np.arange(NTAU + 1) * (beta / NTAU)
    for m, tau in enumerate(taus):
        # e^{-tau w} / (1 + e^{-beta w}) without overflow on either side of w = 0
        f = np.where(w > 0, np.exp(-tau * w) / (1 + np.exp(-beta * w)),
                     np.exp((beta - tau) * w) / (np.exp(beta * w) + 1))
        G.mat[m, 0, 0] = -np.sum(weight * f)


def density(G, t):
    """herm_matrix::density_matrix(t): -G^M(beta) for t = -1, i sig G^<(t,t) otherwise."""
    if t == -1:
        return (-G.mat[NTAU, 0, 0]).real
    return (1j * G.sig * G.les[G.les_index(t, t), 0, 0]).real


class FKM:
    """State of the fkm_bethe_quench.cpp driver: G0, G1, their mean G and the hybridisation Delta."""

    def __init__(self):
        self.G0, self.G1, self.G, self.Delta = (herm_matrix(NT, NTAU, 1, -1) for _ in range(4))
        bethe_mat(self.Delta, BETA)
        self.f0, self.f1 = function(NT, 1), function(NT, 1)
        self.f0.set_value(-1, [[-U0 * 0.5]])
        self.f1.set_value(-1, [[U0 * 0.5]])
        for t in range(NT + 1):
            self.f0.set_value(t, [[-U1 * 0.5]])
            self.f1.set_value(t, [[U1 * 0.5]])
        self.mu = 0.0

    def mix(self, t):
        """G(t) = (G0(t) + G1(t)) / 2."""
        self.G.set_timestep(t, self.G0)
        self.G.smul(t, 0.5)
        self.G.incr_timestep(t, self.G1, 0.5)

    def densities(self):
        return (np.array([density(self.G0, t) for t in range(-1, NT + 1)]),
                np.array([density(self.G1, t) for t in range(-1, NT + 1)]))


def fkm_equilibrium_and_bootstrap(O):
    """Steps 1 and 2 of the reference driver: the Matsubara self-consistency and the bootstrap."""
    s = FKM()
    gtemp = herm_matrix(KT, NTAU, 1, -1)
    converged = False
    for it in range(ITERMAX + 1):
        O.dyson_mat(s.G0, s.Delta, s.mu, s.f0, BETA, KT, method=O.CNTR_MAT_FOURIER)
        O.dyson_mat(s.G1, s.Delta, s.mu, s.f1, BETA, KT, method=O.CNTR_MAT_FOURIER)
        s.mix(-1)
        err = distance_norm2(-1, s.G, gtemp)
        if err < ERRMAX and it > 2:
            converged = True
            break
        gtemp.set_timestep(-1, s.G)
        s.Delta.set_timestep(-1, s.G)
    assert converged
    for it in range(ITERMAX + 1):
        O.dyson_start(s.G0, s.mu, s.f0, s.Delta, BETA, H, KT)
        O.dyson_start(s.G1, s.mu, s.f1, s.Delta, BETA, H, KT)
        for t in range(KT + 1):
            s.mix(t)
        err = sum(distance_norm2(t, s.G, gtemp) for t in range(KT + 1))
        if err < ERRMAX:
            break
        for t in range(KT + 1):
            gtemp.set_timestep(t, s.G)
            s.Delta.set_timestep(t, s.G)
    return s


def run_fkm(O):
    s = fkm_equilibrium_and_bootstrap(O)
    # step 3: time stepping with the predictor for Delta and three corrector sweeps
    for t in range(KT + 1, NT + 1):
        O.extrapolate_timestep(t - 1, s.Delta, KT)
        for _ in range(ITER_RTIME):
            O.dyson_timestep(t, s.G0, s.mu, s.f0, s.Delta, BETA, H, KT)
            O.dyson_timestep(t, s.G1, s.mu, s.f1, s.Delta, BETA, H, KT)
            s.mix(t)
            s.Delta.set_timestep(t, s.G)
    return s.densities()


def golden():
    return json.load(open(os.path.join(HERE, "golden", "fkm_bethe_quench.json")))


def test_golden_fixture_shape():
    ref = golden()
    assert len(ref["den0"]) == len(ref["den1"]) == NT + 2
    # half filling of the two species: rho0 + rho1 = 1 in equilibrium
    assert abs(ref["den0"][0] + ref["den1"][0] - 1.0) < 1e-9


def test_fkm_densities_match_libcntr(oracle):
    ref = golden()
    d0, d1 = run_fkm(oracle)
    err0 = float(np.sum(np.abs(d0 - np.array(ref["den0"])) ** 2))
    err1 = float(np.sum(np.abs(d1 - np.array(ref["den1"])) ** 2))
    assert err0 < ERRMAX and err1 < ERRMAX      # fkm_bethe_quench.cpp:145-151 (errmax)
    # what the restatement reaches: 4.8e-13 (libcntr's output carries its own rounding)
    assert max(np.max(np.abs(d0 - ref["den0"])), np.max(np.abs(d1 - ref["den1"]))) < 1e-11
