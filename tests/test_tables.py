"""Integration weights: the CUDA library's exact-rational tables and the oracle's own
long-double derivation, both against the decimal tables hard-coded in libcntr
(libcntr/cntr/integration.cpp:152-1180, captured in tests/golden/integration_tables.json)
and against the defining identities of the polynomial tables."""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

from nessi_b200 import tables as T

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "integration_tables.json")))


@pytest.mark.parametrize("k", range(0, 6))
def test_exact_tables_match_reference_bitwise(k):
    t = T.integrator(k)
    W = GOLD["gregory"][str(k)]["weights"]
    for m in range(len(W)):
        for j in range(len(W)):
            assert float(t["gregory_weights"][m][j]) == float(W[m][j]), (k, m, j)
    for j in range(k + 1):
        assert float(t["gregory_omega"][j]) == float(GOLD["gregory"][str(k)]["omega"][j])
    bd = GOLD["bd"][str(k + 1)]
    for l in range(k + 2):
        assert float(t["bd_weights"][l]) == float(bd[l])
    if k >= 2:
        rc, k1 = GOLD["rcorr"][str(k)], k + 1
        for m in range(1, k):
            for j in range(k1):
                for l in range(k1):
                    assert float(t["rcorr"][m - 1][j][l]) == float(rc[(m - 1) * k1 * k1 + j * k1 + l])


@pytest.mark.parametrize("k", range(0, 6))
def test_polynomial_tables_identities(k):
    t = T.integrator(k)
    # poly_integration(i,j,l) integrates x^p exactly for p <= k; differentiation likewise
    for p in range(k + 1):
        for i in range(k + 1):
            for j in range(k + 1):
                s = sum(t["poly_integration"][i][j][l] * Fraction(l) ** p for l in range(k + 1))
                assert s == Fraction(j ** (p + 1) - i ** (p + 1), p + 1)
            d = sum(t["poly_differentiation"][i][l] * Fraction(l) ** p for l in range(k + 1))
            assert d == (p * Fraction(i) ** (p - 1) if p > 0 else 0)


@pytest.mark.parametrize("k", range(0, 6))
def test_oracle_tables_match(oracle, k):
    t = T.integrator(k)
    k1, k2 = k + 1, 2 * (k + 1)
    for m in range(k2):
        for j in range(m + 1 if m >= k1 else k1):
            assert oracle.gregory_weights(k, m, j) == pytest.approx(float(t["gregory_weights"][m][j]), abs=2e-16)
    for m in range(k2, k2 + 8):
        for j in range(m + 1):
            assert oracle.gregory_weights(k, m, j) == float(T.gregory_weight(t, m, j))
    for l in range(k + 2):
        assert oracle.bd_weights(k, l) == pytest.approx(float(t["bd_weights"][l]), abs=1e-15)
    for i in range(k1):
        for l in range(k1):
            assert oracle.poly_differentiation(k, i, l) == pytest.approx(float(t["poly_differentiation"][i][l]), abs=1e-13)
            assert oracle.poly_interpolation(k, i, l) == pytest.approx(float(t["poly_interpolation"][i][l]), abs=1e-13)
            for j in range(k1):
                assert oracle.poly_integration(k, i, j, l) == pytest.approx(float(t["poly_integration"][i][j][l]), abs=1e-13)
    for m in range(1, k):
        for j in range(k1):
            for l in range(k1):
                assert oracle.rcorr(k, m, j, l) == pytest.approx(float(t["rcorr"][m - 1][j][l]), abs=1e-14)


def test_rcorr_known_answers(oracle):
    """libcntr/test/integration.cpp:94-125: boundary integrals of two fermionic exponentials."""
    from math import exp
    k, ntau, beta, e1, e2 = 5, 100, 5.0, -0.1, 0.2
    dtau = beta / ntau

    def fermi(b, w):
        return 1.0 / (1.0 + exp(w * b))

    def fermi_exp(b, tau, w):
        return exp(w * tau) * fermi(b, w) if w < 0 else exp((tau - b) * w) * fermi(b, -w)

    A = np.array([-fermi_exp(beta, m * dtau, -e1) for m in range(ntau + 1)])
    B = np.array([-fermi_exp(beta, m * dtau, -e2) for m in range(ntau + 1)])
    R_exact = {1: 0.0137659, 2: 0.0274638, 3: 0.0410948, 4: 0.0546598}
    err = 0.0
    for m in range(1, k):
        R = sum(dtau * oracle.rcorr(k, m, j, l) * A[j] * B[l] for j in range(k + 1) for l in range(k + 1))
        err += abs(R_exact[m] - R)
    assert err < 1.0e-4


def test_emitted_header_matches_tables(tmp_path):
    p = tmp_path / "t.inc"
    T.emit_header(str(p))
    committed = open(os.path.join(os.path.dirname(T.__file__), "csrc", "cntr_tables.inc")).read()
    assert p.read_text() == committed
