"""The oracle's three Matsubara methods against libcntr's own known answer (libcntr/test/
matsubara.cpp:33-106): a level eps1 = -1 hybridised (lambda = 0.2) with a level eps2 = 1, solved
as a 1x1 problem with the embedding self-energy Sigma = lambda^2 g_2; the exact G is the (0,0)
element of the 2x2 equilibrium propagator.  libcntr requires distance_norm2(-1) < 1e-3 for the
Fourier method and < 1e-7 for the fixpoint and steepest-descent methods; the same bounds here."""
import numpy as np
import pytest

from nessi_b200 import distance_norm2, herm_matrix

FOURIER, CG, FIXPOINT = 0, 1, 2


def embedding_case(O):
    beta, ntau, lam, e1, e2 = 20.0, 400, 0.2, -1.0, 1.0
    h2 = np.array([[e1, 1j * lam], [-1j * lam, e2]])
    G2 = herm_matrix(-1, ntau, 2, -1)
    O.green_from_H(G2, 0.0, h2, beta, 1.0)
    exact = herm_matrix(-1, ntau, 1, -1)
    exact.mat[:, 0, 0] = G2.mat[:, 0, 0]
    Sig = herm_matrix(-1, ntau, 1, -1)
    O.green_from_H(Sig, 0.0, np.array([[e2]], complex), beta, 1.0)
    Sig.mat[...] *= lam * lam
    return exact, Sig, np.array([[e1]], complex), beta


@pytest.mark.parametrize("method,tol", [(FOURIER, 1e-3), (FIXPOINT, 1e-7), (CG, 1e-7)])
def test_oracle_matsubara_methods_known_answer(oracle, method, tol):
    from nessi_b200 import function
    exact, Sig, h1, beta = embedding_case(oracle)
    H = function(-1, 1)
    H.set_value(-1, h1)
    G = herm_matrix(-1, exact.ntau, 1, -1)
    oracle.dyson_mat(G, Sig, 0.0, H, beta, 5, method=method)
    assert distance_norm2(-1, exact, G) < tol
