"""The host herm_matrix mirror (nessi_b200.herm_matrix) against libcntr's layout and the algebra
checks of libcntr/test/herm_matrix_member.cpp: element offsets (cntr_herm_matrix_impl.hpp:
457-477), the hermitian continuation of ret and les, incr_timestep and smul with complex and real
weights (herm_matrix_member.cpp:308-445), and the time-step slice round trip
(herm_matrix_member.cpp:447-466, herm_matrix_timestep_decl.hpp:67-75)."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from nessi_b200.herm_matrix import distance_norm2


def _random(rng, nt, ntau, s, sig):
    G = herm_matrix(nt, ntau, s, sig)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(G, c)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    return G


def test_offsets_are_libcntr_layout():
    nt, ntau, s = 6, 4, 3
    G = _random(np.random.default_rng(1), nt, ntau, s, -1)
    flat = {c: getattr(G, c).reshape(-1, s, s) for c in ("ret", "les", "tv", "mat")}
    for t in range(nt + 1):
        for t1 in range(t + 1):
            assert np.array_equal(G.get_ret(t, t1), flat["ret"][t * (t + 1) // 2 + t1])
            assert np.array_equal(G.get_les(t1, t), flat["les"][t * (t + 1) // 2 + t1])
        for m in range(ntau + 1):
            assert np.array_equal(G.get_tv(t, m), flat["tv"][t * (ntau + 1) + m])
        assert np.array_equal(G.ret_row(t), flat["ret"][t * (t + 1) // 2:t * (t + 1) // 2 + t + 1])
        assert np.array_equal(G.les_col(t), flat["les"][t * (t + 1) // 2:t * (t + 1) // 2 + t + 1])
    for m in range(ntau + 1):
        assert np.array_equal(G.get_mat(m), flat["mat"][m])


def test_hermitian_continuation():
    """G^R(t,t') for t < t' and G^<(t,t') for t > t' from the stored triangle:
    X(t,t') = -X(t',t)^dagger (cntr_herm_matrix_impl.hpp get_ret / get_les)."""
    G = _random(np.random.default_rng(2), 5, 3, 2, -1)
    for t in range(6):
        for t1 in range(6):
            if t1 > t:
                assert np.array_equal(G.get_ret(t, t1), -G.get_ret(t1, t).conj().T)
            if t > t1:
                assert np.array_equal(G.get_les(t, t1), -G.get_les(t1, t).conj().T)


@pytest.mark.parametrize("w", [0.3 - 1.7j, 2.5])
def test_incr_timestep_and_smul(w):
    rng = np.random.default_rng(3)
    nt, ntau, s = 8, 5, 2
    G1, G2 = _random(rng, nt, ntau, s, -1), _random(rng, nt, ntau, s, -1)
    G3 = herm_matrix(nt, ntau, s, -1)  # element by element, as the reference test builds it
    for c in ("ret", "les", "tv", "mat"):
        getattr(G3, c)[...] = getattr(G1, c) + w * getattr(G2, c)
    G4 = G1.copy()
    for t in range(-1, nt + 1):
        G4.incr_timestep(t, G2, w)
    assert sum(distance_norm2(t, G3, G4) for t in range(-1, nt + 1)) < 1e-12
    for c in ("ret", "les", "tv", "mat"):
        getattr(G3, c)[...] = w * getattr(G1, c)
    G5 = G1.copy()
    for t in range(-1, nt + 1):
        G5.smul(t, w)
    assert sum(distance_norm2(t, G3, G5) for t in range(-1, nt + 1)) < 1e-12


def test_timestep_slices_round_trip():
    rng = np.random.default_rng(4)
    nt, ntau, s = 7, 4, 3
    G1 = _random(rng, nt, ntau, s, 1)
    G2 = herm_matrix(nt, ntau, s, 1)
    for t in range(-1, nt + 1):
        sl = G1.get_timestep(t)
        assert sl.shape == ((ntau + 1, s, s) if t < 0 else (2 * (t + 1) + ntau + 1, s, s))
        G2.set_timestep_data(t, sl)
    for c in ("ret", "les", "tv", "mat"):
        assert np.array_equal(getattr(G1, c), getattr(G2, c))


def test_bad_dimensions_raise():
    for args in ((-2, 4, 1, -1), (3, -1, 1, -1), (3, 4, 0, -1), (3, 4, 1, 0)):
        with pytest.raises(ValueError):
            herm_matrix(*args)


def test_distance_norm2_definition(oracle):
    """libcntr/test/utilities.cpp:380-450: distance_norm2(tstp) is the sum over the time step's
    elements (ret row, tv row, les column; mat for -1) of the Frobenius norm of the difference;
    the host function, the oracle and an explicit loop agree for two free 2 x 2 propagators."""
    nt, ntau, beta, h = 10, 20, 5.0, 0.05
    h1 = np.array([[-1.0, -0.7j], [0.7j, 0.8]])
    h2 = np.array([[-2.0, -1.4j], [1.4j, 1.6]])
    G1, G2 = herm_matrix(nt, ntau, 2, -1), herm_matrix(nt, ntau, 2, -1)
    oracle.green_from_H(G1, 0.0, h1, beta, h)
    oracle.green_from_H(G2, 0.0, h2, beta, h)
    for t in range(-1, nt + 1):
        if t < 0:
            ref = sum(np.linalg.norm(G1.mat[m] - G2.mat[m]) for m in range(ntau + 1))
        else:
            ref = (sum(np.linalg.norm(G1.get_ret(t, j) - G2.get_ret(t, j)) for j in range(t + 1)) +
                   sum(np.linalg.norm(G1.get_tv(t, m) - G2.get_tv(t, m)) for m in range(ntau + 1)) +
                   sum(np.linalg.norm(G1.get_les(j, t) - G2.get_les(j, t)) for j in range(t + 1)))
        assert abs(distance_norm2(t, G1, G2) - ref) <= 1e-12 * ref
        assert abs(oracle.distance_norm2(t, G1, G2) - ref) <= 1e-12 * ref


def test_force_matsubara_hermitian(oracle):
    """utilities.cpp:452-486: G^M + i G2^M made hermitian again at every tau."""
    ntau, beta = 20, 5.0
    G1, G2 = herm_matrix(-1, ntau, 2, -1), herm_matrix(-1, ntau, 2, -1)
    oracle.green_from_H(G1, 0.0, np.array([[-1.0, -0.7j], [0.7j, 0.8]]), beta, 0.05)
    oracle.green_from_H(G2, 0.0, np.array([[0.8, 0.7], [0.7, -1.0]]), beta, 0.05)
    G1.incr_timestep(-1, G2, 1j)
    assert max(np.linalg.norm(m - m.conj().T) for m in G1.mat) > 1e-3
    oracle.force_matsubara_hermitian(G1)
    assert sum(np.linalg.norm(m - m.conj().T) for m in G1.mat) < 1e-14
