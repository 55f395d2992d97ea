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
