"""The oracle's restatement of the GW self-energy diagrams of examples/programs/gw_selfene_impl.cpp
(the polarisation P_q = -sum_k w_k Bubble1(G_{k-q}, G_k) and Sigma_k = sum_q w_q
Bubble2(G_{k-q}, W_q), with gw_latt_impl.cpp's k-point arithmetic) against closed forms: for
free G_k of a chain and free bosonic W_q every bubble is a product of closed forms, so P and
Sigma are explicit sums over the grid."""
import numpy as np

from nessi_b200 import herm_matrix
from nessi_b200.herm_matrix import distance_norm2
from test_oracle_bubble import FreeLevels, _bubble_ref

NK, NT, NTAU, BETA, H = 6, 10, 20, 2.0, 0.05


def _grid():
    ks = (np.arange(NK) - NK // 2) * 2 * np.pi / NK
    # dispersions without k -> -k or k -> k + pi symmetry, so that k - q and k + q differ
    Gf = [FreeLevels(-2.0 * np.cos(k - 0.4) + 0.5 * np.cos(2 * k) + 0.3, -1, BETA) for k in ks]
    Wf = [FreeLevels(1.0 + 0.5 * np.cos(k) + 0.2 * np.sin(k), 1, BETA) for k in ks]
    return ks, Gf, Wf


def test_add_kpoints_is_the_grid_arithmetic(oracle):
    ks = (np.arange(NK) - NK // 2) * 2 * np.pi / NK
    for k1 in range(NK):
        for k2 in range(NK):
            for s1, s2 in ((1, 1), (1, -1), (-1, 1)):
                i = oracle.add_kpoints(NK, k1, s1, k2, s2)
                d = s1 * ks[k1] + s2 * ks[k2] - ks[i]
                assert abs(np.exp(1j * d) - 1) < 1e-12  # equal modulo 2 pi


def test_polarization_and_gw_sigma_closed_forms(oracle):
    _, Gf, Wf = _grid()
    w = np.full(NK, 1.0 / NK)
    Gs = [g.herm_matrix(NT, NTAU, H) for g in Gf]
    Ws = [x.herm_matrix(NT, NTAU, H) for x in Wf]
    for q in (0, 1, NK // 2):
        P, Pref = herm_matrix(NT, NTAU, 1, 1), herm_matrix(NT, NTAU, 1, 1)
        for kk in range(NK):
            kq = oracle.add_kpoints(NK, kk, 1, q, -1)
            B = _bubble_ref(1, Gf[kq], Gf[kk], NT, NTAU, H)
            for c in ("ret", "les", "tv", "mat"):
                getattr(Pref, c)[...] -= w[kk] * getattr(B, c)
        err = 0.0
        for t in range(-1, NT + 1):
            oracle.gw_polarization_timestep(t, P, q, Gs, w)
            err += distance_norm2(t, P, Pref)
        assert err < 1e-10, (q, err)
    for kk in (0, 2):
        S, Sref = herm_matrix(NT, NTAU, 1, -1), herm_matrix(NT, NTAU, 1, -1)
        for q in range(NK):
            kq = oracle.add_kpoints(NK, kk, 1, q, -1)
            B = _bubble_ref(2, Gf[kq], Wf[q], NT, NTAU, H)
            for c in ("ret", "les", "tv", "mat"):
                getattr(Sref, c)[...] += w[q] * getattr(B, c)
        err = 0.0
        for t in range(-1, NT + 1):
            oracle.gw_sigma_timestep(t, S, kk, Gs, Ws, w)
            err += distance_norm2(t, S, Sref)
        assert err < 1e-10, (kk, err)
