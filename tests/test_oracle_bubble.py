"""Known answers of the bubbles behind Sigma_2B, after libcntr/test/bubble.cpp: for free
equilibrium propagators set from their closed forms, Bubble1 C(t,t') = i A(t,t') B(t',t) and
Bubble2 C(t,t') = i A(t,t') B(t,t') are products of closed forms, and the oracle must reproduce
them at every time step (bubble.cpp:569-816: nt = 200, ntau = 500, beta = 0.5, h = 0.02,
levels 1.123 / 0.345, all four Fermi/Bose pairings, summed distance_norm2 < 1e-8).  The size-N
case (bubble.cpp:818-890: 2 x 2, levels rotated by a unitary) is checked through the whole
Sigma_2B of a rotated G with a time-dependent diagonal U, the function the device kernel
k_sigma_2b is compared with."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from nessi_b200.herm_matrix import distance_norm2
from builders import u_matrices

II = 1j


class FreeLevels:
    """Closed forms of the free equilibrium propagator of H = R^dagger diag(w) R (sign sg):
    n = 1/(e^{beta w} - sg), G^<(t,t') = -sg i n e^{-iw(t-t')}, G^>(t,t') = -i(1+sg n) e^{-iw(t-t')},
    G^tv(t,tau) = -sg i n e^{-iwt} e^{w tau}, G^vt(tau,t) = -i(1+sg n) e^{-w tau} e^{iwt},
    G^M(tau) = -(1+sg n) e^{-w tau} on [0, beta].  Times broadcast: arrays give (..., s, s)."""

    def __init__(self, w, sg, beta, R=None):
        self.w = np.atleast_1d(np.asarray(w, float))
        self.sg, self.beta = sg, beta
        self.R = np.eye(len(self.w)) if R is None else np.asarray(R, complex)
        self.n = 1.0 / (np.exp(beta * self.w) - sg)

    def _rot(self, d):  # R^dagger diag(d) R for every leading index of d (..., s)
        return np.einsum("li,...l,lj->...ij", self.R.conj(), d, self.R)

    @staticmethod
    def _x(a):
        return np.asarray(a, float)[..., None]

    def les(self, t1, t2):
        return self._rot(-self.sg * II * self.n * np.exp(-II * self.w * (self._x(t1) - self._x(t2))))

    def gtr(self, t1, t2):
        return self._rot(-II * (1 + self.sg * self.n) * np.exp(-II * self.w * (self._x(t1) - self._x(t2))))

    def tv(self, t, tau):
        return self._rot(-self.sg * II * self.n * np.exp(-II * self.w * self._x(t)) * np.exp(self.w * self._x(tau)))

    def vt(self, tau, t):
        return self._rot(-II * (1 + self.sg * self.n) * np.exp(-self.w * self._x(tau)) * np.exp(II * self.w * self._x(t)))

    def mat(self, tau):
        return self._rot(-(1 + self.sg * self.n) * np.exp(-self.w * self._x(tau)))

    def herm_matrix(self, nt, ntau, h):
        G = herm_matrix(nt, ntau, len(self.w), self.sg)
        taus = np.arange(ntau + 1) * (self.beta / ntau)
        T, TAU = np.meshgrid(np.arange(nt + 1) * h, taus, indexing="ij")
        a, b = tri_times(nt, h)
        G.mat[...] = self.mat(taus)
        G.tv[...] = self.tv(T, TAU)
        G.ret[...] = self.gtr(a, b) - self.les(a, b)   # ret(t, t1), t1 <= t
        G.les[...] = self.les(b, a)                    # les(t1, t) at les_index(t1, t) = ret_index(t, t1)
        return G


def tri_times(nt, h):
    """(t h, t1 h) of the packed triangle entries in order: ret_index(t, t1) = les_index(t1, t)."""
    t = np.concatenate([np.full(i + 1, i) for i in range(nt + 1)])
    t1 = np.concatenate([np.arange(i + 1) for i in range(nt + 1)])
    return t * h, t1 * h


def _bubble_ref(kind, A, B, nt, ntau, h):
    """Closed form of Bubble1 (kind 1) or Bubble2 (kind 2) of two scalar free propagators."""
    C = herm_matrix(nt, ntau, 1, A.sg * B.sg)
    beta = A.beta
    taus = np.arange(ntau + 1) * (beta / ntau)
    T, TAU = np.meshgrid(np.arange(nt + 1) * h, taus, indexing="ij")
    a, b = tri_times(nt, h)
    if kind == 1:  # C^M(tau) = -A^M(tau) B^M(-tau), B^M(-tau) = sg_b B^M(beta - tau)
        C.mat[...] = -A.mat(taus) * B.sg * B.mat(beta - taus)
        C.tv[...] = II * A.tv(T, TAU) * B.vt(TAU, T)
        C.ret[...] = II * A.gtr(a, b) * B.les(b, a) - II * A.les(a, b) * B.gtr(b, a)
        C.les[...] = II * A.les(b, a) * B.gtr(a, b)
    else:
        C.mat[...] = -A.mat(taus) * B.mat(taus)
        C.tv[...] = II * A.tv(T, TAU) * B.tv(T, TAU)
        C.ret[...] = II * A.gtr(a, b) * B.gtr(a, b) - II * A.les(a, b) * B.les(a, b)
        C.les[...] = II * A.les(b, a) * B.les(b, a)
    return C


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("sa,sb", [(-1, -1), (-1, 1), (1, -1), (1, 1)])
def test_scalar_bubbles_of_free_propagators(oracle, kind, sa, sb):
    nt, ntau, beta, h = 200, 500, 0.5, 0.02
    A, B = FreeLevels(1.123, sa, beta), FreeLevels(0.345, sb, beta)
    GA, GB = A.herm_matrix(nt, ntau, h), B.herm_matrix(nt, ntau, h)
    R = _bubble_ref(kind, A, B, nt, ntau, h)
    C = herm_matrix(nt, ntau, 1, sa * sb)
    f = oracle.bubble1 if kind == 1 else oracle.bubble2
    err = 0.0
    for t in range(-1, nt + 1):
        f(t, C, GA, GA, GB, GB)
        err += distance_norm2(t, C, R)
    assert err < 1e-8, err


def test_sigma_2b_of_rotated_free_levels(oracle):
    """Sigma_2B[G, U] of a 2 x 2 G = R^dagger g(w) R (bubble.cpp:818-849 levels and rotation) with a
    real, time-dependent diagonal U, against its closed form:
      Pol_ij(t,t') = -i G_ij(t,t') G_ji(t',t),  Pol'_ij = U_i(t) Pol_ij U_j(t'),
      Sigma_ij(t,t') = i G_ij(t,t') Pol'_ij(t,t')    (U(-1) on the Matsubara side)."""
    nt, ntau, beta, h, s = 50, 50, 0.5, 0.02, 2
    R = np.array([[np.cos(1.0), -np.sin(1.0)], [np.sin(1.0), np.cos(1.0)]])
    F = FreeLevels([1.123, 0.567], -1, beta, R)
    G = F.herm_matrix(nt, ntau, h)
    rng = np.random.default_rng(7)
    # a physical (real) interaction: with it Pol' keeps the hermitian symmetry that the herm_matrix
    # storage of Pol' assumes, so the closed form over all (t, t') is the reference's result
    U = rng.normal(1.0, 0.3, (nt + 2, s)).astype(complex)
    taus = np.arange(ntau + 1) * (beta / ntau)
    T, TAU = np.meshgrid(np.arange(nt + 1) * h, taus, indexing="ij")
    a, b = tri_times(nt, h)
    it, it1 = np.rint(a / h).astype(int), np.rint(b / h).astype(int)
    sg = -1
    ref = herm_matrix(nt, ntau, s, sg)
    Tr = lambda X: np.swapaxes(X, -1, -2)
    UU = lambda left, right: left[..., :, None] * right[..., None, :]  # U_i(t) x U_j(t')
    pol = sg * F.mat(taus) * Tr(F.mat(beta - taus))              # -Bubble1 on the Matsubara branch
    ref.mat[...] = -F.mat(taus) * pol * UU(U[0], U[0])
    pol = -II * F.tv(T, TAU) * Tr(F.vt(TAU, T))
    ref.tv[...] = II * F.tv(T, TAU) * pol * UU(U[1:][:, None, :], U[0])
    pgtr = -II * F.gtr(a, b) * Tr(F.les(b, a)) * UU(U[it + 1], U[it1 + 1])
    ples = -II * F.les(a, b) * Tr(F.gtr(b, a)) * UU(U[it + 1], U[it1 + 1])
    ref.ret[...] = II * F.gtr(a, b) * pgtr - II * F.les(a, b) * ples
    pl = -II * F.les(b, a) * Tr(F.gtr(a, b)) * UU(U[it1 + 1], U[it + 1])  # Pol'^<(t1, t)
    ref.les[...] = II * F.les(b, a) * pl
    S = herm_matrix(nt, ntau, s, sg)
    err = 0.0
    for t in range(-1, nt + 1):
        oracle.sigma_2b_timestep(t, S, G, u_matrices(U))
        err += distance_norm2(t, S, ref)
    assert err < 1e-8, err


def _bubble_ref_el(kind, A, B, nt, ntau, h):
    """Closed form of the element bubbles with c = a = b = (i, j) for every (i, j):
    Bubble1 C_ij = i A_ij(t,t') B_ji(t',t), Bubble2 C_ij = i A_ij(t,t') B_ij(t,t')."""
    s = len(A.w)
    C = herm_matrix(nt, ntau, s, A.sg * B.sg)
    beta = A.beta
    Tr = lambda X: np.swapaxes(X, -1, -2)
    taus = np.arange(ntau + 1) * (beta / ntau)
    T, TAU = np.meshgrid(np.arange(nt + 1) * h, taus, indexing="ij")
    a, b = tri_times(nt, h)
    if kind == 1:
        C.mat[...] = -A.mat(taus) * B.sg * Tr(B.mat(beta - taus))
        C.tv[...] = II * A.tv(T, TAU) * Tr(B.vt(TAU, T))
        C.ret[...] = II * A.gtr(a, b) * Tr(B.les(b, a)) - II * A.les(a, b) * Tr(B.gtr(b, a))
        C.les[...] = II * A.les(b, a) * Tr(B.gtr(a, b))
    else:
        C.mat[...] = -A.mat(taus) * B.mat(taus)
        C.tv[...] = II * A.tv(T, TAU) * B.tv(T, TAU)
        C.ret[...] = II * A.gtr(a, b) * B.gtr(a, b) - II * A.les(a, b) * B.les(a, b)
        C.les[...] = II * A.les(b, a) * B.les(b, a)
    return C


@pytest.mark.parametrize("kind", [1, 2])
@pytest.mark.parametrize("sa,sb", [(-1, -1), (-1, 1), (1, -1), (1, 1)])
def test_element_bubbles_of_rotated_free_levels(oracle, kind, sa, sb):
    """libcntr/test/bubble.cpp:818-1161: 2 x 2 free propagators with levels (1.123, 0.567) and
    (0.345, 0.876) rotated by 1 and 2 radians, nt = ntau = 50, beta = 0.5, h = 0.02; every
    element bubble C_ij from A_ij and B_ji (Bubble1) or B_ij (Bubble2), all four Fermi/Bose
    pairings, summed distance_norm2 < 1e-8."""
    nt, ntau, beta, h = 50, 50, 0.5, 0.02
    rot = lambda x: np.array([[np.cos(x), -np.sin(x)], [np.sin(x), np.cos(x)]])
    A = FreeLevels([1.123, 0.567], sa, beta, rot(1.0))
    B = FreeLevels([0.345, 0.876], sb, beta, rot(2.0))
    GA, GB = A.herm_matrix(nt, ntau, h), B.herm_matrix(nt, ntau, h)
    R = _bubble_ref_el(kind, A, B, nt, ntau, h)
    C = herm_matrix(nt, ntau, 2, sa * sb)
    f = oracle.bubble1_el if kind == 1 else oracle.bubble2_el
    err = 0.0
    for t in range(-1, nt + 1):
        for i in range(2):
            for j in range(2):
                f(t, C, (i, j), GA, GA, (i, j), GB, GB, (i, j))
        err += distance_norm2(t, C, R)
    assert err < 1e-8, err
