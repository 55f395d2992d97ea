"""Free (non-interacting) Green's functions used to build inputs: the bath of the
self-energies and the problem Hamiltonians.  Host-side set-up code, not on the time-stepping
path.  Follows libcntr's green_from_H for a constant Hamiltonian
(libcntr/cntr/cntr_equilibrium_impl.hpp:873-955) with numpy's Hermitian eigensolver:

  G^M(tau)  = -V f_exp(beta, tau, e) V^dag            (fermions; bosons: +b_exp)
  U(t)      = exp(i h Hmu)^n,   Hmu = -H0 + mu
  G^tv(t,tau) = i U(t) V f_exp(beta, tau, -e) V^dag   (bosons: -i, b_exp)
  G^R(t,t') = -i U(t) U(t')^dag
  G^<(t',t) = i U(t') V f(-e) V^dag U(t)^dag          (bosons: -b(-e))
"""
import numpy as np

from .herm_matrix import herm_matrix

EXPMAX = 100.0


def fermi(beta, w):
    arg = w * beta
    if abs(arg) > EXPMAX:
        return 0.0 if arg > 0 else 1.0
    return 1.0 / (1.0 + np.exp(arg))


def fermi_exp(beta, tau, w):
    if w < 0:
        return np.exp(w * tau) * fermi(beta, w)
    return np.exp((tau - beta) * w) * fermi(beta, -w)


def bose(beta, w):
    arg = w * beta
    if arg < 0:
        return -1.0 - bose(beta, -w)
    if abs(arg) > EXPMAX:
        return 0.0
    if arg < 1e-10:
        return 1.0 / arg
    return 1.0 / (np.exp(arg) - 1.0)


def bose_exp(beta, tau, w):
    if w < 0:
        return np.exp(tau * w) * bose(beta, w)
    return -np.exp((tau - beta) * w) * bose(beta, -w)


def green_from_H(G, mu, H0, beta, h):
    """Fill herm_matrix G with the free propagator of the constant Hamiltonian H0."""
    s, nt, ntau, sign = G.size1, G.nt, G.ntau, G.sig
    H0 = np.asarray(H0, np.complex128).reshape(s, s)
    Hmu = -H0 + mu * np.eye(s)
    ev, V = np.linalg.eigh(Hmu)
    Vh = V.conj().T
    dtau = beta / ntau
    for m in range(ntau + 1):
        tau = m * dtau
        d = [-fermi_exp(beta, tau, e) if sign == -1 else bose_exp(beta, tau, e) for e in ev]
        G.mat[m] = (V * d) @ Vh
    if nt < 0:
        return
    Udt = (V * np.exp(1j * h * ev)) @ Vh
    U = np.empty((nt + 1, s, s), np.complex128)
    U[0] = np.eye(s)
    for n in range(1, nt + 1):
        U[n] = U[n - 1] @ Udt
    pref = 1j if sign == -1 else -1j
    for m in range(ntau + 1):
        tau = m * dtau
        d = [fermi_exp(beta, tau, -e) if sign == -1 else bose_exp(beta, tau, -e) for e in ev]
        f = (V * d) @ Vh
        G.tv[:, m] = pref * (U @ f)
    d = [fermi(beta, -e) if sign == -1 else -bose(beta, -e) for e in ev]
    val = (V * d) @ Vh
    Ud = U.conj().transpose(0, 2, 1)
    for t in range(nt + 1):
        # ret(t, 0..t) = -i U(t) U(t')^dag ; les(t', t) = i U(t') val U(t)^dag
        G.ret_row(t)[...] = -1j * np.einsum("ab,nbc->nac", U[t], Ud[:t + 1])
        G.les_col(t)[...] = 1j * np.einsum("nab,bc->nac", U[:t + 1] @ val, Ud[t])


def semicircle_bath(nt, ntau, beta, h, nlev=201, half_bandwidth=2.0, sig=-1):
    """G_bath = sum_i w_i green_from_H(eps_i): nlev equidistant levels in [-D, D] weighted by
    the semicircle density sqrt(D^2 - e^2), normalised to 1 (scalar, size1 = 1)."""
    D = half_bandwidth
    eps = np.linspace(-D, D, nlev)
    w = np.sqrt(np.maximum(D * D - eps * eps, 0.0))
    w /= w.sum()
    Gb = herm_matrix(nt, ntau, 1, sig)
    # scalar closed form of green_from_H, vectorised over the triangle
    R = np.repeat(np.arange(nt + 1), np.arange(1, nt + 2)) if nt >= 0 else np.zeros(0, int)
    C = (np.arange(R.size) - R * (R + 1) // 2) if nt >= 0 else R
    taus = np.arange(ntau + 1) * (beta / ntau)
    ret = Gb.ret[:, 0, 0]
    les = Gb.les[:, 0, 0]
    tv = Gb.tv[:, :, 0, 0]
    mat = Gb.mat[:, 0, 0]
    fer = sig == -1
    for e, wi in zip(eps, w):
        if wi == 0.0:
            continue
        ev = -e  # eigenvalue of -H0 + mu, mu = 0
        fexp = np.array([fermi_exp(beta, t, ev) if fer else bose_exp(beta, t, ev) for t in taus])
        mat += wi * (-fexp if fer else fexp)
        if nt < 0:
            continue
        u = np.exp(1j * h * ev * np.arange(nt + 1))
        fexm = np.array([fermi_exp(beta, t, -ev) if fer else bose_exp(beta, t, -ev) for t in taus])
        tv += wi * (1j if fer else -1j) * np.outer(u, fexm)
        f0 = fermi(beta, -ev) if fer else -bose(beta, -ev)
        ret += wi * (-1j) * u[R] * np.conj(u[C])
        les += wi * 1j * f0 * u[C] * np.conj(u[R])
    return Gb


def kron_identity(G1, s, scale=1.0):
    """scale * G1 (x) 1_s: a scalar contour function repeated on the diagonal of s x s blocks."""
    G = herm_matrix(G1.nt, G1.ntau, s, G1.sig)
    for i in range(s):
        G.ret[:, i, i] = scale * G1.ret[:, 0, 0]
        G.les[:, i, i] = scale * G1.les[:, 0, 0]
        G.tv[..., i, i] = scale * G1.tv[..., 0, 0]
        G.mat[:, i, i] = scale * G1.mat[:, 0, 0]
    return G
