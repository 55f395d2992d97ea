"""ctypes binding of the oracle (oracle/libcntr_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the nessi_b200 package.  Functions take
any object with the attributes of ``nessi_b200.herm_matrix.herm_matrix``
(nt, ntau, size1, sig and contiguous complex128 arrays ret/les/tv/mat) and
operate on those arrays in place, following libcntr's serial routines (see
cntr_oracle.hpp for the reference lines).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "libcntr_oracle.so")
_lib = None

CNTR_MAT_FOURIER = 0
CNTR_MAT_CG = 1
CNTR_MAT_FIXPOINT = 2


class _OrcHM(ctypes.Structure):
    _fields_ = [("nt", ctypes.c_int), ("ntau", ctypes.c_int), ("size", ctypes.c_int), ("sig", ctypes.c_int),
                ("ret", ctypes.c_void_p), ("les", ctypes.c_void_p), ("tv", ctypes.c_void_p),
                ("mat", ctypes.c_void_p)]


def build():
    """Compile the oracle with its Makefile (system g++, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        P = ctypes.POINTER(_OrcHM)
        d, i, vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
        sig = {
            "orc_gregory_weights": (d, [i, i, i]),
            "orc_gregory_omega": (d, [i, i]),
            "orc_poly_integration": (d, [i, i, i, i]),
            "orc_poly_differentiation": (d, [i, i, i]),
            "orc_poly_interpolation": (d, [i, i, i]),
            "orc_bd_weights": (d, [i, i]),
            "orc_rcorr": (d, [i, i, i, i]),
            "orc_cplx_solve": (i, [i, i, vp, vp, vp]),
            "orc_green_from_H_const": (None, [P, d, vp, d, d]),
            "orc_convolution_timestep": (None, [i, P, P, P, P, P, i, d, d]),
            "orc_convolution_matsubara": (None, [P, P, P, i, d]),
            "orc_dyson_mat": (None, [P, P, d, vp, i, d, i, i]),
            "orc_dyson_start": (None, [P, d, vp, P, i, d, d]),
            "orc_dyson_timestep": (None, [i, P, d, vp, P, i, d, d]),
            "orc_vie2_mat": (None, [P, P, P, P, d, i, i]),
            "orc_vie2_start": (None, [P, P, P, P, i, d, d]),
            "orc_vie2_timestep": (None, [i, P, P, P, P, i, d, d, i]),
            "orc_extrapolate_timestep": (None, [i, P, i]),
            "orc_distance_norm2": (d, [i, P, P]),
            "orc_force_matsubara_hermitian": (None, [P]),
            "orc_bubble1_scalar": (None, [i, P, P, P, P, P]),
            "orc_bubble2_scalar": (None, [i, P, P, P, P, P]),
            "orc_vie2_timestep_sin": (None, [i, P, vp, P, P, vp, P, vp, i, d, d]),
            "orc_bubble1": (None, [i, P, i, i, P, P, i, i, P, P, i, i]),
            "orc_bubble2": (None, [i, P, i, i, P, P, i, i, P, P, i, i]),
            "orc_dyson_timestep_batch": (None, [i, i, i, P, d, vp, ctypes.c_long, P, i, d, d, i]),
            "orc_sigma_2b_timestep": (None, [i, P, P, vp]),
            "orc_gloc_timestep": (None, [i, i, P, P]),
            "orc_lattice2b_start": (i, [i, P, P, P, vp, d, vp, ctypes.c_long, i, d, d, i, d,
                                        ctypes.POINTER(ctypes.c_double), i]),
            "orc_lattice2b_timestep": (None, [i, i, P, P, P, vp, d, vp, ctypes.c_long, i, d, d, i, i]),
            "orc_incr_convolution_part": (None, [i, i, vp, d, d, P, P, P, vp, P, P, i, d, d]),
            "orc_incr_convolution": (None, [i, d, d, P, P, P, vp, P, P, i, d, d]),
            "orc_dyson_timestep_omp": (None, [i, P, d, vp, P, i, d, d]),
            "orc_vie2_timestep_omp": (None, [i, P, P, P, P, i, d, d, i]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    if a is None or a.size == 0:
        return None
    assert a.dtype == np.complex128 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def hm(G):
    """ctypes view of a herm_matrix-like object (keeps no copy)."""
    return _OrcHM(G.nt, G.ntau, G.size1, G.sig, _ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat))


def _H(H):
    a = H.data if hasattr(H, "data") and not isinstance(H, np.ndarray) else H
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a, a.ctypes.data


# --- tables -------------------------------------------------------------------------
def gregory_weights(k, m, j):
    return lib().orc_gregory_weights(k, m, j)


def gregory_omega(k, j):
    return lib().orc_gregory_omega(k, j)


def poly_integration(k, i, j, l):
    return lib().orc_poly_integration(k, i, j, l)


def poly_differentiation(k, i, l):
    return lib().orc_poly_differentiation(k, i, l)


def poly_interpolation(k, a, l):
    return lib().orc_poly_interpolation(k, a, l)


def bd_weights(k, l):
    return lib().orc_bd_weights(k, l)


def rcorr(k, m, j, l):
    return lib().orc_rcorr(k, m, j, l)


def cplx_solve(M, Q):
    M = np.ascontiguousarray(M, np.complex128)
    Q = np.ascontiguousarray(Q, np.complex128)
    n = M.shape[0]
    Q2 = Q.reshape(n, -1)
    X = np.zeros_like(Q2)
    st = lib().orc_cplx_solve(n, Q2.shape[1], M.ctypes.data, Q2.ctypes.data, X.ctypes.data)
    return st, X.reshape(Q.shape)


# --- contour routines ------------------------------------------------------------------
def green_from_H(G, mu, H0, beta, h):
    H0 = np.ascontiguousarray(np.asarray(H0, np.complex128).reshape(G.size1, G.size1))
    g = hm(G)
    lib().orc_green_from_H_const(ctypes.byref(g), mu, H0.ctypes.data, beta, h)


def convolution_timestep(n, C, A, Acc, B, Bcc, beta, h, k=5):
    c, a, acc, b, bcc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    lib().orc_convolution_timestep(n, ctypes.byref(c), ctypes.byref(a), ctypes.byref(acc), ctypes.byref(b),
                                   ctypes.byref(bcc), k, beta, h)


def convolution_matsubara(C, A, B, beta, k=5):
    c, a, b = hm(C), hm(A), hm(B)
    lib().orc_convolution_matsubara(ctypes.byref(c), ctypes.byref(a), ctypes.byref(b), k, beta)


def dyson_mat(G, Sigma, mu, H, beta, k=5, method=CNTR_MAT_FIXPOINT, force_hermitian=True):
    g, s = hm(G), hm(Sigma)
    Ha, hp = _H(H)
    lib().orc_dyson_mat(ctypes.byref(g), ctypes.byref(s), mu, hp, k, beta, method, int(force_hermitian))


def dyson_start(G, mu, H, Sigma, beta, h, k=5):
    g, s = hm(G), hm(Sigma)
    Ha, hp = _H(H)
    lib().orc_dyson_start(ctypes.byref(g), mu, hp, ctypes.byref(s), k, beta, h)


def dyson_timestep(n, G, mu, H, Sigma, beta, h, k=5):
    g, s = hm(G), hm(Sigma)
    Ha, hp = _H(H)
    lib().orc_dyson_timestep(n, ctypes.byref(g), mu, hp, ctypes.byref(s), k, beta, h)


def _ft(ft):
    """function data with F(-1) first (a cntr::function-like object or its array), or None"""
    if ft is None:
        return None, None
    a = ft.data if hasattr(ft, "data") and not isinstance(ft, np.ndarray) else ft
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a, a.ctypes.data


def incr_convolution(tstp, alpha, C, A, Acc, B, Bcc, beta, h, k=5, ft=None):
    """cntr incr_convolution (cntr_convolution_impl.hpp:4786-4807): C += alpha A * ft * B at tstp."""
    c, a, acc, b, bcc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    fa, fp = _ft(ft)
    alpha = complex(alpha)
    lib().orc_incr_convolution(tstp, alpha.real, alpha.imag, ctypes.byref(c), ctypes.byref(a), ctypes.byref(acc), fp,
                               ctypes.byref(b), ctypes.byref(bcc), k, beta, h)


def incr_convolution_part(which, tstp, mask, alpha, C, A, Acc, B, Bcc, beta, h, k=5, ft=None):
    """One component of incr_convolution (0 mat, 1 ret, 2 tv, 3 les) restricted to a mask
    (sequence of bools, ntau+1 or tstp+1 entries; None = all)."""
    c, a, acc, b, bcc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    fa, fp = _ft(ft)
    mk = None if mask is None else np.ascontiguousarray(np.asarray(mask, dtype=np.int8))
    alpha = complex(alpha)
    lib().orc_incr_convolution_part(which, tstp, None if mk is None else mk.ctypes.data, alpha.real, alpha.imag,
                                    ctypes.byref(c), ctypes.byref(a), ctypes.byref(acc), fp, ctypes.byref(b),
                                    ctypes.byref(bcc), k, beta, h)


def convolution_timestep_new(n, C, A, Acc, B, Bcc, beta, h, k=5, ft=None):
    """cntr convolution_timestep_new (cntr_convolution_impl.hpp:4811-4976): time step n of C
    zeroed, then incr_convolution with alpha = 1."""
    if n == -1:
        C.mat[...] = 0
    else:
        _zero_timestep(C, n)
    incr_convolution(n, 1.0, C, A, Acc, B, Bcc, beta, h, k, ft)


def dyson_timestep_omp(n, G, mu, H, Sigma, beta, h, k=5):
    """cntr::dyson_timestep_omp (cntr_dyson_omp_impl.hpp:577-605), k + 1 <= n."""
    assert k + 1 <= n
    g, s = hm(G), hm(Sigma)
    Ha, hp = _H(H)
    lib().orc_dyson_timestep_omp(n, ctypes.byref(g), mu, hp, ctypes.byref(s), k, beta, h)


def vie2_timestep_omp(n, G, F, Fcc, Q, beta, h, k=5, method=CNTR_MAT_FIXPOINT):
    """cntr::vie2_timestep_omp (cntr_vie2_impl.hpp:2125-2190)."""
    g, f, fc, q = hm(G), hm(F), hm(Fcc), hm(Q)
    lib().orc_vie2_timestep_omp(n, ctypes.byref(g), ctypes.byref(f), ctypes.byref(fc), ctypes.byref(q), k, beta, h,
                                method)


def vie2_mat(G, F, Fcc, Q, beta, k=5, method=CNTR_MAT_FIXPOINT):
    g, f, fc, q = hm(G), hm(F), hm(Fcc), hm(Q)
    lib().orc_vie2_mat(ctypes.byref(g), ctypes.byref(f), ctypes.byref(fc), ctypes.byref(q), beta, k, method)


def vie2_start(G, F, Fcc, Q, beta, h, k=5):
    g, f, fc, q = hm(G), hm(F), hm(Fcc), hm(Q)
    lib().orc_vie2_start(ctypes.byref(g), ctypes.byref(f), ctypes.byref(fc), ctypes.byref(q), k, beta, h)


def vie2_timestep(n, G, F, Fcc, Q, beta, h, k=5, method=CNTR_MAT_FIXPOINT):
    g, f, fc, q = hm(G), hm(F), hm(Fcc), hm(Q)
    lib().orc_vie2_timestep(n, ctypes.byref(g), ctypes.byref(f), ctypes.byref(fc), ctypes.byref(q), k, beta, h,
                            method)


def vie2_timestep_sin(n, G, Gsin, F, Fcc, Fsin, Q, Qsin, beta, h, k=5):
    """cntr::vie2_timestep_sin (cntr_vie2_impl.hpp:1779-1838); Gsin, Fsin, Qsin are cntr::function
    objects (or their (nt+2, s, s) data); Gsin is written for t = -1..max(n, k)."""
    g, f, fc, q = hm(G), hm(F), hm(Fcc), hm(Q)
    arr = lambda X: X.data if hasattr(X, "data") and not isinstance(X, np.ndarray) else X
    gs, fs, qs = arr(Gsin), np.ascontiguousarray(arr(Fsin), np.complex128), np.ascontiguousarray(arr(Qsin), np.complex128)
    assert gs.dtype == np.complex128 and gs.flags["C_CONTIGUOUS"]
    lib().orc_vie2_timestep_sin(n, ctypes.byref(g), gs.ctypes.data, ctypes.byref(f), ctypes.byref(fc),
                                fs.ctypes.data, ctypes.byref(q), qs.ctypes.data, k, beta, h)


def extrapolate_timestep(n, G, k=5):
    g = hm(G)
    lib().orc_extrapolate_timestep(n, ctypes.byref(g), k)


def distance_norm2(tstp, g1, g2):
    a, b = hm(g1), hm(g2)
    return lib().orc_distance_norm2(tstp, ctypes.byref(a), ctypes.byref(b))


def force_matsubara_hermitian(G):
    g = hm(G)
    lib().orc_force_matsubara_hermitian(ctypes.byref(g))


def bubble1(tstp, C, A, Acc, B, Bcc):
    c, a, acc, b, bcc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    lib().orc_bubble1_scalar(tstp, ctypes.byref(c), ctypes.byref(a), ctypes.byref(acc), ctypes.byref(b),
                             ctypes.byref(bcc))


def bubble2(tstp, C, A, Acc, B, Bcc):
    c, a, acc, b, bcc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    lib().orc_bubble2_scalar(tstp, ctypes.byref(c), ctypes.byref(a), ctypes.byref(acc), ctypes.byref(b),
                             ctypes.byref(bcc))


def bubble1_el(tstp, C, c, A, Acc, a, B, Bcc, b):
    """C_{c1c2}(t,t') = i A_{a1a2}(t,t') B_{b2b1}(t',t) at tstp; c, a, b are index pairs."""
    hc, ha, hac, hb, hbc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    lib().orc_bubble1(tstp, ctypes.byref(hc), c[0], c[1], ctypes.byref(ha), ctypes.byref(hac), a[0], a[1],
                      ctypes.byref(hb), ctypes.byref(hbc), b[0], b[1])


def bubble2_el(tstp, C, c, A, Acc, a, B, Bcc, b):
    """C_{c1c2}(t,t') = i A_{a1a2}(t,t') B_{b1b2}(t,t') at tstp; c, a, b are index pairs."""
    hc, ha, hac, hb, hbc = hm(C), hm(A), hm(Acc), hm(B), hm(Bcc)
    lib().orc_bubble2(tstp, ctypes.byref(hc), c[0], c[1], ctypes.byref(ha), ctypes.byref(hac), a[0], a[1],
                      ctypes.byref(hb), ctypes.byref(hbc), b[0], b[1])


def add_kpoints(nk, k1, s1, k2, s2):
    """Index of s1 k1 + s2 k2 on the 1-d grid k_i = (i - nk/2) 2 pi / nk (gw_latt_impl.cpp:46-51)."""
    g = nk // 2
    return (s1 * (k1 - g) + s2 * (k2 - g) + g) % nk


def _zero_timestep(G, tstp):
    if tstp == -1:
        G.mat[...] = 0
    else:
        G.ret_row(tstp)[...] = 0
        G.tv[tstp] = 0
        G.les_col(tstp)[...] = 0


def gw_polarization_timestep(tstp, P, q, Gs, weights):
    """get_Polarization_Bubble (examples/programs/gw_selfene_impl.cpp:133-153):
    P_q(tstp) = -sum_k w_k Bubble1(G_{k-q}, G_k), element by element (a1 a2 = b1 b2 = c1 c2)."""
    from nessi_b200 import herm_matrix
    s = P.size1
    _zero_timestep(P, tstp)
    tmp = herm_matrix(P.nt, P.ntau, s, P.sig)
    for kk in range(len(Gs)):
        kq = add_kpoints(len(Gs), kk, 1, q, -1)
        _zero_timestep(tmp, tstp)
        for i1 in range(s):
            for i2 in range(s):
                bubble1_el(tstp, tmp, (i1, i2), Gs[kq], Gs[kq], (i1, i2), Gs[kk], Gs[kk], (i1, i2))
        P.incr_timestep(tstp, tmp, -weights[kk])


def gw_sigma_timestep(tstp, S, kk, Gs, Ws, weights):
    """sigma_GW (examples/programs/gw_selfene_impl.cpp:114-131):
    Sigma_k(tstp) = sum_q w_q Bubble2(G_{k-q}, W_q), element by element."""
    from nessi_b200 import herm_matrix
    s = S.size1
    _zero_timestep(S, tstp)
    tmp = herm_matrix(S.nt, S.ntau, s, S.sig)
    for q in range(len(Ws)):
        kq = add_kpoints(len(Gs), kk, 1, q, -1)
        _zero_timestep(tmp, tstp)
        for i1 in range(s):
            for i2 in range(s):
                bubble2_el(tstp, tmp, (i1, i2), Gs[kq], Gs[kq], (i1, i2), Ws[q], Ws[q], (i1, i2))
        S.incr_timestep(tstp, tmp, weights[q])


def dyson_timestep_batch(n0, n1, Gs, mu, Hs, Sigma, beta, h, k=5, nthreads=0):
    """Time steps n0..n1 for every problem in ``Gs`` (shared Sigma), OpenMP over problems.
    ``Hs`` is an array (nprob, nt+2, s, s)."""
    arr = (_OrcHM * len(Gs))(*[hm(G) for G in Gs])
    Ha = np.ascontiguousarray(Hs, np.complex128)
    stride = Ha[0].size
    s = hm(Sigma)
    lib().orc_dyson_timestep_batch(n0, n1, len(Gs), arr, mu, Ha.ctypes.data, stride, ctypes.byref(s), k, beta, h,
                                   nthreads)


def _U(U):
    a = np.ascontiguousarray(U, np.complex128)
    return a, a.ctypes.data


def sigma_2b_timestep(tstp, Sigma, G, U):
    """Sigma(tstp) = Sigma_2B[G, U] (hubbard_chain_selfen_impl.cpp:63-75).  ``U`` is an
    (nt+2, s, s) array, U(-1) first."""
    s, g = hm(Sigma), hm(G)
    Ua, up = _U(U)
    lib().orc_sigma_2b_timestep(tstp, ctypes.byref(s), ctypes.byref(g), up)


def gloc_timestep(tstp, Gs, Gloc):
    arr = (_OrcHM * len(Gs))(*[hm(G) for G in Gs])
    l = hm(Gloc)
    lib().orc_gloc_timestep(tstp, len(Gs), arr, ctypes.byref(l))


def lattice2b_start(Gs, Gloc, Sigma, U, mu, Hs, beta, h, k=5, max_iter=20, tol=1e-12, nthreads=0):
    """Bootstrap of the lattice (hubbard_chain_2b.cpp:245-290 with G -> G_loc).
    Returns (iterations, last error)."""
    arr = (_OrcHM * len(Gs))(*[hm(G) for G in Gs])
    Ha = np.ascontiguousarray(Hs, np.complex128)
    Ua, up = _U(U)
    l, s = hm(Gloc), hm(Sigma)
    err = ctypes.c_double()
    it = lib().orc_lattice2b_start(len(Gs), arr, ctypes.byref(l), ctypes.byref(s), up, mu, Ha.ctypes.data,
                                   Ha[0].size, k, beta, h, max_iter, tol, ctypes.byref(err), nthreads)
    return it, err.value


def lattice2b_timestep(n, Gs, Gloc, Sigma, U, mu, Hs, beta, h, k=5, ncorr=3, nthreads=0):
    """One lattice time step: predictor + ncorr x [G_loc, Sigma_2B, dyson_timestep]."""
    arr = (_OrcHM * len(Gs))(*[hm(G) for G in Gs])
    Ha = np.ascontiguousarray(Hs, np.complex128)
    Ua, up = _U(U)
    l, s = hm(Gloc), hm(Sigma)
    lib().orc_lattice2b_timestep(n, len(Gs), arr, ctypes.byref(l), ctypes.byref(s), up, mu, Ha.ctypes.data,
                                 Ha[0].size, k, beta, h, ncorr, nthreads)
