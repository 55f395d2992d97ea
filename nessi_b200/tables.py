"""Quadrature and differentiation weights of libcntr's ``integration::Integrator``.

Every table is derived here from its mathematical definition in exact rational
arithmetic and rounded once to IEEE double.  The definitions follow the
documentation block of ``libcntr/cntr/integration.hpp:35-105``:

* ``poly_interpolation(a, l)``   coefficient of x**a in the Lagrange basis
  polynomial L_l on the nodes 0..k (the inverse Vandermonde matrix,
  integration.cpp:15-34).
* ``poly_differentiation(i, l)`` = L_l'(i)              (integration.cpp:37-57)
* ``poly_integration(i, j, l)``  = int_i^j L_l(x) dx     (integration.cpp:59-85)
* ``bd_weights(l)``, l=0..k+1: backward differentiation of order k+1,
  d/dx f(x0) = sum_l bd(l) f(x0-l)                       (integration.hpp:67-74)
* ``gregory_weights(m, j)``: Gregory quadrature int_0^m f = sum_j w(m,j) f_j.
  For m >= 2k+2 the weights are omega_j at both ends and 1 inside
  (integration.hpp:382-390).  omega_j are the end weights of Gregory's formula
  with differences up to order k.  Rows m <= k are polynomial (Newton-Cotes
  type) integrals over the nodes 0..k; rows k < m < 2k+2 overlap the two end
  corrections: w(m,j) = a_j + a_{m-j} - 1 with a_j = omega_j (j<=k) or 1.
* ``rcorr(m, j, l)``, 0<m<k: int_0^m L_j(m-x) L_l(x) dx, the Matsubara boundary
  correction (integration.hpp:50-62).

``tests/test_tables.py`` checks the Gregory, BD and rcorr tables against the
decimal tables hard-coded in libcntr (golden fixture), and the polynomial tables
against their defining identities.

Running this module writes ``csrc/cntr_tables.inc`` (hex-float literals) that the
CUDA library compiles in.
"""
from fractions import Fraction
import os

KMAX = 5  # MAX_SOLVE_ORDER of libcntr (cntr_global_settings.hpp:37)


def _poly_mul(a, b):
    out = [Fraction(0)] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        if x == 0:
            continue
        for j, y in enumerate(b):
            out[i + j] += x * y
    return out


def _poly_eval(p, x):
    acc = Fraction(0)
    for c in reversed(p):
        acc = acc * x + c
    return acc


def _poly_int(p, a, b):
    """int_a^b p(x) dx."""
    P = [Fraction(0)] + [c / (i + 1) for i, c in enumerate(p)]
    return _poly_eval(P, b) - _poly_eval(P, a)


def _poly_deriv(p):
    return [c * i for i, c in enumerate(p)][1:] or [Fraction(0)]


def lagrange_basis(nodes):
    """Coefficient lists (ascending powers) of the Lagrange basis on ``nodes``."""
    basis = []
    for l, xl in enumerate(nodes):
        p = [Fraction(1)]
        for j, xj in enumerate(nodes):
            if j != l:
                p = _poly_mul(p, [Fraction(-xj, 1) / (xl - xj), Fraction(1) / (xl - xj)])
        basis.append(p)
    return basis


def gregory_end_coeffs(kmax):
    """c_p, p=1..kmax: magnitudes of the Gregory coefficients (Bernoulli numbers of
    the second kind) G_{p+1} of x/ln(1+x) = sum_n G_n x**n."""
    G = [Fraction(1)]
    for n in range(1, kmax + 2):
        # sum_{j=0}^{n} G_j (-1)^(n-j)/(n-j+1) = 0
        s = sum(G[j] * Fraction((-1) ** (n - j), n - j + 1) for j in range(n))
        G.append(-s)
    return [None] + [(-1) ** p * G[p + 1] for p in range(1, kmax + 1)]


def _binom(n, r):
    from math import comb
    return comb(n, r)


def integrator(k):
    """All tables of the order-k integrator as exact Fractions."""
    assert 0 <= k <= KMAX
    k1, k2 = k + 1, 2 * (k + 1)
    L = lagrange_basis(list(range(k1)))
    interp = [[L[l][a] if a < len(L[l]) else Fraction(0) for l in range(k1)] for a in range(k1)]
    dL = [_poly_deriv(p) for p in L]
    diff = [[_poly_eval(dL[l], i) for l in range(k1)] for i in range(k1)]
    integ = [[[_poly_int(L[l], i, j) for l in range(k1)] for j in range(k1)] for i in range(k1)]

    # backward differentiation of order k+1 (nodes 0..k+1 in the backward direction)
    Lb = lagrange_basis(list(range(k + 2)))
    bd = [-_poly_eval(_poly_deriv(p), 0) for p in Lb]

    c = gregory_end_coeffs(max(k, 1))
    omega = []
    for j in range(k1):
        base = Fraction(1, 2) if j == 0 else Fraction(1)
        corr = sum(c[p] * _binom(p, j) for p in range(max(j, 1), k + 1))
        omega.append(base - (-1) ** j * corr)

    greg = [[Fraction(0)] * k2 for _ in range(k2)]
    for m in range(k1):
        for j in range(k1):
            greg[m][j] = integ[0][m][j]
    a = lambda j: omega[j] if j <= k else Fraction(1)
    for m in range(k1, k2):
        for j in range(m + 1):
            greg[m][j] = a(j) + a(m - j) - 1

    rcorr = []
    for m in range(1, k):
        blk = []
        for j in range(k1):
            # L_j(m - x): substitute
            pj = L[j]
            # compose p(m - x): expand sum c_i (m-x)^i
            comp = [Fraction(0)] * len(pj)
            for i, ci in enumerate(pj):
                term = [Fraction(1)]
                for _ in range(i):
                    term = _poly_mul(term, [Fraction(m), Fraction(-1)])
                for d, t in enumerate(term):
                    comp[d] += ci * t
            row = []
            for l in range(k1):
                row.append(_poly_int(_poly_mul(comp, L[l]), 0, m))
            blk.append(row)
        rcorr.append(blk)
    return {
        "k": k,
        "poly_interpolation": interp,
        "poly_differentiation": diff,
        "poly_integration": integ,
        "bd_weights": bd,
        "gregory_omega": omega,
        "gregory_weights": greg,
        "rcorr": rcorr,
    }


def gregory_weight(tab, m, j):
    """Integrator::gregory_weights(m, j) (integration.hpp:382-390) on a table."""
    k = tab["k"]
    k1, k2 = k + 1, 2 * (k + 1)
    if m >= k2:
        if k < j < m - k:
            return Fraction(1)
        if j < k1:
            return tab["gregory_omega"][j]
        return tab["gregory_omega"][m - j]
    return tab["gregory_weights"][m][j]


def _hex(x):
    return float(x).hex()


def emit_header(path):
    """Write the tables for k = 0..KMAX as C arrays of doubles.

    Layout per k (padded to KMAX): gregory[12*12] (row m, column j), omega[6],
    poly_int[6*6*6] (i, j, l), poly_diff[6*6] (i, l), poly_interp[6*6] (a, l),
    bd[7], rcorr[4*6*6] ((m-1), j, l).
    """
    K1 = KMAX + 1
    K2 = 2 * K1
    lines = ["/* Generated by nessi_b200/tables.py from exact rational arithmetic. Do not edit. */",
             "#define CNTR_KMAX %d" % KMAX]

    def arr(name, per_k, size):
        lines.append("static const double %s[%d][%d] = {" % (name, K1, size))
        for k in range(K1):
            vals = per_k(k)
            vals = vals + [0.0] * (size - len(vals))
            lines.append("  {" + ", ".join(_hex(v) for v in vals) + "},")
        lines.append("};")

    tabs = [integrator(k) for k in range(K1)]

    def greg(k):
        t = tabs[k]
        out = [Fraction(0)] * (K2 * K2)
        for m in range(2 * (k + 1)):
            for j in range(2 * (k + 1)):
                out[m * K2 + j] = t["gregory_weights"][m][j]
        return out

    def pint(k):
        t = tabs[k]
        out = [Fraction(0)] * (K1 * K1 * K1)
        for i in range(k + 1):
            for j in range(k + 1):
                for l in range(k + 1):
                    out[(i * K1 + j) * K1 + l] = t["poly_integration"][i][j][l]
        return out

    def sq(name):
        def f(k):
            t = tabs[k]
            out = [Fraction(0)] * (K1 * K1)
            for i in range(k + 1):
                for l in range(k + 1):
                    out[i * K1 + l] = t[name][i][l]
            return out
        return f

    def rc(k):
        t = tabs[k]
        out = [Fraction(0)] * ((K1 - 2) * K1 * K1)
        for m in range(1, k):
            for j in range(k + 1):
                for l in range(k + 1):
                    out[((m - 1) * K1 + j) * K1 + l] = t["rcorr"][m - 1][j][l]
        return out

    arr("cntr_tab_gregory", greg, K2 * K2)
    arr("cntr_tab_omega", lambda k: list(tabs[k]["gregory_omega"]), K1)
    arr("cntr_tab_poly_int", pint, K1 * K1 * K1)
    arr("cntr_tab_poly_diff", sq("poly_differentiation"), K1 * K1)
    arr("cntr_tab_poly_interp", sq("poly_interpolation"), K1 * K1)
    arr("cntr_tab_bd", lambda k: list(tabs[k]["bd_weights"]), K1 + 1)
    arr("cntr_tab_rcorr", rc, (K1 - 2) * K1 * K1)
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    emit_header(os.path.join(here, "csrc", "cntr_tables.inc"))
    print("wrote csrc/cntr_tables.inc")
