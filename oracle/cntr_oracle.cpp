// Oracle: CPU restatement of libcntr's serial Kadanoff-Baym path (test infrastructure).
// See cntr_oracle.hpp for scope and storage conventions.  Reference paths below are
// relative to the libcntr project root (libcntr/cntr/...).
#include "cntr_oracle.hpp"

#include <cassert>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef ocplx cplx;
static const double kPi = 3.14159265358979323846;  // fourier.hpp:25
static const cplx kI(0.0, 1.0);

// ------------------------------------------------------------------------------------
// Integrator (integration.hpp:128-504).  Tables are derived from their definitions in
// long double: Lagrange basis on nodes 0..k, Gregory end weights from Gregory's
// coefficients, overlap rows for k < m < 2k+2.  tests/test_tables.py pins them against
// the reference's decimal tables.
// ------------------------------------------------------------------------------------
namespace {

typedef long double ld;

struct Poly {
    std::vector<ld> c;  // ascending powers
};

static Poly pmul(const Poly &a, const Poly &b) {
    Poly r;
    r.c.assign(a.c.size() + b.c.size() - 1, 0.0L);
    for (size_t i = 0; i < a.c.size(); i++)
        for (size_t j = 0; j < b.c.size(); j++) r.c[i + j] += a.c[i] * b.c[j];
    return r;
}
static ld peval(const Poly &p, ld x) {
    ld acc = 0;
    for (size_t i = p.c.size(); i-- > 0;) acc = acc * x + p.c[i];
    return acc;
}
static ld pint(const Poly &p, ld a, ld b) {
    ld sa = 0, sb = 0, pa = a, pb = b;
    for (size_t i = 0; i < p.c.size(); i++) {
        sa += p.c[i] * pa / (ld)(i + 1);
        sb += p.c[i] * pb / (ld)(i + 1);
        pa *= a;
        pb *= b;
    }
    return sb - sa;
}
static ld pderiv_at(const Poly &p, ld x) {
    ld acc = 0, xp = 1;
    for (size_t i = 1; i < p.c.size(); i++) {
        acc += (ld)i * p.c[i] * xp;
        xp *= x;
    }
    return acc;
}
static std::vector<Poly> lagrange(int npts) {
    std::vector<Poly> out;
    for (int l = 0; l < npts; l++) {
        Poly p;
        p.c = {1.0L};
        for (int j = 0; j < npts; j++) {
            if (j == l) continue;
            Poly f;
            f.c = {-(ld)j / (ld)(l - j), 1.0L / (ld)(l - j)};
            p = pmul(p, f);
        }
        out.push_back(p);
    }
    return out;
}

struct Integ {
    int k = -1;
    std::vector<double> interp, diff, integ, bd, greg, omega, rc;

    void init(int kk) {
        k = kk;
        int k1 = k + 1, k2 = 2 * k1;
        std::vector<Poly> L = lagrange(k1);
        interp.assign(k1 * k1, 0.0);
        diff.assign(k1 * k1, 0.0);
        integ.assign(k1 * k1 * k1, 0.0);
        for (int a = 0; a < k1; a++)
            for (int l = 0; l < k1; l++)
                interp[a * k1 + l] = (double)(a < (int)L[l].c.size() ? L[l].c[a] : 0.0L);
        for (int i = 0; i < k1; i++)
            for (int l = 0; l < k1; l++) diff[i * k1 + l] = (double)pderiv_at(L[l], (ld)i);
        for (int i = 0; i < k1; i++)
            for (int j = 0; j < k1; j++)
                for (int l = 0; l < k1; l++)
                    integ[(i * k1 + j) * k1 + l] = (double)pint(L[l], (ld)i, (ld)j);
        // BDF of order k+1: bd(l) = -L'_l(0) on nodes 0..k+1
        std::vector<Poly> Lb = lagrange(k + 2);
        bd.assign(k + 2, 0.0);
        for (int l = 0; l < k + 2; l++) bd[l] = (double)(-pderiv_at(Lb[l], 0.0L));
        // Gregory coefficients G_n of x/ln(1+x); c_p = (-1)^p G_{p+1}
        int kc = k < 1 ? 1 : k;
        std::vector<ld> G(kc + 2, 0.0L);
        G[0] = 1.0L;
        for (int n = 1; n <= kc + 1; n++) {
            ld s = 0;
            for (int j = 0; j < n; j++) s += G[j] * (((n - j) % 2) ? -1.0L : 1.0L) / (ld)(n - j + 1);
            G[n] = -s;
        }
        std::vector<ld> omg(k1);
        for (int j = 0; j < k1; j++) {
            ld base = (j == 0) ? 0.5L : 1.0L, corr = 0;
            for (int p = (j > 1 ? j : 1); p <= k; p++) {
                ld cp = ((p % 2) ? -1.0L : 1.0L) * G[p + 1];
                ld binom = 1;
                for (int r = 0; r < j; r++) binom = binom * (ld)(p - r) / (ld)(r + 1);
                corr += cp * binom;
            }
            omg[j] = base - ((j % 2) ? -1.0L : 1.0L) * corr;
        }
        omega.assign(k1, 0.0);
        for (int j = 0; j < k1; j++) omega[j] = (double)omg[j];
        greg.assign(k2 * k2, 0.0);
        for (int m = 0; m < k1; m++)
            for (int j = 0; j < k1; j++) greg[m * k2 + j] = (double)pint(L[j], 0.0L, (ld)m);
        for (int m = k1; m < k2; m++)
            for (int j = 0; j <= m; j++) {
                ld aj = j <= k ? omg[j] : 1.0L, am = (m - j) <= k ? omg[m - j] : 1.0L;
                greg[m * k2 + j] = (double)(aj + am - 1.0L);
            }
        rc.assign(k > 1 ? (k - 1) * k1 * k1 : 0, 0.0);
        for (int m = 1; m < k; m++)
            for (int j = 0; j < k1; j++) {
                // L_j(m - x) as a polynomial in x
                Poly comp;
                comp.c.assign(k1, 0.0L);
                for (int i = 0; i < (int)L[j].c.size(); i++) {
                    Poly t;
                    t.c = {1.0L};
                    Poly f;
                    f.c = {(ld)m, -1.0L};
                    for (int r = 0; r < i; r++) t = pmul(t, f);
                    for (size_t d = 0; d < t.c.size(); d++) comp.c[d] += L[j].c[i] * t.c[d];
                }
                for (int l = 0; l < k1; l++)
                    rc[((m - 1) * k1 + j) * k1 + l] = (double)pint(pmul(comp, L[l]), 0.0L, (ld)m);
            }
    }
    double poly_interpolation(int a, int l) const { return interp[a * (k + 1) + l]; }
    double poly_differentiation(int i, int l) const { return diff[i * (k + 1) + l]; }
    double poly_integration(int i, int j, int l) const {
        return integ[(i * (k + 1) + j) * (k + 1) + l];
    }
    double bd_weights(int l) const { return bd[l]; }
    double gregory_omega(int j) const { return omega[j]; }
    // integration.hpp:382-390
    double gregory_weights(int n, int j) const {
        int k1 = k + 1, k2 = 2 * k1;
        if (n >= k2) {
            if (j > k && j < n - k) return 1.0;
            if (j < k1) return omega[j];
            return omega[n - j];
        }
        return greg[n * k2 + j];
    }
    // integration.hpp:439-444
    double rcorr(int m, int j, int l) const {
        if (k < 2) return 0.0;
        return rc[((m - 1) * (k + 1) + j) * (k + 1) + l];
    }
};

// integration::I<T>(k) (integration.hpp:506-514); built once, before any threads.
static Integ g_integ[6];
static bool g_integ_ready = false;
static void integ_init_all() {
    if (g_integ_ready) return;
    for (int k = 0; k <= 5; k++) g_integ[k].init(k);
    g_integ_ready = true;
}
static const Integ &I(int k) {
    integ_init_all();
    return g_integ[k];
}

// ------------------------------------------------------------------------------------
// herm_matrix view (cntr_herm_matrix_impl.hpp:457-477)
// ------------------------------------------------------------------------------------
struct HM {
    orc_hm *h;
    int s, es;
    explicit HM(orc_hm *hh) : h(hh), s(hh->size), es(hh->size * hh->size) {}
    int nt() const { return h->nt; }
    int ntau() const { return h->ntau; }
    int sig() const { return h->sig; }
    cplx *retptr(int i, int j) const { return h->ret + ((long)i * (i + 1) / 2 + j) * es; }
    cplx *lesptr(int i, int j) const { return h->les + ((long)j * (j + 1) / 2 + i) * es; }
    cplx *tvptr(int i, int m) const { return h->tv + ((long)i * (h->ntau + 1) + m) * es; }
    cplx *matptr(int m) const { return h->mat + (long)m * es; }
};

// ------------------------------------------------------------------------------------
// Element kernels (cntr_elements.hpp).  S1 == 1 selects the scalar specialisation.
// ------------------------------------------------------------------------------------
template <int S1> struct El {
    int s, es;
    explicit El(int ss) : s(ss), es(ss * ss) {}
    void zero(cplx *z) const {
        if (S1 == 1) *z = 0; else for (int i = 0; i < es; i++) z[i] = 0;
    }
    void set(cplx *z, const cplx *z1) const {
        if (S1 == 1) *z = *z1; else for (int i = 0; i < es; i++) z[i] = z1[i];
    }
    void set_diag(cplx *z, cplx z0) const {
        zero(z);
        for (int i = 0; i < s; i++) z[i * s + i] = z0;
    }
    // z = z1^dagger (element_conj, cntr_elements.hpp:41-52)
    void conj(cplx *z, const cplx *z1) const {
        if (S1 == 1) { *z = std::conj(*z1); return; }
        for (int l = 0; l < s; l++)
            for (int m = 0; m < s; m++) z[l * s + m] = std::conj(z1[m * s + l]);
    }
    void conj_inplace(cplx *z) const {
        if (S1 == 1) { *z = std::conj(*z); return; }
        std::vector<cplx> t(z, z + es);
        conj(z, t.data());
    }
    // z = -z1^dagger (element_minusconj)
    void minusconj(cplx *z, const cplx *z1) const {
        if (S1 == 1) { *z = -std::conj(*z1); return; }
        for (int l = 0; l < s; l++)
            for (int m = 0; m < s; m++) z[l * s + m] = -std::conj(z1[m * s + l]);
    }
    void smul(cplx *z, cplx a) const {
        if (S1 == 1) *z *= a; else for (int i = 0; i < es; i++) z[i] *= a;
    }
    void incr(cplx *z, const cplx *z1) const {
        if (S1 == 1) *z += *z1; else for (int i = 0; i < es; i++) z[i] += z1[i];
    }
    void incr(cplx *z, cplx a, const cplx *z1) const {
        if (S1 == 1) *z += a * (*z1); else for (int i = 0; i < es; i++) z[i] += a * z1[i];
    }
    // z += z1 * z2
    void incr(cplx *z, const cplx *z1, const cplx *z2) const {
        if (S1 == 1) { *z += (*z1) * (*z2); return; }
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) {
                cplx acc = 0;
                for (int l = 0; l < s; l++) acc += z1[i * s + l] * z2[l * s + j];
                z[i * s + j] += acc;
            }
    }
    // z += a * (z1 * z2)
    void incr(cplx *z, cplx a, const cplx *z1, const cplx *z2) const {
        if (S1 == 1) { *z += a * (*z1) * (*z2); return; }
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) {
                cplx acc = 0;
                for (int l = 0; l < s; l++) acc += z1[i * s + l] * z2[l * s + j];
                z[i * s + j] += a * acc;
            }
    }
    void mult(cplx *z, const cplx *z1, const cplx *z2) const {
        if (S1 == 1) { *z = (*z1) * (*z2); return; }
        std::vector<cplx> t(es, 0.0);
        incr(t.data(), z1, z2);
        set(z, t.data());
    }
    void inverse(cplx *z, const cplx *z1) const;
    void linsolve_right(int n, cplx *X, const cplx *M, const cplx *Q) const;
    void linsolve_left(int n, cplx *X, const cplx *M, const cplx *Q) const;
};

}  // namespace

// Solve M X = Q by Gaussian elimination with complete pivoting (FullPivLU,
// linalg_eigen.cpp:91-104).  M is n x n row-major, Q/X are n x nrhs row-major.
extern "C" int orc_cplx_solve(int n, int nrhs, const cplx *M, const cplx *Q, cplx *X) {
    std::vector<cplx> A(M, M + (long)n * n), B(Q, Q + (long)n * nrhs);
    std::vector<int> colp(n);
    for (int i = 0; i < n; i++) colp[i] = i;
    int status = 0;
    for (int c = 0; c < n; c++) {
        int pr = c, pc = c;
        double best = -1;
        for (int i = c; i < n; i++)
            for (int j = c; j < n; j++) {
                double a = std::abs(A[(long)i * n + j]);
                if (a > best) { best = a; pr = i; pc = j; }
            }
        if (best == 0.0) { status = 1; break; }
        if (pr != c) {
            for (int j = 0; j < n; j++) std::swap(A[(long)c * n + j], A[(long)pr * n + j]);
            for (int j = 0; j < nrhs; j++) std::swap(B[(long)c * nrhs + j], B[(long)pr * nrhs + j]);
        }
        if (pc != c) {
            for (int i = 0; i < n; i++) std::swap(A[(long)i * n + c], A[(long)i * n + pc]);
            std::swap(colp[c], colp[pc]);
        }
        cplx piv = A[(long)c * n + c];
        for (int i = c + 1; i < n; i++) {
            cplx f = A[(long)i * n + c] / piv;
            if (f == cplx(0)) continue;
            for (int j = c; j < n; j++) A[(long)i * n + j] -= f * A[(long)c * n + j];
            for (int j = 0; j < nrhs; j++) B[(long)i * nrhs + j] -= f * B[(long)c * nrhs + j];
        }
    }
    std::vector<cplx> Y((long)n * nrhs, 0.0);
    if (status == 0) {
        for (int i = n - 1; i >= 0; i--)
            for (int j = 0; j < nrhs; j++) {
                cplx acc = B[(long)i * nrhs + j];
                for (int l = i + 1; l < n; l++) acc -= A[(long)i * n + l] * Y[(long)l * nrhs + j];
                Y[(long)i * nrhs + j] = acc / A[(long)i * n + i];
            }
    }
    for (int i = 0; i < n; i++)
        for (int j = 0; j < nrhs; j++) X[(long)colp[i] * nrhs + j] = Y[(long)i * nrhs + j];
    return status;
}

namespace {

template <int S1> void El<S1>::inverse(cplx *z, const cplx *z1) const {
    if (S1 == 1) { *z = 1.0 / (*z1); return; }
    std::vector<cplx> id(es, 0.0);
    for (int i = 0; i < s; i++) id[i * s + i] = 1.0;
    orc_cplx_solve(s, s, z1, id.data(), z);
}

// element_linsolve_right (cntr_elements.hpp:443-480): block system sum_m M(l,m) X(m) = Q(l)
// with n x n blocks of s x s.
template <int S1> void El<S1>::linsolve_right(int n, cplx *X, const cplx *M, const cplx *Q) const {
    if (S1 == 1 && n == 1) { *X = *Q / (*M); return; }
    int L = n * s;
    std::vector<cplx> A((long)L * L), B((long)L * s), Y((long)L * s);
    for (int l = 0; l < n; l++)
        for (int m = 0; m < n; m++)
            for (int p = 0; p < s; p++)
                for (int q = 0; q < s; q++)
                    A[(long)(l * s + p) * L + m * s + q] = M[(long)(l * n + m) * es + p * s + q];
    for (int l = 0; l < n; l++)
        for (int p = 0; p < s; p++)
            for (int q = 0; q < s; q++) B[(long)(l * s + p) * s + q] = Q[(long)l * es + p * s + q];
    orc_cplx_solve(L, s, A.data(), B.data(), Y.data());
    for (int l = 0; l < n; l++)
        for (int p = 0; p < s; p++)
            for (int q = 0; q < s; q++) X[(long)l * es + p * s + q] = Y[(long)(l * s + p) * s + q];
}

// element_linsolve_left (cntr_elements.hpp:482-497): X M = Q via the adjoint system.
template <int S1> void El<S1>::linsolve_left(int n, cplx *X, const cplx *M, const cplx *Q) const {
    if (S1 == 1 && n == 1) { *X = *Q / (*M); return; }
    std::vector<cplx> Mc((long)n * n * es), Qc((long)n * es);
    for (int l = 0; l < n * n; l++) conj(Mc.data() + (long)l * es, M + (long)l * es);
    for (int l = 0; l < n; l++) conj(Qc.data() + (long)l * es, Q + (long)l * es);
    // the reference conjugates block-wise without transposing the block matrix
    linsolve_right(n, X, Mc.data(), Qc.data());
    for (int l = 0; l < n; l++) conj_inplace(X + (long)l * es);
}

// ------------------------------------------------------------------------------------
// Matsubara integrals (cntr_convolution_impl.hpp:86-224, 410-540)
// ------------------------------------------------------------------------------------
template <int S1>
void matsubara_integral_1(const El<S1> &E, int m, int ntau, cplx *C, const cplx *A, const cplx *B,
                          const Integ &In, int sig) {
    int k = In.k, k1 = k + 1, k2 = 2 * k1, es = E.es;
    std::vector<cplx> c1(es, 0.0), c2(es, 0.0);
    if (m >= k2 - 1) {
        const cplx *a = A + (long)m * es, *b = B;
        for (int j = 0; j <= k; j++, a -= es, b += es) E.incr(c1.data(), In.gregory_omega(j), a, b);
        for (int j = k1; j < m - k; j++, a -= es, b += es) E.incr(c1.data(), a, b);
        for (int j = m - k; j <= m; j++, a -= es, b += es) E.incr(c1.data(), In.gregory_omega(m - j), a, b);
    } else if (m >= k) {
        const cplx *a = A + (long)m * es, *b = B;
        for (int j = 0; j <= m; j++, a -= es, b += es) E.incr(c1.data(), In.gregory_weights(m, j), a, b);
    } else if (m > 0) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                E.incr(c1.data(), In.rcorr(m, l, j), A + (long)l * es, B + (long)j * es);
    }
    if (ntau - m >= k2 - 1) {
        const cplx *a = A + (long)ntau * es, *b = B + (long)m * es;
        for (int j = m; j <= m + k; j++, a -= es, b += es) E.incr(c2.data(), In.gregory_omega(j - m), a, b);
        for (int j = m + k1; j < ntau - k; j++, a -= es, b += es) E.incr(c2.data(), a, b);
        for (int j = ntau - k; j <= ntau; j++, a -= es, b += es) E.incr(c2.data(), In.gregory_omega(ntau - j), a, b);
    } else if (ntau - m >= k) {
        const cplx *a = A + (long)ntau * es, *b = B + (long)m * es;
        for (int j = m; j <= ntau; j++, a -= es, b += es)
            E.incr(c2.data(), In.gregory_weights(ntau - m, ntau - j), a, b);
    } else if (ntau - m > 0) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                E.incr(c2.data(), In.rcorr(ntau - m, l, j), A + (long)(ntau - l) * es,
                       B + (long)(ntau - j) * es);
    }
    for (int l = 0; l < es; l++) C[l] = c1[l] + cplx(sig, 0.0) * c2[l];
}

template <int S1>
void matsubara_integral_2(const El<S1> &E, int m, int ntau, cplx *C, const cplx *A, const cplx *B,
                          const Integ &In, int sig) {
    int k = In.k, k1 = k + 1, k2 = 2 * k1, es = E.es;
    std::vector<cplx> c1(es, 0.0), c2(es, 0.0);
    if (m == 0) {
    } else if (m < k) {
        for (int j = 0; j <= k; j++)
            for (int l = 0; l <= k; l++)
                E.incr(c1.data(), In.rcorr(m, l, j), A + (long)j * es, B + (long)(ntau - l) * es);
    } else if (m < k2 - 1) {
        const cplx *a = A + (long)m * es, *b = B + (long)ntau * es;
        for (int l = 0; l <= m; l++, a -= es, b -= es) E.incr(c1.data(), In.gregory_weights(m, l), a, b);
    } else {
        const cplx *a = A + (long)m * es, *b = B + (long)ntau * es;
        for (int l = 0; l <= k; l++, a -= es, b -= es) E.incr(c1.data(), In.gregory_omega(l), a, b);
        for (int l = k1; l < m - k; l++, a -= es, b -= es) E.incr(c1.data(), a, b);
        for (int l = m - k; l <= m; l++, a -= es, b -= es) E.incr(c1.data(), In.gregory_omega(m - l), a, b);
    }
    if (m == ntau) {
    } else if (m > ntau - k) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                E.incr(c2.data(), In.rcorr(ntau - m, l, j), A + (long)(ntau - l) * es, B + (long)j * es);
    } else if (m > ntau - k2 + 1) {
        const cplx *a = A + (long)m * es, *b = B;
        for (int l = 0; l <= ntau - m; l++, a += es, b += es)
            E.incr(c2.data(), In.gregory_weights(ntau - m, l), a, b);
    } else {
        const cplx *a = A + (long)m * es, *b = B;
        for (int l = m; l <= m + k; l++, a += es, b += es) E.incr(c2.data(), In.gregory_omega(l - m), a, b);
        for (int l = m + k1; l < ntau - k; l++, a += es, b += es) E.incr(c2.data(), a, b);
        for (int l = ntau - k; l <= ntau; l++, a += es, b += es) E.incr(c2.data(), In.gregory_omega(ntau - l), a, b);
    }
    for (int l = 0; l < es; l++) C[l] = c2[l] + cplx(sig, 0.0) * c1[l];
}

// convolution_matsubara_dispatch (cntr_convolution_impl.hpp:560-582)
template <int S1> void convolution_matsubara_t(HM &C, HM &A, HM &B, const Integ &In, double beta) {
    El<S1> E(C.s);
    int ntau = A.ntau();
    for (int m = 0; m <= ntau; m++)
        matsubara_integral_1<S1>(E, m, ntau, C.matptr(m), A.matptr(0), B.matptr(0), In, A.sig());
    double dtau = beta / ntau;
    long n = (long)(ntau + 1) * C.es;
    for (long l = 0; l < n; l++) C.matptr(0)[l] *= dtau;
}

// ------------------------------------------------------------------------------------
// convolution_timestep (cntr_convolution_impl.hpp:741-1580)
// ------------------------------------------------------------------------------------
template <int S1>
void conv_ret(int n, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, const Integ &In, double h) {
    El<S1> E(C.s);
    int k = In.k, es = C.es;
    std::vector<cplx> res((long)(n + 1) * es, 0.0), at(es), bt(es);
    if (n >= k) {
        for (int m = 0; m <= n; m++) {
            const cplx *ar = A.retptr(n, m);
            for (int l = 0; l < es; l++) at[l] = ar[l] * h;
            const cplx *br = B.retptr(m, 0);
            cplx *cr = res.data();
            if (m < n - k) {
                for (int j = 0; j < m - k; j++, br += es, cr += es) E.incr(cr, at.data(), br);
            } else {
                double w = In.gregory_omega(n - m);
                for (int j = 0; j < m - k; j++, br += es, cr += es) E.incr(cr, w, at.data(), br);
            }
            int j1 = m - k < 0 ? 0 : m - k;
            for (int j = j1; j <= m; j++, br += es, cr += es)
                E.incr(cr, In.gregory_weights(n - j, n - m), at.data(), br);
        }
        for (int m = n - k; m < n; m++) {
            const cplx *ar = A.retptr(n, m);
            for (int l = 0; l < es; l++) at[l] = ar[l] * h;
            for (int j = m + 1; j <= n; j++) {
                double w = In.gregory_weights(n - j, n - m);
                E.conj(bt.data(), Bcc.retptr(j, m));
                E.incr(res.data() + (long)j * es, -w, at.data(), bt.data());
            }
        }
    } else {
        for (int j = 0; j <= n; j++) {
            cplx *cr = res.data() + (long)j * es;
            for (int m = 0; m <= k; m++) {
                double w = In.poly_integration(j, n, m) * h;
                if (m >= j) E.set(bt.data(), B.retptr(m, j));
                else { E.conj(bt.data(), Bcc.retptr(j, m)); w = -w; }
                if (n >= m) E.set(at.data(), A.retptr(n, m));
                else { E.conj(at.data(), Acc.retptr(m, n)); w = -w; }
                E.incr(cr, w, at.data(), bt.data());
            }
        }
    }
    std::memcpy(C.retptr(n, 0), res.data(), sizeof(cplx) * (n + 1) * es);
}

template <int S1>
void conv_tv(int n, cplx *ctv, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, const Integ &In,
             double beta, double h) {
    El<S1> E(C.s);
    int k = In.k, es = C.es, ntau = A.ntau(), n1 = n > k ? n : k;
    double dtau = beta / ntau;
    std::vector<cplx> ct(es), at(es);
    for (int m = 0; m <= ntau; m++) {
        matsubara_integral_2<S1>(E, m, ntau, ct.data(), A.tvptr(n, 0), B.matptr(0), In, B.sig());
        for (int l = 0; l < es; l++) ctv[(long)m * es + l] = dtau * ct[l];
    }
    for (int j = 0; j <= n1; j++) {
        double w = In.gregory_weights(n, j);
        if (n < j) { E.conj(at.data(), Acc.retptr(j, n)); E.smul(at.data(), -1.0); }
        else E.set(at.data(), A.retptr(n, j));
        E.smul(at.data(), h);
        const cplx *btv = B.tvptr(j, 0);
        cplx *c1 = ctv;
        if (w != 1.0) {
            for (int m = 0; m <= ntau; m++, btv += es, c1 += es) E.incr(c1, w, at.data(), btv);
        } else {
            for (int m = 0; m <= ntau; m++, btv += es, c1 += es) E.incr(c1, at.data(), btv);
        }
    }
}

template <int S1>
void conv_tv_into(int n, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, const Integ &In, double beta,
                  double h) {
    std::vector<cplx> ctv((long)(C.ntau() + 1) * C.es);
    conv_tv<S1>(n, ctv.data(), C, A, Acc, B, Bcc, In, beta, h);
    std::memcpy(C.tvptr(n, 0), ctv.data(), sizeof(cplx) * ctv.size());
}

template <int S1>
void conv_les_tvvt(int n, int j1, int j2, cplx *cles, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc,
                   const Integ &In, double beta, double h) {
    El<S1> E(C.s);
    int k = In.k, k1 = k + 1, k2 = 2 * k1, es = C.es, ntau = A.ntau(), sig = A.sig();
    double dtau = beta / ntau;
    std::vector<cplx> bt((long)(ntau + 1) * es);
    cplx idt(0, -dtau);
    for (int m = 0; m <= ntau; m++) E.conj(bt.data() + (long)m * es, Bcc.tvptr(n, ntau - m));
    for (auto &x : bt) x *= idt * (-(double)sig);
    for (int j = j1; j <= j2; j++) {
        const cplx *btv = bt.data(), *atv = A.tvptr(j, 0);
        cplx *c1 = cles + (long)j * es;
        if (ntau < k2 - 1) {
            for (int m = 0; m <= ntau; m++, atv += es, btv += es) E.incr(c1, In.gregory_weights(ntau, m), atv, btv);
        } else {
            int m = 0;
            for (; m <= k; m++, atv += es, btv += es) E.incr(c1, In.gregory_omega(m), atv, btv);
            for (m = k1; m < ntau - k; m++, atv += es, btv += es) E.incr(c1, atv, btv);
            for (m = ntau - k; m <= ntau; m++, atv += es, btv += es) E.incr(c1, In.gregory_omega(ntau - m), atv, btv);
        }
    }
}

template <int S1>
void conv_les_lesadv(int n, int j1, int j2, cplx *cles, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc,
                     const Integ &In, double beta, double h) {
    El<S1> E(C.s);
    int k = In.k, es = C.es, n1 = n < k ? k : n;
    std::vector<cplx> ales(es), badv((long)(n1 + 1) * es);
    for (int m = 0; m <= n1; m++) {
        double w = h * In.gregory_weights(n, m);
        if (m <= n) {
            E.conj(badv.data() + (long)m * es, Bcc.retptr(n, m));
            for (int l = 0; l < es; l++) badv[(long)m * es + l] *= w;
        } else {
            for (int l = 0; l < es; l++) badv[(long)m * es + l] = -w * B.retptr(m, n)[l];
        }
    }
    for (int j = j1; j <= j2; j++)
        for (int m = 0; m < j; m++) {
            E.minusconj(ales.data(), Acc.lesptr(m, j));
            E.incr(cles + (long)j * es, ales.data(), badv.data() + (long)m * es);
        }
    for (int m = 0; m <= n1; m++) {
        int jmax = j2 < m ? j2 : m;
        for (int j = j1; j <= jmax; j++) E.incr(cles + (long)j * es, A.lesptr(j, m), badv.data() + (long)m * es);
    }
}

template <int S1>
void conv_les_retles(int n, cplx *cles, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, const Integ &In,
                     double beta, double h) {
    El<S1> E(C.s);
    int k = In.k, k1 = k + 1, k2 = 2 * k1, es = C.es, n1 = n < k ? k : n;
    std::vector<cplx> bt((long)(n1 + 1) * es), at(es);
    for (int m = 0; m <= n1; m++) {
        if (m <= n) {
            for (int l = 0; l < es; l++) bt[(long)m * es + l] = h * B.lesptr(m, n)[l];
        } else {
            E.conj(bt.data() + (long)m * es, Bcc.lesptr(n, m));
            for (int l = 0; l < es; l++) bt[(long)m * es + l] *= -h;
        }
    }
    for (int j = 0; j <= n; j++) {
        cplx *c1 = cles + (long)j * es;
        const cplx *ar = A.retptr(j, 0), *bl = bt.data();
        if (j >= k2 - 1) {
            int m = 0;
            for (; m <= k; m++, ar += es, bl += es) E.incr(c1, In.gregory_omega(m), ar, bl);
            for (m = k1; m < j - k; m++, ar += es, bl += es) E.incr(c1, ar, bl);
            for (m = j - k; m <= j; m++, ar += es, bl += es) E.incr(c1, In.gregory_omega(j - m), ar, bl);
        } else {
            for (int m = 0; m <= j; m++, ar += es, bl += es) E.incr(c1, In.gregory_weights(j, m), ar, bl);
        }
        if (j < k) {
            for (int m = j + 1; m <= k; m++) {
                E.conj(at.data(), Acc.retptr(m, j));
                E.incr(c1, -In.gregory_weights(j, m), at.data(), bt.data() + (long)m * es);
            }
        }
    }
}

template <int S1>
void conv_les(int n, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, const Integ &In, double beta, double h) {
    int k = In.k, es = C.es, n1 = k > n ? k : n;
    std::vector<cplx> cles((long)(n1 + 1) * es, 0.0);
    conv_les_tvvt<S1>(n, 0, n1, cles.data(), C, A, Acc, B, Bcc, In, beta, h);
    conv_les_lesadv<S1>(n, 0, n1, cles.data(), C, A, Acc, B, Bcc, In, beta, h);
    conv_les_retles<S1>(n, cles.data(), C, A, Acc, B, Bcc, In, beta, h);
    for (int m = 0; m <= n; m++) std::memcpy(C.lesptr(m, n), cles.data() + (long)m * es, sizeof(cplx) * es);
}

// ------------------------------------------------------------------------------------
// Matsubara Fourier helpers (cntr_matsubara_impl.hpp, fourier.cpp)
// ------------------------------------------------------------------------------------
double get_omega(int m, double beta, int sig) {
    int one = (1 - sig) >> 1;
    return kPi / beta * (2 * m + one);
}

// Endpoint-corrected DFT weights, cubic order (Numerical Recipes 2nd ed. section 13.9,
// routine dftcor; fourier.cpp:43-99 uses the same published formulas).
void dftcorr_cubic(double th, double *corfac, cplx *endcor) {
    double ar[4], ai[4];
    if (std::fabs(th) < 5.0e-2) {
        double t = th, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
        *corfac = 1.0 - (11.0 / 720.0) * t4 + (23.0 / 15120.0) * t6;
        ar[0] = (-2.0 / 3.0) + t2 / 45.0 + (103.0 / 15120.0) * t4 - (169.0 / 226800.0) * t6;
        ar[1] = (7.0 / 24.0) - (7.0 / 180.0) * t2 + (5.0 / 3456.0) * t4 - (7.0 / 259200.0) * t6;
        ar[2] = (-1.0 / 6.0) + t2 / 45.0 - (5.0 / 6048.0) * t4 + t6 / 64800.0;
        ar[3] = (1.0 / 24.0) - t2 / 180.0 + (5.0 / 24192.0) * t4 - t6 / 259200.0;
        ai[0] = t * (2.0 / 45.0 + (2.0 / 105.0) * t2 - (8.0 / 2835.0) * t4 + (86.0 / 467775.0) * t6);
        ai[1] = t * (7.0 / 72.0 - t2 / 168.0 + (11.0 / 72576.0) * t4 - (13.0 / 5987520.0) * t6);
        ai[2] = t * (-7.0 / 90.0 + t2 / 210.0 - (11.0 / 90720.0) * t4 + (13.0 / 7484400.0) * t6);
        ai[3] = t * (7.0 / 360.0 - t2 / 840.0 + (11.0 / 362880.0) * t4 - (13.0 / 29937600.0) * t6);
    } else {
        double c = std::cos(th), s = std::sin(th), c2 = c * c - s * s, s2 = 2.0 * s * c;
        double t2 = th * th, t4 = t2 * t2, tm = 3.0 - t2, sp = 6.0 + t2;
        double sth4i = 1.0 / (6.0 * t4), tth4i = 2.0 * sth4i;
        *corfac = tth4i * sp * (3.0 - 4.0 * c + c2);
        ar[0] = sth4i * (-42.0 + 5.0 * t2 + sp * (8.0 * c - c2));
        ai[0] = sth4i * (th * (-12.0 + 6.0 * t2) + sp * s2);
        ar[1] = sth4i * (14.0 * tm - 7.0 * sp * c);
        ai[1] = sth4i * (30.0 * th - 5.0 * sp * s);
        ar[2] = tth4i * (-4.0 * tm + 2.0 * sp * c);
        ai[2] = tth4i * (-12.0 * th + 2.0 * sp * s);
        ar[3] = sth4i * (2.0 * tm - sp * c);
        ai[3] = sth4i * (6.0 * th - sp * s);
    }
    for (int j = 0; j < 4; j++) endcor[j] = cplx(ar[j], ai[j]);
}

void dftcorr_linear(double th, double *corfac, cplx *endcor) {
    double ar, ai;
    if (std::fabs(th) < 5.0e-2) {
        double t2 = th * th, t4 = t2 * t2, t6 = t4 * t2;
        *corfac = 1.0 - (1.0 / 12.0) * t2 + (1.0 / 360.0) * t4 - (1.0 / 20160.0) * t6;
        ar = -0.5 + t2 / 24.0 - (1.0 / 720.0) * t4 + (1.0 / 40320.0) * t6;
        ai = th * (1.0 / 6.0 - (1.0 / 120.0) * t2 + (1.0 / 5040.0) * t4 - (1.0 / 362880.0) * t6);
    } else {
        double c = std::cos(th), s = std::sin(th), t2 = th * th;
        *corfac = 2.0 * (1.0 - c) / t2;
        ar = (c - 1.0) / t2;
        ai = (th - s) / t2;
    }
    endcor[0] = cplx(ar, ai);
    endcor[1] = 0;
}

// cntr_matsubara_impl.hpp:71-88
template <int S1>
void set_first_order_tail(const El<S1> &E, cplx *xmat, const cplx *coeff, double beta, int ntau, int sig) {
    int es = E.es;
    for (int r = 0; r <= ntau; r++) {
        E.set(xmat + (long)r * es, coeff);
        E.smul(xmat + (long)r * es, -0.5);
        if (sig == 1) {
            double tau = r * (beta / ntau);
            for (int l = 0; l < es; l++) xmat[(long)r * es + l] += coeff[l] * (tau / beta);
        }
    }
}

// cntr_matsubara_impl.hpp:134-160
template <int S1> void matsubara_dft(const El<S1> &E, cplx *mdft, HM &G, int sig) {
    int ntau = G.ntau(), es = E.es;
    double one = sig == -1 ? 1.0 : 0.0;
    std::vector<cplx> z(es), z1(es);
    for (int m = 0; m <= ntau; m++) {
        E.zero(z.data());
        for (int r = 0; r <= ntau; r++) {
            double arg = ((2 * m + one) * r * kPi) / ntau;
            cplx ef(std::cos(arg), std::sin(arg));
            E.set(z1.data(), G.matptr(r));
            E.smul(z1.data(), ef);
            E.incr(z.data(), z1.data());
        }
        E.set(mdft + (long)m * es, z.data());
    }
}

// cntr_matsubara_impl.hpp:191-248
template <int S1>
void matsubara_ft(const El<S1> &E, cplx *result, int m, HM &G, const cplx *mdft, int sig, double beta,
                  int order) {
    int ntau = G.ntau(), es = E.es;
    double one = sig == -1 ? 1.0 : 0.0, dtau = beta / ntau, corfac;
    cplx bcorr[4];
    double arg = (2 * m + one) * kPi / ntau;
    if (order == 0) { corfac = 1.0; bcorr[0] = 0.0; }
    else if (order == 1) dftcorr_linear(arg, &corfac, bcorr);
    else dftcorr_cubic(arg, &corfac, bcorr);
    int m1 = m;
    while (m1 < 0) m1 += ntau;
    while (m1 >= ntau) m1 -= ntau;
    std::vector<cplx> z1(es, 0.0), z2(es), dft(es);
    for (int l = 0; l < es; l++) dft[l] = mdft[(long)m1 * es + l] * corfac;
    for (int r = 0; r <= order; r++) {
        E.set(z2.data(), G.matptr(r));
        E.smul(z2.data(), bcorr[r]);
        E.incr(z1.data(), z2.data());
        E.set(z2.data(), G.matptr(ntau - r));
        E.smul(z2.data(), (1.0 * sig) * cplx(bcorr[r].real(), -bcorr[r].imag()));
        E.incr(z1.data(), z2.data());
    }
    for (int l = 0; l < es; l++) result[l] = dtau * (z1[l] + dft[l]);
}

// ------------------------------------------------------------------------------------
// Equilibrium inputs (cntr_equilibrium_impl.hpp:30-160, 873-955)
// ------------------------------------------------------------------------------------
const double kExpMax = 100;
double fermi(double beta, double w) {
    double arg = w * beta;
    if (std::fabs(arg) > kExpMax) return arg > 0.0 ? 0.0 : 1.0;
    return 1.0 / (1.0 + std::exp(arg));
}
double fermi_exp(double beta, double tau, double w) {
    if (w < 0) return std::exp(w * tau) * fermi(beta, w);
    return std::exp((tau - beta) * w) * fermi(beta, -w);
}
double bose(double beta, double w) {
    double arg = w * beta;
    if (arg < 0) return -1.0 - bose(beta, -w);
    if (std::fabs(arg) > kExpMax) return 0.0;
    if (arg < 1e-10) return 1.0 / arg;
    return 1.0 / (std::exp(arg) - 1.0);
}
double bose_exp(double beta, double tau, double w) {
    if (w < 0) return std::exp(tau * w) * bose(beta, w);
    return -std::exp((tau - beta) * w) * bose(beta, -w);
}

// Hermitian eigen-decomposition by cyclic complex Jacobi rotations: A = V diag(ev) V^dagger.
void herm_eig(int n, const cplx *A0, double *ev, cplx *V) {
    std::vector<cplx> A(A0, A0 + n * n);
    for (int i = 0; i < n * n; i++) V[i] = 0;
    for (int i = 0; i < n; i++) V[i * n + i] = 1;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) off += std::norm(A[p * n + q]);
        if (off < 1e-30) break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++) {
                cplx apq = A[p * n + q];
                double mag = std::abs(apq);
                if (mag < 1e-300) continue;
                double app = A[p * n + p].real(), aqq = A[q * n + q].real();
                cplx ph = apq / mag;  // e^{i phi}
                double theta = 0.5 * std::atan2(2.0 * mag, aqq - app);
                double c = std::cos(theta), s = std::sin(theta);
                // rotation R with columns p,q: R_pp = c, R_qq = c, R_pq = s*ph, R_qp = -s*conj(ph)
                cplx rpp = c, rqq = c, rpq = s * ph, rqp = -s * std::conj(ph);
                // A <- R^dagger A R
                for (int i = 0; i < n; i++) {  // A R
                    cplx aip = A[i * n + p], aiq = A[i * n + q];
                    A[i * n + p] = aip * rpp + aiq * rqp;
                    A[i * n + q] = aip * rpq + aiq * rqq;
                }
                for (int j = 0; j < n; j++) {  // R^dagger (A R)
                    cplx apj = A[p * n + j], aqj = A[q * n + j];
                    A[p * n + j] = std::conj(rpp) * apj + std::conj(rqp) * aqj;
                    A[q * n + j] = std::conj(rpq) * apj + std::conj(rqq) * aqj;
                }
                for (int i = 0; i < n; i++) {
                    cplx vip = V[i * n + p], viq = V[i * n + q];
                    V[i * n + p] = vip * rpp + viq * rqp;
                    V[i * n + q] = vip * rpq + viq * rqq;
                }
            }
    }
    for (int i = 0; i < n; i++) ev[i] = A[i * n + i].real();
}

// out = V diag(d) V^dagger
void vdv(int n, const cplx *V, const cplx *d, cplx *out) {
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
            cplx acc = 0;
            for (int l = 0; l < n; l++) acc += V[i * n + l] * d[l] * std::conj(V[j * n + l]);
            out[i * n + j] = acc;
        }
}
void matmul(int n, const cplx *a, const cplx *b, cplx *c) {
    std::vector<cplx> t(n * n, 0.0);
    for (int i = 0; i < n; i++)
        for (int l = 0; l < n; l++)
            for (int j = 0; j < n; j++) t[i * n + j] += a[i * n + l] * b[l * n + j];
    std::memcpy(c, t.data(), sizeof(cplx) * n * n);
}
void adjoint(int n, const cplx *a, cplx *b) {
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) b[i * n + j] = std::conj(a[j * n + i]);
}

}  // namespace

// green_from_H_const_dispatch (cntr_equilibrium_impl.hpp:873-955)
extern "C" void orc_green_from_H_const(orc_hm *Gh, double mu, const cplx *H0, double beta, double h) {
    HM G(Gh);
    int s = G.s, es = G.es, nt = G.nt(), ntau = G.ntau(), sign = G.sig();
    double dtau = beta / ntau;
    std::vector<cplx> Hmu(es), V(es), d(s), val(es);
    std::vector<double> ev(s);
    for (int i = 0; i < es; i++) Hmu[i] = -H0[i];
    for (int i = 0; i < s; i++) Hmu[i * s + i] += mu;
    herm_eig(s, Hmu.data(), ev.data(), V.data());
    for (int m = 0; m <= ntau; m++) {
        double tau = m * dtau;
        for (int i = 0; i < s; i++)
            d[i] = sign == -1 ? -fermi_exp(beta, tau, ev[i]) : bose_exp(beta, tau, ev[i]);
        vdv(s, V.data(), d.data(), G.matptr(m));
    }
    if (nt < 0) return;
    // Udt = exp(i h Hmu); U(n) = U(n-1) Udt
    std::vector<cplx> Udt(es), U((long)(nt + 1) * es);
    for (int i = 0; i < s; i++) d[i] = std::exp(kI * h * ev[i]);
    vdv(s, V.data(), d.data(), Udt.data());
    for (int i = 0; i < es; i++) U[i] = 0;
    for (int i = 0; i < s; i++) U[i * s + i] = 1;
    for (int n = 1; n <= nt; n++) matmul(s, U.data() + (long)(n - 1) * es, Udt.data(), U.data() + (long)n * es);
    std::vector<cplx> f(es), tmp(es), tmp2(es);
    for (int m = 0; m <= ntau; m++) {
        double tau = m * dtau;
        for (int i = 0; i < s; i++)
            d[i] = sign == -1 ? fermi_exp(beta, tau, -ev[i]) : bose_exp(beta, tau, -ev[i]);
        vdv(s, V.data(), d.data(), f.data());
        for (int n = 0; n <= nt; n++) {
            matmul(s, U.data() + (long)n * es, f.data(), tmp.data());
            cplx pref = sign == -1 ? kI : -kI;
            for (int i = 0; i < es; i++) G.tvptr(n, m)[i] = pref * tmp[i];
        }
    }
    for (int i = 0; i < s; i++) d[i] = sign == -1 ? fermi(beta, -ev[i]) : -bose(beta, -ev[i]);
    vdv(s, V.data(), d.data(), val.data());
    std::vector<cplx> adj(es);
    for (int m = 0; m <= nt; m++)
        for (int n = 0; n <= m; n++) {
            adjoint(s, U.data() + (long)n * es, adj.data());
            matmul(s, U.data() + (long)m * es, adj.data(), tmp.data());
            for (int i = 0; i < es; i++) G.retptr(m, n)[i] = -kI * tmp[i];
            adjoint(s, U.data() + (long)m * es, adj.data());
            matmul(s, val.data(), adj.data(), tmp2.data());
            matmul(s, U.data() + (long)n * es, tmp2.data(), tmp.data());
            for (int i = 0; i < es; i++) G.lesptr(n, m)[i] = kI * tmp[i];
        }
}

namespace {

// ------------------------------------------------------------------------------------
// VIE2 Matsubara (cntr_vie2_impl.hpp:305-484)
// ------------------------------------------------------------------------------------
template <int S1>
void vie2_mat_fourier_t(HM &G, HM &F, HM &Fcc, HM &Q, double beta, int pcf, int order) {
    El<S1> E(G.s);
    int es = E.es, ntau = G.ntau(), sig = G.sig();
    double dtau = beta / ntau;
    int matsub_one = sig == -1 ? 1 : 0;
    int m2 = ntau / 2;
    std::vector<cplx> xmat((long)(ntau + 1) * es), fmdft((long)(ntau + 1) * es), qmdft((long)(ntau + 1) * es);
    std::vector<cplx> qmasy(es), z1(es), z2(es), z3(es), zinv(es), fiomn(es), qiomn(es), qiomn1(es), one(es);
    E.set_diag(one.data(), 1.0);
    E.set(qmasy.data(), Q.matptr(0));
    E.smul(qmasy.data(), -1.0);
    E.set(z1.data(), Q.matptr(ntau));
    E.smul(z1.data(), (double)sig);
    E.incr(qmasy.data(), z1.data());
    set_first_order_tail<S1>(E, xmat.data(), qmasy.data(), beta, ntau, sig);
    matsubara_dft<S1>(E, fmdft.data(), F, sig);
    matsubara_dft<S1>(E, qmdft.data(), Q, sig);
    for (int p = -pcf; p <= pcf; p++) {
        int m_low = 0, m_high = 0;
        if (sig == 1) { m_high = p < 0 ? 0 : 1; m_low = p > 0 ? -1 : 0; }
        for (int m = -m2 - m_low; m <= m2 - 1 + m_high; m++) {
            double omn = (2 * (m + p * ntau) + matsub_one) * kPi / (ntau * dtau);
            matsubara_ft<S1>(E, fiomn.data(), m + p * ntau, F, fmdft.data(), sig, beta, order);
            matsubara_ft<S1>(E, qiomn.data(), m + p * ntau, Q, qmdft.data(), sig, beta, order);
            E.set(z3.data(), qmasy.data());
            if (sig == 1 && m + p * ntau == 0) E.smul(z3.data(), cplx(0.0, 0.0));
            else E.smul(z3.data(), cplx(0.0, -1.0 / omn));
            for (int l = 0; l < es; l++) qiomn1[l] = qiomn[l] - z3[l];
            for (int l = 0; l < es; l++) z1[l] = fiomn[l] + one[l];
            E.mult(z2.data(), fiomn.data(), z3.data());
            for (int l = 0; l < es; l++) z2[l] = qiomn1[l] - z2[l];
            E.inverse(zinv.data(), z1.data());
            E.mult(z1.data(), zinv.data(), z2.data());
            E.smul(z1.data(), 1.0 / beta);
            for (int r = 0; r <= ntau; r++) {
                double arg = omn * r * dtau;
                cplx ef(std::cos(arg), -std::sin(arg));
                for (int l = 0; l < es; l++) xmat[(long)r * es + l] += z1[l] * ef;
            }
        }
    }
    std::memcpy(G.matptr(0), xmat.data(), sizeof(cplx) * xmat.size());
}

// vie2_mat_steep_dispatch (cntr_vie2_impl.hpp:486-600): a Fourier solve with pcf = 3 as the start,
// then conjugate-gradient iterations on A X = X + (F*X + X*Fcc)/2 with the inner product
// <X, Y> = sum_r w_r sum_ab Re (X(r)^dagger Y(r))_ab, w_r = Gregory omega at both ends of the tau
// grid; stops after maxiter iterations or when sqrt(<R, R>) < tol; no iteration when <R, R> <= tol.
template <int S1>
void vie2_mat_steep_t(HM &G, HM &F, HM &Fcc, HM &Q, double beta, const Integ &In, int maxiter, double tol) {
    vie2_mat_fourier_t<S1>(G, F, Fcc, Q, beta, 3, 3);
    if (maxiter <= 0) return;
    const int ntau = G.ntau(), es = G.es, k = In.k;
    El<S1> E(G.s);
    auto buf = [&](std::vector<cplx> &v, orc_hm &h) {
        v.assign((long)(ntau + 1) * es, 0.0);
        h = {-1, ntau, G.s, G.sig(), nullptr, nullptr, nullptr, v.data()};
    };
    std::vector<cplx> vr, vap, vp, vc1, vc2;
    orc_hm hr, hap, hp, hc1, hc2;
    buf(vr, hr); buf(vap, hap); buf(vp, hp); buf(vc1, hc1); buf(vc2, hc2);
    HM R(&hr), AP(&hap), P(&hp), C1(&hc1), C2(&hc2);
    std::vector<cplx> tmp(es), xcc(es);
    auto dot = [&](HM &X, HM &Y) {
        double acc = 0.0;
        for (int r = 0; r <= ntau; r++) {
            const double w = r <= k ? In.gregory_omega(r) : (r >= ntau - k ? In.gregory_omega(ntau - r) : 1.0);
            E.conj(xcc.data(), X.matptr(r));
            E.mult(tmp.data(), xcc.data(), Y.matptr(r));
            for (int l = 0; l < es; l++) acc += w * tmp[l].real();
        }
        return acc;
    };
    // R = Q - (G + (F*G + G*Fcc)/2), P = R
    convolution_matsubara_t<S1>(C1, F, G, In, beta);
    convolution_matsubara_t<S1>(C2, G, Fcc, In, beta);
    for (int r = 0; r <= ntau; r++) {
        cplx *x = R.matptr(r);
        E.set(x, C1.matptr(r));
        E.incr(x, C2.matptr(r));
        E.smul(x, 0.5);
        E.incr(x, G.matptr(r));
        E.incr(x, -1.0, Q.matptr(r));
        E.smul(x, -1.0);
        E.set(P.matptr(r), x);
    }
    double rsold = dot(R, R);
    if (rsold <= tol) return;
    for (int iter = 0; iter < maxiter; iter++) {
        convolution_matsubara_t<S1>(C1, F, P, In, beta);
        convolution_matsubara_t<S1>(C2, P, Fcc, In, beta);
        for (int r = 0; r <= ntau; r++) {
            cplx *x = AP.matptr(r);
            E.set(x, C1.matptr(r));
            E.incr(x, C2.matptr(r));
            E.smul(x, 0.5);
            E.incr(x, P.matptr(r));
        }
        const double alpha = rsold / dot(P, AP);
        for (int r = 0; r <= ntau; r++) {
            E.incr(G.matptr(r), alpha, P.matptr(r));
            E.incr(R.matptr(r), -alpha, AP.matptr(r));
        }
        const double rsnew = dot(R, R);
        for (int r = 0; r <= ntau; r++) {
            E.set(tmp.data(), R.matptr(r));
            E.incr(tmp.data(), rsnew / rsold, P.matptr(r));
            E.set(P.matptr(r), tmp.data());
        }
        rsold = rsnew;
        if (std::sqrt(rsold) < tol) break;
    }
}

template <int S1>
void vie2_mat_fixpoint_t(HM &G, HM &F, HM &Fcc, HM &Q, double beta, const Integ &In, int nfix, int pcf,
                         int order) {
    vie2_mat_fourier_t<S1>(G, F, Fcc, Q, beta, pcf, order);
    if (nfix <= 0) return;
    int ntau = G.ntau(), es = G.es;
    std::vector<cplx> qn_mat((long)(ntau + 1) * es), dg_mat((long)(ntau + 1) * es);
    orc_hm qn = {-1, ntau, G.s, Q.sig(), nullptr, nullptr, nullptr, qn_mat.data()};
    orc_hm dg = {-1, ntau, G.s, G.sig(), nullptr, nullptr, nullptr, dg_mat.data()};
    HM Qn(&qn), dG(&dg);
    El<S1> E(G.s);
    for (int it = 0; it < nfix; it++) {
        convolution_matsubara_t<S1>(Qn, F, G, In, beta);
        for (int r = 0; r <= ntau; r++) {
            E.incr(Qn.matptr(r), G.matptr(r));
            E.incr(Qn.matptr(r), -1.0, Q.matptr(r));
        }
        vie2_mat_fourier_t<S1>(dG, F, Fcc, Qn, beta, pcf, order);
        for (int r = 0; r <= ntau; r++) E.incr(G.matptr(r), -1.0, dG.matptr(r));
    }
}

// dyson_mat_fourier_dispatch (cntr_dyson_impl.hpp:356-446)
template <int S1>
void dyson_mat_fourier_t(HM &G, HM &Sigma, double mu, const cplx *H0, double beta, int order) {
    El<S1> E(G.s);
    int es = E.es, ntau = G.ntau(), sig = G.sig();
    std::vector<cplx> sdft((long)(ntau + 1) * es), siomn(es), gmat((long)(ntau + 1) * es);
    std::vector<cplx> z1(es), z2(es), hj(es), one(es), zinv(es);
    E.set_diag(one.data(), 1.0);
    E.set(hj.data(), H0);
    for (int l = 0; l < es; l++) hj[l] -= mu * one[l];
    int pcf = 10, m2 = ntau / 2;
    matsubara_dft<S1>(E, sdft.data(), Sigma, sig);
    set_first_order_tail<S1>(E, gmat.data(), one.data(), beta, ntau, sig);
    for (int m = -m2; m <= m2 - 1; m++)
        for (int p = -pcf; p <= pcf; p++) {
            cplx iomn(0, get_omega(m + p * ntau, beta, sig));
            matsubara_ft<S1>(E, siomn.data(), m + p * ntau, Sigma, sdft.data(), sig, beta, order);
            E.set(z1.data(), siomn.data());
            E.incr(z1.data(), hj.data());
            if (sig == 1 && m + p * ntau == 0) {
                E.inverse(zinv.data(), z1.data());
                E.set(z2.data(), zinv.data());
                E.smul(z2.data(), -1.0);
            } else {
                for (int l = 0; l < es; l++) z2[l] = iomn * one[l] - z1[l];
                E.inverse(zinv.data(), z2.data());
                E.smul(zinv.data(), 1.0 / iomn);
                E.mult(z2.data(), zinv.data(), z1.data());
            }
            E.smul(z2.data(), 1.0 / beta);
            for (int r = 0; r <= ntau; r++) {
                cplx ef = std::exp(-(r * (beta / ntau)) * iomn);
                for (int l = 0; l < es; l++) gmat[(long)r * es + l] += z2[l] * ef;
            }
        }
    std::memcpy(G.matptr(0), gmat.data(), sizeof(cplx) * gmat.size());
}

// ------------------------------------------------------------------------------------
// Dyson (cntr_dyson_impl.hpp)
// ------------------------------------------------------------------------------------
// Time step n of G^R: row n zeroed, G^R(n,n) = -i, and the start values G^R(n, n-j), j = 1..k,
// from the k x k block system of the conjugate equation (cntr_dyson_impl.hpp:98-170; the
// OpenMP variant repeats it, cntr_dyson_omp_impl.hpp:55-129).
template <int S1>
void ret_start_block_t(int n, HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double h) {
    El<S1> E(G.s);
    int k = In.k, es = E.es;
    std::vector<cplx> gtemp((long)k * es), qq((long)k * es), one(es), mm((long)k * k * es), stemp(es);
    E.set_diag(one.data(), 1.0);
    for (long i = 0; i < (long)(n + 1) * es; i++) G.retptr(n, 0)[i] = 0;
    E.set_diag(G.retptr(n, n), -kI);
    for (auto &x : mm) x = 0;
    for (long i = 0; i < (long)k * es; i++) qq[i] = 0;
    for (int j = 1; j <= k; j++) {
        int p = j - 1;
        for (int l = 0; l <= k; l++) {
            cplx cw = kI / h * In.poly_differentiation(j, l);
            if (l == 0) E.incr(qq.data() + (long)p * es, -cw, G.retptr(n, n));
            else {
                int q = l - 1;
                for (int i = 0; i < G.s; i++) mm[(long)(p * k + q) * es + i * G.s + i] += cw;
            }
        }
        E.set(gtemp.data(), H + (long)(n - j) * es);
        E.smul(gtemp.data(), -1.0);
        for (int i = 0; i < es; i++) gtemp[i] += mu * one[i];
        E.incr(mm.data() + (long)(p + k * p) * es, gtemp.data());
        for (int l = 0; l <= k; l++) {
            double w = h * In.gregory_weights(j, l);
            if (n - l >= n - j) E.set(stemp.data(), Sigma.retptr(n - l, n - j));
            else { E.set(stemp.data(), Sigma.retptr(n - j, n - l)); E.conj_inplace(stemp.data()); w = -w; }
            if (l == 0) E.incr(qq.data() + (long)p * es, w, G.retptr(n, n), stemp.data());
            else {
                int q = l - 1;
                E.incr(mm.data() + (long)(p * k + q) * es, -w, stemp.data());
            }
        }
    }
    E.linsolve_left(k, gtemp.data(), mm.data(), qq.data());
    for (int j = 1; j <= k; j++) E.set(G.retptr(n, n - j), gtemp.data() + (long)(j - 1) * es);
}

// dyson_timestep_ret (:80-222)
template <int S1>
void dyson_timestep_ret_t(int n, HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, k2 = 2 * k1, es = E.es, ss = Sigma.es;
    std::vector<cplx> diffw(k1 + 1), qq((long)(n + 1) * es), one(es), mm((long)k * k * es), hj(es), stemp(es);
    E.set_diag(one.data(), 1.0);
    ret_start_block_t<S1>(n, G, mu, H, Sigma, In, h);
    for (long i = 0; i < (long)(n + 1) * es; i++) qq[i] = 0;
    for (int m = n - k; m <= n; m++) {
        const cplx *gret = G.retptr(n, m);
        for (int j = 0; j <= n - k2; j++)
            E.incr(qq.data() + (long)j * es, In.gregory_weights(n - j, n - m), gret, Sigma.retptr(m, j));
        int j1 = n - k2 + 1 < 0 ? 0 : n - k2 + 1;
        for (int j = j1; j < n - k; j++)
            E.incr(qq.data() + (long)j * es, In.gregory_weights(n - j, n - m), gret, Sigma.retptr(m, j));
    }
    for (int p = 0; p <= k1; p++) diffw[p] = In.bd_weights(p) * kI / h;
    cplx w0 = h * In.gregory_omega(0);
    for (int l = k + 1; l <= n; l++) {
        int j = n - l;
        E.conj(hj.data(), H + (long)j * es);
        cplx *qqj = qq.data() + (long)j * es;
        for (int i = 0; i < es; i++) {
            qqj[i] *= h;
            for (int p = 1; p <= k1; p++) qqj[i] += -diffw[p] * G.retptr(n, n - l + p)[i];
        }
        E.set(stemp.data(), Sigma.retptr(j, j));
        for (int i = 0; i < es; i++) mm[i] = diffw[0] * one[i] + mu * one[i] - hj[i] - w0 * stemp[i];
        E.linsolve_left(1, G.retptr(n, j), mm.data(), qqj);
        const cplx *gret = G.retptr(n, j);
        const cplx *sret = Sigma.retptr(j, 0);
        for (int j2 = 0; j2 < j; j2++, sret += ss)
            E.incr(qq.data() + (long)j2 * es, In.gregory_weights(n - j2, n - j), gret, sret);
    }
}

// dyson_start_ret (:258-352)
template <int S1>
void dyson_start_ret_t(HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double h) {
    El<S1> E(G.s);
    int k = In.k, es = E.es, s = G.s;
    std::vector<cplx> qq((long)k * es), mm((long)k * k * es), one(es), hj(es), gtemp((long)k * es), stemp(es);
    E.set_diag(one.data(), 1.0);
    cplx minusi(0, -1);
    for (int n = 0; n <= k; n++) E.set_diag(G.retptr(n, n), cplx(0, -1.0));
    for (int j = 0; j < k; j++) {
        int dim = k - j;
        for (auto &x : qq) x = 0;
        for (auto &x : mm) x = 0;
        for (int n = j + 1; n <= k; n++) {
            int p = n - (j + 1);
            for (int l = 0; l <= k; l++) {
                int q = l - (j + 1);
                if (l <= j) {
                    E.conj(gtemp.data(), G.retptr(j, l));
                    E.smul(gtemp.data(), -1.0);
                    E.zero(stemp.data());
                    E.incr(stemp.data(), Sigma.retptr(n, l), gtemp.data());
                    for (int i = 0; i < es; i++)
                        qq[(long)p * es + i] += minusi / h * In.poly_differentiation(n, l) * gtemp[i] +
                                                h * In.poly_integration(j, n, l) * stemp[i];
                } else {
                    cplx *mpq = mm.data() + (long)(p * dim + q) * es;
                    for (int i = 0; i < es; i++) mpq[i] = -minusi / h * In.poly_differentiation(n, l) * one[i];
                    if (l == n) {
                        E.set(hj.data(), H + (long)l * es);
                        for (int i = 0; i < es; i++) mpq[i] += mu * one[i] - hj[i];
                    }
                    double w = h * In.poly_integration(j, n, l);
                    if (n >= l) E.set(stemp.data(), Sigma.retptr(n, l));
                    else { E.set(stemp.data(), Sigma.retptr(l, n)); E.conj_inplace(stemp.data()); w = -w; }
                    for (int i = 0; i < es; i++) mpq[i] -= w * stemp[i];
                }
            }
        }
        E.linsolve_right(dim, gtemp.data(), mm.data(), qq.data());
        for (int n = j + 1; n <= k; n++) E.set(G.retptr(n, j), gtemp.data() + (long)(n - (j + 1)) * es);
    }
    (void)s;
}

// dyson_timestep_tv (:651-741)
template <int S1>
void dyson_timestep_tv_t(int n, HM &G, double mu, const cplx *Hn, HM &Sigma, const Integ &In, double beta,
                         double h) {
    El<S1> E(G.s);
    int k = In.k, es = E.es, ntau = G.ntau();
    std::vector<cplx> one(es), qq(es), mm(es), stemp(es);
    E.set_diag(one.data(), 1.0);
    long n1 = (long)(ntau + 1) * es;
    cplx *gtv = G.tvptr(n, 0);
    for (long l = 0; l < n1; l++) gtv[l] = 0;
    conv_tv_into<S1>(n, G, Sigma, Sigma, G, G, In, beta, h);
    cplx ih(0, 1 / h);
    for (int m = n - k - 1; m < n; m++) {
        cplx cw = ih * In.bd_weights(n - m);
        const cplx *g0 = G.tvptr(m, 0);
        cplx *g1 = G.tvptr(n, 0);
        for (long l = 0; l < n1; l++) g1[l] -= cw * g0[l];
    }
    E.set(stemp.data(), Sigma.retptr(n, n));
    double w = -h * In.gregory_weights(n, 0);
    for (int l = 0; l < es; l++) mm[l] = ih * In.bd_weights(0) * one[l] + w * stemp[l] + mu * one[l] - Hn[l];
    for (int j = 0; j <= ntau; j++) {
        for (int l = 0; l < es; l++) qq[l] = G.tvptr(n, j)[l];
        E.linsolve_right(1, G.tvptr(n, j), mm.data(), qq.data());
    }
}

// dyson_start_tv (:747-888)
template <int S1>
void dyson_start_tv_t(HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double beta, double h) {
    El<S1> E(G.s);
    int k = In.k, es = E.es, ntau = G.ntau(), sig = G.sig();
    double dtau = beta / ntau;
    std::vector<cplx> one(es), qq((long)k * es), mm((long)k * k * es), stemp(es), gtemp((long)k * es);
    E.set_diag(one.data(), 1.0);
    for (int m = 0; m <= ntau; m++)
        for (int l = 0; l < es; l++) G.tvptr(0, m)[l] = ((double)sig) * kI * G.matptr(ntau - m)[l];
    for (int n = 1; n <= k; n++)
        for (int m = 0; m <= ntau; m++) {
            matsubara_integral_2<S1>(E, m, ntau, gtemp.data(), Sigma.tvptr(n, 0), G.matptr(0), In, G.sig());
            for (int l = 0; l < es; l++) G.tvptr(n, m)[l] = dtau * gtemp[l];
        }
    for (int m = 0; m <= ntau; m++) {
        for (auto &x : mm) x = 0;
        for (auto &x : qq) x = 0;
        for (int n = 1; n <= k; n++) {
            int p = n - 1;
            for (int j = 0; j <= k; j++) {
                cplx cw = kI / h * In.poly_differentiation(n, j);
                if (j == 0) { for (int l = 0; l < es; l++) qq[(long)p * es + l] -= cw * G.tvptr(0, m)[l]; }
                else {
                    int q = j - 1;
                    for (int l = 0; l < es; l++) mm[(long)(p * k + q) * es + l] += cw * one[l];
                }
            }
            E.set(gtemp.data(), H + (long)n * es);
            E.smul(gtemp.data(), -1.0);
            for (int l = 0; l < es; l++) gtemp[l] += mu * one[l];
            E.incr(mm.data() + (long)(p * k + p) * es, gtemp.data());
            for (int j = 0; j <= k; j++) {
                double cw = h * In.gregory_weights(n, j);
                if (j == 0) E.incr(qq.data() + (long)p * es, cw, Sigma.retptr(n, 0), G.tvptr(0, m));
                else {
                    int q = j - 1;
                    if (n >= j) E.set(stemp.data(), Sigma.retptr(n, j));
                    else { E.set(stemp.data(), Sigma.retptr(j, n)); E.conj_inplace(stemp.data()); E.smul(stemp.data(), -1.0); }
                    for (int l = 0; l < es; l++) mm[(long)(p * k + q) * es + l] += -cw * stemp[l];
                }
            }
            E.incr(qq.data() + (long)p * es, G.tvptr(n, m));
        }
        E.linsolve_right(k, gtemp.data(), mm.data(), qq.data());
        for (int n = 1; n <= k; n++) E.set(G.tvptr(n, m), gtemp.data() + (long)(n - 1) * es);
    }
}

// dyson_timestep_les (:893-1056); also the start for n <= k (dyson_start_les :1059-1066)
template <int S1>
void dyson_timestep_les_t(int n, HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double beta,
                          double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, es = E.es;
    int n1 = n > k ? n : k;
    std::vector<cplx> one(es), qq((long)k * es), mm((long)k * k * es), gtemp(es), stemp(es),
        gles((long)(n1 + 1) * es, 0.0);
    E.set_diag(one.data(), 1.0);
    conv_les_tvvt<S1>(n, 0, n1, gles.data(), G, Sigma, Sigma, G, G, In, beta, h);
    conv_les_lesadv<S1>(n, 0, n1, gles.data(), G, Sigma, Sigma, G, G, In, beta, h);
    E.conj(gles.data(), G.tvptr(n, 0));
    E.smul(gles.data(), -1.0);
    for (auto &x : mm) x = 0;
    for (auto &x : qq) x = 0;
    for (int j = 1; j <= k; j++) {
        int p = j - 1;
        E.incr(qq.data() + (long)p * es, gles.data() + (long)j * es);
        for (int m = 0; m <= k; m++) {
            cplx cw = kI / h * In.poly_differentiation(j, m);
            if (m == 0) { for (int l = 0; l < es; l++) qq[(long)p * es + l] -= cw * gles[l]; }
            else {
                int q = m - 1;
                for (int l = 0; l < es; l++) mm[(long)(p * k + q) * es + l] += cw * one[l];
            }
        }
        E.set(gtemp.data(), H + (long)j * es);
        E.smul(gtemp.data(), -1.0);
        for (int l = 0; l < es; l++) gtemp[l] += mu * one[l];
        E.incr(mm.data() + (long)(p * k + p) * es, gtemp.data());
        for (int m = 0; m <= k; m++) {
            double cw = h * In.gregory_weights(j, m);
            if (m == 0) E.incr(qq.data() + (long)p * es, cw, Sigma.retptr(j, 0), gles.data());
            else {
                int q = m - 1;
                if (j >= m) E.set(stemp.data(), Sigma.retptr(j, m));
                else { E.set(stemp.data(), Sigma.retptr(m, j)); E.conj_inplace(stemp.data()); E.smul(stemp.data(), -1.0); }
                for (int l = 0; l < es; l++) mm[(long)(p * k + q) * es + l] += -cw * stemp[l];
            }
        }
    }
    E.linsolve_right(k, gles.data() + es, mm.data(), qq.data());
    for (int j = k + 1; j <= n; j++) {
        E.zero(mm.data());
        E.set(qq.data(), gles.data() + (long)j * es);
        for (int p = 1; p <= k1; p++) {
            cplx cw = -kI / h * In.bd_weights(p);
            for (int l = 0; l < es; l++) qq[l] += cw * gles[(long)(j - p) * es + l];
        }
        for (int l = 0; l < es; l++) mm[l] += kI / h * In.bd_weights(0) * one[l];
        E.set(gtemp.data(), H + (long)j * es);
        E.smul(gtemp.data(), -1.0);
        for (int l = 0; l < es; l++) gtemp[l] += mu * one[l];
        E.incr(mm.data(), gtemp.data());
        E.set(stemp.data(), Sigma.retptr(j, j));
        for (int l = 0; l < es; l++) mm[l] += -h * stemp[l] * In.gregory_weights(j, j);
        for (int m = 0; m < j; m++)
            E.incr(qq.data(), h * In.gregory_weights(j, m), Sigma.retptr(j, m), gles.data() + (long)m * es);
        E.linsolve_right(1, gles.data() + (long)j * es, mm.data(), qq.data());
    }
    for (int j = 0; j <= n; j++) E.set(G.lesptr(j, n), gles.data() + (long)j * es);
}

// ------------------------------------------------------------------------------------
// VIE2 (cntr_vie2_impl.hpp)
// ------------------------------------------------------------------------------------
// vie2_timestep_ret (:60-210); called as (n, G, Fcc, F, Q) by vie2_timestep (:1523)
template <int S1>
void vie2_timestep_ret_t(int n, HM &G, HM &F, HM &Fcc, HM &Q, const Integ &In, double h) {
    El<S1> E(G.s);
    int k = In.k, k2 = 2 * (k + 1), es = E.es, ss = F.es;
    std::vector<cplx> gtemp((long)k * es), qq((long)(n + 1) * es), one(es), mm((long)k * k * es), stemp(es);
    E.set_diag(one.data(), 1.0);
    for (long i = 0; i < (long)(n + 1) * es; i++) G.retptr(n, 0)[i] = 0;
    E.set(G.retptr(n, n), Q.retptr(n, n));
    for (auto &x : mm) x = 0;
    for (long i = 0; i < (long)k * es; i++) qq[i] = 0;
    for (int j = 1; j <= k; j++) {
        int p = j - 1;
        E.incr(qq.data() + (long)p * es, Q.retptr(n, n - j));
        E.incr(mm.data() + (long)(p + k * p) * es, one.data());
        for (int l = 0; l <= k; l++) {
            double w = -h * In.gregory_weights(j, l);
            if (n - l >= n - j) E.set(stemp.data(), F.retptr(n - l, n - j));
            else { E.set(stemp.data(), Fcc.retptr(n - j, n - l)); E.conj_inplace(stemp.data()); w = -w; }
            if (l == 0) E.incr(qq.data() + (long)p * es, w, G.retptr(n, n), stemp.data());
            else E.incr(mm.data() + (long)(p * k + l - 1) * es, -w, stemp.data());
        }
    }
    E.linsolve_left(k, gtemp.data(), mm.data(), qq.data());
    for (int j = 1; j <= k; j++) E.set(G.retptr(n, n - j), gtemp.data() + (long)(j - 1) * es);
    for (long i = 0; i < (long)(n + 1) * es; i++) qq[i] = 0;
    for (int m = n - k; m <= n; m++) {
        const cplx *gret = G.retptr(n, m);
        for (int j = 0; j <= n - k2; j++)
            E.incr(qq.data() + (long)j * es, -In.gregory_weights(n - j, n - m), gret, F.retptr(m, j));
        int j1 = n - k2 + 1 < 0 ? 0 : n - k2 + 1;
        for (int j = j1; j < n - k; j++)
            E.incr(qq.data() + (long)j * es, -In.gregory_weights(n - j, n - m), gret, F.retptr(m, j));
    }
    cplx w0 = -h * In.gregory_omega(0);
    for (int l = k + 1; l <= n; l++) {
        int j = n - l;
        cplx *qqj = qq.data() + (long)j * es;
        for (int i = 0; i < es; i++) qqj[i] *= h;
        E.set(stemp.data(), F.retptr(j, j));
        for (int i = 0; i < es; i++) mm[i] = one[i] - w0 * stemp[i];
        E.incr(qqj, Q.retptr(n, j));
        E.linsolve_left(1, G.retptr(n, j), mm.data(), qqj);
        const cplx *gret = G.retptr(n, j);
        const cplx *sret = F.retptr(j, 0);
        for (int j2 = 0; j2 < j; j2++, sret += ss)
            E.incr(qq.data() + (long)j2 * es, -In.gregory_weights(n - j2, n - j), gret, sret);
    }
}

// vie2_start_ret (:215-300)
template <int S1>
void vie2_start_ret_t(HM &G, HM &F, HM &Fcc, HM &Q, const Integ &In, double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, es = E.es;
    std::vector<cplx> qq((long)k1 * es), mm((long)k1 * k1 * es), one(es), gtemp((long)k1 * es), stemp(es);
    E.set_diag(one.data(), 1.0);
    for (int n = 0; n <= k; n++) E.set(G.retptr(n, n), Q.retptr(n, n));
    for (int j = 0; j < k; j++) {
        int dim = k - j;
        for (long i = 0; i < (long)k * es; i++) qq[i] = 0;
        for (long i = 0; i < (long)k * k * es; i++) mm[i] = 0;
        for (int n = j + 1; n <= k; n++) {
            int p = n - (j + 1);
            E.incr(qq.data() + (long)p * es, Q.retptr(n, j));
            for (int l = 0; l <= k; l++) {
                int q = l - (j + 1);
                if (l <= j) {
                    E.conj(gtemp.data(), G.retptr(j, l));
                    E.smul(gtemp.data(), -1.0);
                    E.zero(stemp.data());
                    E.incr(stemp.data(), F.retptr(n, l), gtemp.data());
                    for (int i = 0; i < es; i++) qq[(long)p * es + i] += -h * In.poly_integration(j, n, l) * stemp[i];
                } else {
                    cplx *mpq = mm.data() + (long)(p * dim + q) * es;
                    for (int i = 0; i < es; i++) mpq[i] = 0.0;
                    if (l == n) for (int i = 0; i < es; i++) mpq[i] += one[i];
                    double w = -h * In.poly_integration(j, n, l);
                    if (n >= l) E.set(stemp.data(), F.retptr(n, l));
                    else { E.set(stemp.data(), Fcc.retptr(l, n)); E.conj_inplace(stemp.data()); w = -w; }
                    for (int i = 0; i < es; i++) mpq[i] -= w * stemp[i];
                }
            }
        }
        E.linsolve_right(dim, gtemp.data(), mm.data(), qq.data());
        for (int n = j + 1; n <= k; n++) E.set(G.retptr(n, j), gtemp.data() + (long)(n - (j + 1)) * es);
    }
}

// vie2_timestep_tv (:645-725)
template <int S1>
void vie2_timestep_tv_t(int n, HM &G, HM &F, HM &Fcc, HM &Q, const Integ &In, double beta, double h) {
    El<S1> E(G.s);
    int es = E.es, ntau = G.ntau();
    std::vector<cplx> one(es), qq(es), mm(es), stemp(es);
    E.set_diag(one.data(), 1.0);
    long n1 = (long)(ntau + 1) * es;
    for (long l = 0; l < n1; l++) G.tvptr(n, 0)[l] = 0;
    conv_tv_into<S1>(n, G, F, Fcc, G, G, In, beta, h);
    E.set(stemp.data(), F.retptr(n, n));
    double w = h * In.gregory_weights(n, 0);
    for (int l = 0; l < es; l++) mm[l] = one[l] + w * stemp[l];
    for (int j = 0; j <= ntau; j++) {
        for (int l = 0; l < es; l++) qq[l] = -G.tvptr(n, j)[l] + Q.tvptr(n, j)[l];
        E.linsolve_right(1, G.tvptr(n, j), mm.data(), qq.data());
    }
}

// vie2_start_tv (:727-842)
template <int S1>
void vie2_start_tv_t(HM &G, HM &F, HM &Fcc, HM &Q, const Integ &In, double beta, double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, es = E.es, ntau = G.ntau();
    double dtau = beta / ntau;
    std::vector<cplx> one(es), qq((long)k1 * es), mm((long)k1 * k1 * es), stemp(es), gtemp((long)k1 * es);
    E.set_diag(one.data(), 1.0);
    for (int n = 0; n <= k; n++)
        for (int m = 0; m <= ntau; m++) {
            matsubara_integral_2<S1>(E, m, ntau, gtemp.data(), F.tvptr(n, 0), G.matptr(0), In, G.sig());
            for (int l = 0; l < es; l++) G.tvptr(n, m)[l] = -dtau * gtemp[l];
        }
    for (int m = 0; m <= ntau; m++) {
        for (auto &x : mm) x = 0;
        for (auto &x : qq) x = 0;
        for (int n = 0; n <= k; n++) {
            E.incr(mm.data() + (long)(n * k1 + n) * es, one.data());
            for (int j = 0; j <= k; j++) {
                double cw = h * In.gregory_weights(n, j);
                if (n >= j) E.set(stemp.data(), F.retptr(n, j));
                else { E.set(stemp.data(), Fcc.retptr(j, n)); E.conj_inplace(stemp.data()); E.smul(stemp.data(), -1.0); }
                for (int l = 0; l < es; l++) mm[(long)(n * k1 + j) * es + l] += cw * stemp[l];
            }
            E.incr(qq.data() + (long)n * es, G.tvptr(n, m));
            E.incr(qq.data() + (long)n * es, Q.tvptr(n, m));
        }
        E.linsolve_right(k1, gtemp.data(), mm.data(), qq.data());
        for (int n = 0; n <= k; n++) E.set(G.tvptr(n, m), gtemp.data() + (long)n * es);
    }
}

// vie2_timestep_les (:847-990); vie2_start_les (:993-1000) calls it for n = 0..k
template <int S1>
void vie2_timestep_les_t(int n, HM &G, HM &F, HM &Fcc, HM &Q, const Integ &In, double beta, double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, es = E.es, n1 = n > k ? n : k;
    std::vector<cplx> one(es), qq((long)k1 * es), mm((long)k1 * k1 * es), qtemp(es), stemp(es),
        gles((long)(n1 + 1) * es, 0.0);
    E.set_diag(one.data(), 1.0);
    conv_les_tvvt<S1>(n, 0, n1, gles.data(), G, F, Fcc, G, G, In, beta, h);
    conv_les_lesadv<S1>(n, 0, n1, gles.data(), G, F, Fcc, G, G, In, beta, h);
    for (int j = 0; j <= n1; j++) E.smul(gles.data() + (long)j * es, -1.0);
    for (auto &x : mm) x = 0;
    for (auto &x : qq) x = 0;
    for (int j = 0; j <= k; j++) {
        int p = j;
        if (j <= n) E.incr(qq.data() + (long)p * es, Q.lesptr(j, n));
        else {
            E.conj(qtemp.data(), Q.lesptr(n, j));
            E.smul(qtemp.data(), -1.0);
            E.incr(qq.data() + (long)p * es, qtemp.data());
        }
        E.incr(qq.data() + (long)p * es, gles.data() + (long)j * es);
        E.incr(mm.data() + (long)(p * k1 + p) * es, one.data());
        for (int m = 0; m <= k; m++) {
            double cw = -h * In.gregory_weights(j, m);
            if (j >= m) E.set(stemp.data(), F.retptr(j, m));
            else { E.set(stemp.data(), Fcc.retptr(m, j)); E.conj_inplace(stemp.data()); E.smul(stemp.data(), -1.0); }
            for (int l = 0; l < es; l++) mm[(long)(p * k1 + m) * es + l] += -cw * stemp[l];
        }
    }
    E.linsolve_right(k1, gles.data(), mm.data(), qq.data());
    for (int j = k + 1; j <= n; j++) {
        E.zero(mm.data());
        E.set(qq.data(), gles.data() + (long)j * es);
        E.incr(qq.data(), Q.lesptr(j, n));
        E.incr(mm.data(), one.data());
        E.set(stemp.data(), F.retptr(j, j));
        for (int l = 0; l < es; l++) mm[l] += h * stemp[l] * In.gregory_weights(j, j);
        for (int m = 0; m < j; m++)
            E.incr(qq.data(), -h * In.gregory_weights(j, m), F.retptr(j, m), gles.data() + (long)m * es);
        E.linsolve_right(1, gles.data() + (long)j * es, mm.data(), qq.data());
    }
    for (int j = 0; j <= n; j++) E.set(G.lesptr(j, n), gles.data() + (long)j * es);
}

// extrapolate_timestep_dispatch (cntr_utilities_impl.hpp:22-130)
template <int S1> void extrapolate_t(int n, HM &G, const Integ &In) {
    El<S1> E(G.s);
    int ntau = G.ntau(), n1 = n + 1, k = In.k, es = E.es;
    std::vector<cplx> gt(es), gt1(es);
    if (k == 0) {
        for (int m = 0; m <= ntau; m++) E.set(G.tvptr(n1, m), G.tvptr(n, m));
        for (int j = 0; j <= n; j++) E.set(G.retptr(n1, n1 - j), G.retptr(n, n - j));
        E.set(G.retptr(n1, 0), G.retptr(n, 0));
        for (int j = 1; j <= n1; j++) E.set(G.lesptr(j, n1), G.lesptr(j - 1, n));
        E.set(G.lesptr(0, n1), G.lesptr(0, n));
        return;
    }
    std::vector<double> p1(k + 1, 0.0);
    for (int m = 0; m <= k; m++)
        for (int l = 0; l <= k; l++) p1[m] += (1 - 2 * (l % 2)) * In.poly_interpolation(l, m);
    for (int m = 0; m <= ntau; m++) {
        E.zero(gt.data());
        for (int l = 0; l <= k; l++) E.incr(gt.data(), p1[l], G.tvptr(n - l, m));
        E.set(G.tvptr(n1, m), gt.data());
    }
    for (int j = 0; j <= n - k; j++) {
        E.zero(gt.data());
        for (int l = 0; l <= k; l++) E.incr(gt.data(), p1[l], G.retptr(n - l, n - l - j));
        E.set(G.retptr(n1, n1 - j), gt.data());
    }
    for (int j = 0; j <= k; j++) {
        E.zero(gt.data());
        for (int l = 0; l <= k; l++) {
            if (n - l <= j) { E.set(gt1.data(), G.retptr(j, n - l)); E.conj_inplace(gt1.data()); E.smul(gt1.data(), -1.0); }
            else E.set(gt1.data(), G.retptr(n - l, j));
            E.incr(gt.data(), p1[l], gt1.data());
        }
        E.set(G.retptr(n1, j), gt.data());
    }
    for (int j = 0; j <= k; j++) {
        E.zero(gt.data());
        for (int l = 0; l <= k; l++) {
            if (n - l < j) { E.set(gt1.data(), G.lesptr(n - l, j)); E.conj_inplace(gt1.data()); E.smul(gt1.data(), -1.0); }
            else E.set(gt1.data(), G.lesptr(j, n - l));
            E.incr(gt.data(), p1[l], gt1.data());
        }
        E.set(G.lesptr(j, n1), gt.data());
    }
    for (int j = k + 1; j <= n1; j++) {
        E.zero(gt.data());
        for (int l = 0; l <= k; l++) E.incr(gt.data(), p1[l], G.lesptr(j - l - 1, n - l));
        E.set(G.lesptr(j, n1), gt.data());
    }
}

// ------------------------------------------------------------------------------------
// incr_convolution (cntr_convolution_impl.hpp:4164-4810): C += alpha [A * ft * B] at time
// step tstp, output element by output element, for the elements whose mask entry is set (the
// OpenMP solvers split the masks over threads).  ft points to F(0) of function data (F(t) at
// ft + t s^2) or is null; f0 = F(-1).  Run here in one thread's order.
// ------------------------------------------------------------------------------------
// incr_convolution_mat (:4164-4200)
template <int S1>
void incr_conv_mat_t(const char *mask, cplx alpha, HM &C, HM &A, const cplx *f0, HM &B, const Integ &In,
                     double beta) {
    El<S1> E(C.s);
    int ntau = A.ntau(), es = C.es;
    cplx adtau = alpha * beta * (1.0 / ntau);
    std::vector<cplx> ctemp(es), bmat1;
    const cplx *bm = B.matptr(0);
    if (f0) {
        bmat1.resize((long)(ntau + 1) * es);
        for (int m = 0; m <= ntau; m++) E.mult(bmat1.data() + (long)m * es, f0, B.matptr(m));
        bm = bmat1.data();
    }
    for (int m = 0; m <= ntau; m++) {
        if (!mask[m]) continue;
        matsubara_integral_1<S1>(E, m, ntau, ctemp.data(), A.matptr(0), bm, In, A.sig());
        E.incr(C.matptr(m), adtau, ctemp.data());
    }
}

// aret[j] = A^R(tstp, j) F(j), j = 0..n1, with A^R(tstp, j) = -Acc^R(j, tstp)^dagger for j > tstp
// (:4265-4297, 4417-4445)
template <int S1>
std::vector<cplx> incr_aret(const El<S1> &E, int tstp, int n1, HM &A, HM &Acc, const cplx *ft) {
    int es = E.es;
    std::vector<cplx> aret((long)(n1 + 1) * es), at(es);
    for (int j = 0; j <= n1; j++) {
        if (j <= tstp) E.set(at.data(), A.retptr(tstp, j));
        else E.minusconj(at.data(), Acc.retptr(j, tstp));
        if (ft) E.mult(aret.data() + (long)j * es, at.data(), ft + (long)j * es);
        else E.set(aret.data() + (long)j * es, at.data());
    }
    return aret;
}

// incr_convolution_ret (:4243-4360): C^R(tstp, n) += alpha h int_n^tstp A^R(tstp, j) F(j) B^R(j, n)
template <int S1>
void incr_conv_ret_t(int tstp, const char *mask, cplx alpha, HM &C, HM &A, HM &Acc, const cplx *ft, HM &B,
                     HM &Bcc, const Integ &In, double h) {
    El<S1> E(C.s);
    int es = C.es, k = In.k, n1 = tstp >= k ? tstp : k;
    cplx adt = alpha * h;
    std::vector<cplx> aret = incr_aret<S1>(E, tstp, n1, A, Acc, ft), ct(es), bt(es);
    auto ar = [&](int j) { return aret.data() + (long)j * es; };
    for (int n = 0; n <= tstp; n++) {
        if (!mask[n]) continue;
        int n2 = tstp - n;
        // B^R(j, n), continued by -Bcc^R(n, j)^dagger for j < n
        auto bx = [&](int j) -> const cplx * {
            if (j >= n) return B.retptr(j, n);
            E.minusconj(bt.data(), Bcc.retptr(n, j));
            return bt.data();
        };
        E.zero(ct.data());
        if (tstp < k) {
            for (int j = 0; j <= k; j++) E.incr(ct.data(), In.poly_integration(n, tstp, j), ar(j), bx(j));
        } else if (n2 < k) {
            for (int l = 0; l <= k; l++) E.incr(ct.data(), In.gregory_weights(n2, l), ar(tstp - l), bx(tstp - l));
        } else if (n2 <= 2 * k + 2) {
            for (int l = 0; l <= n2; l++) E.incr(ct.data(), In.gregory_weights(n2, l), ar(n + l), B.retptr(n + l, n));
        } else {
            for (int j = n; j <= n + k; j++) E.incr(ct.data(), In.gregory_omega(j - n), ar(j), B.retptr(j, n));
            for (int j = n + k + 1; j < tstp - k; j++) E.incr(ct.data(), ar(j), B.retptr(j, n));
            for (int l = 0; l <= k; l++) E.incr(ct.data(), In.gregory_omega(l), ar(tstp - l), B.retptr(tstp - l, n));
        }
        E.incr(C.retptr(tstp, n), adt, ct.data());
    }
}

// incr_convolution_tv (:4396-4500): C^tv(tstp, m) += alpha [ dtau int A^tv(tstp, .) f0 B^mat
//   + h sum_j w(tstp, j) A^R(tstp, j) F(j) B^tv(j, m) ]
template <int S1>
void incr_conv_tv_t(int tstp, const char *mask, cplx alpha, HM &C, HM &A, HM &Acc, const cplx *f0,
                    const cplx *ft, HM &B, HM &Bcc, const Integ &In, double beta, double h) {
    El<S1> E(C.s);
    int es = C.es, k = In.k, ntau = A.ntau(), n1 = tstp >= k ? tstp : k;
    cplx adt = alpha * h, adtau = alpha * beta * (1.0 / ntau);
    std::vector<cplx> aret = incr_aret<S1>(E, tstp, n1, A, Acc, ft), bmat1, c1(es), c2(es);
    const cplx *bm = B.matptr(0);
    if (f0) {
        bmat1.resize((long)(ntau + 1) * es);
        for (int m = 0; m <= ntau; m++) E.mult(bmat1.data() + (long)m * es, f0, B.matptr(m));
        bm = bmat1.data();
    }
    auto ar = [&](int j) { return aret.data() + (long)j * es; };
    for (int m = 0; m <= ntau; m++) {
        if (!mask[m]) continue;
        matsubara_integral_2<S1>(E, m, ntau, c1.data(), A.tvptr(tstp, 0), bm, In, B.sig());
        E.smul(c1.data(), adtau);
        E.zero(c2.data());
        if (tstp <= 2 * k + 2) {
            for (int n = 0; n <= n1; n++) E.incr(c2.data(), In.gregory_weights(tstp, n), ar(n), B.tvptr(n, m));
        } else {
            for (int n = 0; n <= k; n++) E.incr(c2.data(), In.gregory_omega(n), ar(n), B.tvptr(n, m));
            for (int n = k + 1; n < tstp - k; n++) E.incr(c2.data(), ar(n), B.tvptr(n, m));
            for (int n = tstp - k; n <= tstp; n++) E.incr(c2.data(), In.gregory_omega(tstp - n), ar(n), B.tvptr(n, m));
        }
        E.smul(c2.data(), adt);
        E.incr(C.tvptr(tstp, m), c1.data());
        E.incr(C.tvptr(tstp, m), c2.data());
    }
}

// incr_convolution_les (:4539-4760): C^<(n, tstp) += alpha [ h A^R * F B^< + h A^< * F B^A
//   - i dtau A^tv * f0 B^vt ](n, tstp); the tau integral always uses the end-corrected
//   (omega) weights.
template <int S1>
void incr_conv_les_t(int tstp, const char *mask, cplx alpha, HM &C, HM &A, HM &Acc, const cplx *f0,
                     const cplx *ft, HM &B, HM &Bcc, const Integ &In, double beta, double h) {
    El<S1> E(C.s);
    int es = C.es, k = In.k, ntau = A.ntau(), n1 = tstp >= k ? tstp : k;
    cplx adt = alpha * h, adtau = alpha * beta * (1.0 / ntau);
    std::vector<cplx> badv((long)(n1 + 1) * es), bles((long)(n1 + 1) * es), bvt((long)(ntau + 1) * es), bt(es),
        at(es), c1(es), c2(es), c3(es);
    auto lmul = [&](cplx *z, const cplx *f, const cplx *x) {  // z = f x (f may be null)
        if (f) E.mult(z, f, x); else E.set(z, x);
    };
    for (int j = 0; j <= n1; j++) {
        const cplx *fj = ft ? ft + (long)j * es : nullptr;
        if (j <= tstp) {
            E.conj(bt.data(), Bcc.retptr(tstp, j));
            lmul(badv.data() + (long)j * es, fj, bt.data());
            lmul(bles.data() + (long)j * es, fj, B.lesptr(j, tstp));
        } else {
            lmul(badv.data() + (long)j * es, fj, B.retptr(j, tstp));
            E.smul(badv.data() + (long)j * es, -1.0);
            E.minusconj(bt.data(), Bcc.lesptr(tstp, j));
            lmul(bles.data() + (long)j * es, fj, bt.data());
        }
    }
    for (int m = 0; m <= ntau; m++) {
        if (B.sig() == -1) E.conj(bt.data(), Bcc.tvptr(tstp, ntau - m));
        else E.minusconj(bt.data(), Bcc.tvptr(tstp, ntau - m));
        lmul(bvt.data() + (long)m * es, f0, bt.data());
    }
    auto bl = [&](int j) { return bles.data() + (long)j * es; };
    auto ba = [&](int j) { return badv.data() + (long)j * es; };
    auto bv = [&](int m) { return bvt.data() + (long)m * es; };
    for (int n = 0; n <= tstp; n++) {
        if (!mask[n]) continue;
        // A^<(n, j), continued by -Acc^<(j, n)^dagger (j < n)
        auto lx = [&](int j) -> const cplx * {
            if (j < n) { E.minusconj(at.data(), Acc.lesptr(j, n)); return at.data(); }
            return A.lesptr(n, j);
        };
        int nup = n > k ? n : k;
        E.zero(c1.data());
        if (n <= 2 * k + 2) {
            for (int j = 0; j <= nup; j++) {
                if (j <= n) E.incr(c1.data(), In.gregory_weights(n, j), A.retptr(n, j), bl(j));
                else {
                    E.minusconj(at.data(), Acc.retptr(j, n));
                    E.incr(c1.data(), In.gregory_weights(n, j), at.data(), bl(j));
                }
            }
        } else {
            for (int j = 0; j <= k; j++) E.incr(c1.data(), In.gregory_omega(j), A.retptr(n, j), bl(j));
            for (int j = k + 1; j < n - k; j++) E.incr(c1.data(), A.retptr(n, j), bl(j));
            for (int j = n - k; j <= n; j++) E.incr(c1.data(), In.gregory_omega(n - j), A.retptr(n, j), bl(j));
        }
        E.zero(c2.data());
        for (int m = 0; m <= k; m++) E.incr(c2.data(), In.gregory_omega(m), A.tvptr(n, m), bv(m));
        for (int m = k + 1; m < ntau - k; m++) E.incr(c2.data(), A.tvptr(n, m), bv(m));
        for (int m = ntau - k; m <= ntau; m++) E.incr(c2.data(), In.gregory_omega(ntau - m), A.tvptr(n, m), bv(m));
        E.zero(c3.data());
        if (tstp <= 2 * k + 2) {
            for (int j = 0; j <= n; j++) {
                E.minusconj(at.data(), Acc.lesptr(j, n));
                E.incr(c3.data(), In.gregory_weights(tstp, j), at.data(), ba(j));
            }
            for (int j = n + 1; j <= n1; j++) E.incr(c3.data(), In.gregory_weights(tstp, j), A.lesptr(n, j), ba(j));
        } else {
            for (int j = 0; j <= k; j++) E.incr(c3.data(), In.gregory_omega(j), lx(j), ba(j));
            for (int j = k + 1; j < tstp - k; j++) E.incr(c3.data(), lx(j), ba(j));
            for (int j = tstp - k; j <= tstp; j++) E.incr(c3.data(), In.gregory_omega(tstp - j), lx(j), ba(j));
        }
        E.incr(C.lesptr(n, tstp), adt, c1.data());
        E.incr(C.lesptr(n, tstp), adt, c3.data());
        E.incr(C.lesptr(n, tstp), adtau * cplx(0.0, -1.0), c2.data());
    }
}

// ------------------------------------------------------------------------------------
// dyson_timestep_omp (cntr_dyson_omp_impl.hpp:37-611): G^R(n, j) and G^<(j, n) for
// j < n - k from the equation in the other time argument, every j independent (the
// OpenMP loop), with BD(k+1) derivatives; G^tv as the serial step, with the masked
// convolution.  In one thread's order: every convolution of a component is complete
// before its solves.
// ------------------------------------------------------------------------------------
// dyson_timestep_ret_omp (:37-176)
template <int S1>
void dyson_timestep_ret_omp_t(int n, HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, es = E.es;
    ret_start_block_t<S1>(n, G, mu, H, Sigma, In, h);
    std::vector<char> mask(n + 1, 0);
    for (int i = 0; i < n - k; i++) mask[i] = 1;
    incr_conv_ret_t<S1>(n, mask.data(), 1.0, G, Sigma, Sigma, nullptr, G, G, In, h);
    std::vector<cplx> diffw(k1 + 1), qq(es), mm(es);
    for (int p = 0; p <= k1; p++) diffw[p] = In.bd_weights(p) * kI / h;
    cplx w0 = h * In.gregory_omega(0);
    for (int j = 0; j < n - k; j++) {
        E.set(qq.data(), G.retptr(n, j));
        for (int p = 1; p <= k1; p++) E.incr(qq.data(), -diffw[p], G.retptr(n - p, j));
        E.set_diag(mm.data(), diffw[0] + mu);
        E.incr(mm.data(), -w0, Sigma.retptr(j, j));
        E.incr(mm.data(), -1.0, H + (long)n * es);
        E.linsolve_right(1, G.retptr(n, j), mm.data(), qq.data());
    }
}

// dyson_timestep_tv_omp (:179-235)
template <int S1>
void dyson_timestep_tv_omp_t(int n, HM &G, double mu, const cplx *Hn, HM &Sigma, const Integ &In, double beta,
                             double h) {
    El<S1> E(G.s);
    int k = In.k, k1 = k + 1, es = E.es, ntau = G.ntau();
    cplx ih(0, 1.0 / h);
    for (int m = 0; m <= ntau; m++) E.zero(G.tvptr(n, m));
    std::vector<char> mask(ntau + 1, 1);
    incr_conv_tv_t<S1>(n, mask.data(), 1.0, G, Sigma, Sigma, nullptr, nullptr, G, G, In, beta, h);
    std::vector<cplx> diffw(k1 + 1), qq(es), mm(es);
    E.set_diag(mm.data(), ih * In.bd_weights(0) + mu);
    E.incr(mm.data(), -1.0, Hn);
    E.incr(mm.data(), -h * In.gregory_weights(n, 0), Sigma.retptr(n, n));
    for (int p = 0; p <= k1; p++) diffw[p] = ih * In.bd_weights(p);
    for (int m = 0; m <= ntau; m++) {
        E.set(qq.data(), G.tvptr(n, m));
        for (int p = 1; p <= k1; p++) E.incr(qq.data(), -diffw[p], G.tvptr(n - p, m));
        E.linsolve_right(1, G.tvptr(n, m), mm.data(), qq.data());
    }
}

// dyson_timestep_les_omp (:298-414); the serial step for n < 2k+1
template <int S1>
void dyson_timestep_les_omp_t(int n, HM &G, double mu, const cplx *H, HM &Sigma, const Integ &In, double beta,
                              double h) {
    int k = In.k, k1 = k + 1;
    if (n < 2 * k + 1) { dyson_timestep_les_t<S1>(n, G, mu, H, Sigma, In, beta, h); return; }
    El<S1> E(G.s);
    int es = E.es;
    for (int j = 0; j <= n; j++) E.zero(G.lesptr(j, n));
    std::vector<char> mask(n + 1, 0);
    for (int i = 0; i < n - k; i++) mask[i] = 1;
    // G^<(j, n) from the conjugate equation: [G * Sigma]^<(j, n) into G
    incr_conv_les_t<S1>(n, mask.data(), 1.0, G, G, G, nullptr, nullptr, Sigma, Sigma, In, beta, h);
    std::vector<cplx> diffw(k1 + 1), qq(es), mm(es), stemp(es);
    for (int p = 0; p <= k1; p++) diffw[p] = In.bd_weights(p) * kI / h;
    cplx w0 = h * In.gregory_omega(0);
    for (int j = 0; j < n - k; j++) {
        E.set(qq.data(), G.lesptr(j, n));
        for (int p = 1; p <= k1; p++) E.incr(qq.data(), diffw[p], G.lesptr(j, n - p));
        E.set_diag(mm.data(), -diffw[0] + mu);
        E.conj(stemp.data(), Sigma.retptr(j, j));
        E.incr(mm.data(), -w0, stemp.data());
        E.incr(mm.data(), -1.0, H + (long)n * es);
        E.linsolve_left(1, G.lesptr(j, n), mm.data(), qq.data());
    }
    // G^<(j, n), j = n-k..n, from the equation in the first argument (:370-410)
    std::vector<cplx> gles((long)(n + 1) * es, 0.0);
    conv_les_tvvt<S1>(n, n - k, n, gles.data(), G, Sigma, Sigma, G, G, In, beta, h);
    conv_les_lesadv<S1>(n, n - k, n, gles.data(), G, Sigma, Sigma, G, G, In, beta, h);
    for (int j = n - k; j <= n; j++) {
        E.set(qq.data(), gles.data() + (long)j * es);
        for (int p = 1; p <= k1; p++) E.incr(qq.data(), -kI / h * In.bd_weights(p), G.lesptr(j - p, n));
        E.set_diag(mm.data(), kI / h * In.bd_weights(0) + mu);
        E.incr(mm.data(), -1.0, H + (long)j * es);
        E.incr(mm.data(), -h * In.gregory_weights(j, j), Sigma.retptr(j, j));
        for (int m = 0; m < j; m++) E.incr(qq.data(), h * In.gregory_weights(j, m), Sigma.retptr(j, m), G.lesptr(m, n));
        E.linsolve_right(1, G.lesptr(j, n), mm.data(), qq.data());
    }
}

// vie2_timestep_omp_dispatch (cntr_vie2_impl.hpp:1851-1980) for tstp > k: [1 + F] G = Q with
// every element of the time step independent.  G^R(tstp, .), G^tv(tstp, .) and G^<(. , tstp)
// enter their own convolutions as zero; G^<(tstp, tstp) last.  Q is left unchanged (the
// reference restores it).
template <int S1>
void vie2_timestep_omp_t(int tstp, HM &G, HM &F, HM &Fcc, HM &Q, const Integ &In, double beta, double h) {
    El<S1> E(G.s);
    int es = E.es, kt = In.k, ntau = G.ntau();
    std::vector<cplx> qret((long)(tstp + 1) * es), qtv((long)(ntau + 1) * es), qles((long)(tstp + 1) * es);
    for (int n = 0; n <= tstp; n++) {
        E.set(qret.data() + (long)n * es, Q.retptr(tstp, n));
        E.set(qles.data() + (long)n * es, Q.lesptr(n, tstp));
    }
    for (int m = 0; m <= ntau; m++) E.set(qtv.data() + (long)m * es, Q.tvptr(tstp, m));
    for (int n = 0; n <= tstp; n++) { E.zero(G.retptr(tstp, n)); E.zero(G.lesptr(n, tstp)); }
    for (int m = 0; m <= ntau; m++) E.zero(G.tvptr(tstp, m));
    std::vector<cplx> mtemp(es), one(es), mm(es);
    E.set(mtemp.data(), F.retptr(tstp, tstp));
    E.smul(mtemp.data(), h);
    E.set_diag(one.data(), 1.0);
    std::vector<char> all_ret(tstp + 1, 1), all_tv(ntau + 1, 1), les_mask(tstp + 1, 1);
    les_mask[tstp] = 0;
    // retarded: Q1 = Q - F * G with G^R(tstp, .) = 0
    incr_conv_ret_t<S1>(tstp, all_ret.data(), -1.0, Q, F, Fcc, nullptr, G, G, In, h);
    for (int n = 0; n <= tstp; n++) {
        double wt = tstp < kt ? In.poly_integration(n, tstp, tstp) : In.gregory_weights(tstp - n, 0);
        E.set(mm.data(), one.data());
        E.incr(mm.data(), wt, mtemp.data());
        E.linsolve_right(1, G.retptr(tstp, n), mm.data(), Q.retptr(tstp, n));
    }
    // left-mixing
    incr_conv_tv_t<S1>(tstp, all_tv.data(), -1.0, Q, F, Fcc, nullptr, nullptr, G, G, In, beta, h);
    for (int m = 0; m <= ntau; m++) {
        E.set(mm.data(), one.data());
        E.incr(mm.data(), In.gregory_weights(tstp, tstp), mtemp.data());
        E.linsolve_right(1, G.tvptr(tstp, m), mm.data(), Q.tvptr(tstp, m));
    }
    // lesser, n < tstp: Q1 = Q - G * Fcc with G^<(., tstp) = 0
    incr_conv_les_t<S1>(tstp, les_mask.data(), -1.0, Q, G, G, nullptr, nullptr, Fcc, F, In, beta, h);
    for (int n = 0; n < tstp; n++) {
        E.set(mm.data(), one.data());
        E.incr(mm.data(), In.gregory_weights(tstp, tstp), mtemp.data());
        E.conj_inplace(mm.data());
        E.linsolve_left(1, G.lesptr(n, tstp), mm.data(), Q.lesptr(n, tstp));
    }
    // G^<(tstp, tstp), which reads this step's G^R, G^tv and G^<(n < tstp, tstp)
    std::vector<char> last(tstp + 1, 0);
    last[tstp] = 1;
    incr_conv_les_t<S1>(tstp, last.data(), -1.0, Q, G, G, nullptr, nullptr, Fcc, F, In, beta, h);
    E.set(mm.data(), one.data());
    E.incr(mm.data(), In.gregory_weights(tstp, tstp), mtemp.data());
    E.conj_inplace(mm.data());
    E.linsolve_left(1, G.lesptr(tstp, tstp), mm.data(), Q.lesptr(tstp, tstp));
    for (int n = 0; n <= tstp; n++) {
        E.set(Q.retptr(tstp, n), qret.data() + (long)n * es);
        E.set(Q.lesptr(n, tstp), qles.data() + (long)n * es);
    }
    for (int m = 0; m <= ntau; m++) E.set(Q.tvptr(tstp, m), qtv.data() + (long)m * es);
}

#define ORC_DISPATCH(fn, ...) do { if (s1 == 1) fn<1>(__VA_ARGS__); else fn<0>(__VA_ARGS__); } while (0)

}  // namespace

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
extern "C" {

double orc_gregory_weights(int k, int m, int j) { return I(k).gregory_weights(m, j); }
double orc_gregory_omega(int k, int j) { return I(k).gregory_omega(j); }
double orc_poly_integration(int k, int i, int j, int l) { return I(k).poly_integration(i, j, l); }
double orc_poly_differentiation(int k, int i, int l) { return I(k).poly_differentiation(i, l); }
double orc_poly_interpolation(int k, int a, int l) { return I(k).poly_interpolation(a, l); }
double orc_bd_weights(int k, int l) { return I(k).bd_weights(l); }
double orc_rcorr(int k, int m, int j, int l) { return I(k).rcorr(m, j, l); }

void orc_convolution_matsubara(orc_hm *C, orc_hm *A, orc_hm *B, int k, double beta) {
    HM c(C), a(A), b(B);
    int s1 = c.s;
    ORC_DISPATCH(convolution_matsubara_t, c, a, b, I(k), beta);
}

// convolution_timestep (cntr_convolution_impl.hpp:1582-1620)
void orc_convolution_timestep(int n, orc_hm *C, orc_hm *A, orc_hm *Acc, orc_hm *B, orc_hm *Bcc, int k,
                              double beta, double h) {
    if (n == -1) { orc_convolution_matsubara(C, A, B, k, beta); return; }
    HM c(C), a(A), acc(Acc), b(B), bcc(Bcc);
    int s1 = c.s;
    const Integ &In = I(k);
    ORC_DISPATCH(conv_ret, n, c, a, acc, b, bcc, In, h);
    ORC_DISPATCH(conv_tv_into, n, c, a, acc, b, bcc, In, beta, h);
    ORC_DISPATCH(conv_les, n, c, a, acc, b, bcc, In, beta, h);
}

void orc_force_matsubara_hermitian(orc_hm *Gh) {
    HM G(Gh);
    int s = G.s;
    std::vector<cplx> t(G.es);
    for (int m = 0; m <= G.ntau(); m++) {
        cplx *g = G.matptr(m);
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) t[i * s + j] = 0.5 * (g[i * s + j] + std::conj(g[j * s + i]));
        std::memcpy(g, t.data(), sizeof(cplx) * G.es);
    }
}

// vie2_mat (cntr_vie2_impl.hpp:1229-1250): method 0 = Fourier (pcf 20), 1 = steepest descent
// (40 iterations, tol 1e-12), 2 = fixpoint (6 corrections, pcf 5)
void orc_vie2_mat(orc_hm *G, orc_hm *F, orc_hm *Fcc, orc_hm *Q, double beta, int k, int method) {
    HM g(G), f(F), fcc(Fcc), q(Q);
    int s1 = g.s;
    if (method == 0) ORC_DISPATCH(vie2_mat_fourier_t, g, f, fcc, q, beta, 20, 3);
    else if (method == 1) ORC_DISPATCH(vie2_mat_steep_t, g, f, fcc, q, beta, I(k), 40, 1.0e-12);
    else ORC_DISPATCH(vie2_mat_fixpoint_t, g, f, fcc, q, beta, I(k), 6, 5, 3);
}

// dyson_mat (cntr_dyson_impl.hpp:1393-1450); method 0 = Fourier, 1 = steepest descent
// (dyson_mat_steep_dispatch, :519-540: F = -G0*Sigma, Fcc = -Sigma*G0, 40 iterations, tol 1e-12),
// 2 = fixpoint (default)
void orc_dyson_mat(orc_hm *Gh, orc_hm *Sh, double mu, const cplx *H, int k, double beta, int method,
                   int force_hermitian) {
    HM G(Gh), S(Sh);
    int s1 = G.s, ntau = G.ntau(), es = G.es;
    if (method == 0) {
        ORC_DISPATCH(dyson_mat_fourier_t, G, S, mu, H, beta, 3);
    } else {
        // dyson_mat_fixpoint_dispatch (:451-470): G0 = green_from_H, F = -G0*Sigma, Q = G0
        std::vector<cplx> g0m((long)(ntau + 1) * es), fm((long)(ntau + 1) * es);
        orc_hm g0 = {-1, ntau, G.s, G.sig(), nullptr, nullptr, nullptr, g0m.data()};
        orc_hm gf = {-1, ntau, G.s, G.sig(), nullptr, nullptr, nullptr, fm.data()};
        orc_green_from_H_const(&g0, mu, H, beta, 1.0);
        orc_convolution_matsubara(&gf, &g0, Sh, k, beta);
        for (auto &x : fm) x = -x;
        HM hg0(&g0), hf(&gf);
        if (method == 1) {
            std::vector<cplx> fcm((long)(ntau + 1) * es);
            orc_hm gfc = {-1, ntau, G.s, G.sig(), nullptr, nullptr, nullptr, fcm.data()};
            orc_convolution_matsubara(&gfc, Sh, &g0, k, beta);
            for (auto &x : fcm) x = -x;
            HM hfc(&gfc);
            ORC_DISPATCH(vie2_mat_steep_t, G, hf, hfc, hg0, beta, I(k), 40, 1.0e-12);
        } else {
            ORC_DISPATCH(vie2_mat_fixpoint_t, G, hf, hf, hg0, beta, I(k), 6, 5, 3);
        }
    }
    if (force_hermitian) orc_force_matsubara_hermitian(Gh);
}

// dyson_start (cntr_dyson_impl.hpp:1502-1535)
void orc_dyson_start(orc_hm *Gh, double mu, const cplx *H, orc_hm *Sh, int k, double beta, double h) {
    HM G(Gh), S(Sh);
    int s1 = G.s;
    const cplx *H0 = H + G.es;  // H.ptr(0)
    const Integ &In = I(k);
    ORC_DISPATCH(dyson_start_ret_t, G, mu, H0, S, In, h);
    ORC_DISPATCH(dyson_start_tv_t, G, mu, H0, S, In, beta, h);
    for (int n = 0; n <= k; n++) ORC_DISPATCH(dyson_timestep_les_t, n, G, mu, H0, S, In, beta, h);
}

// dyson_timestep (cntr_dyson_impl.hpp:1618-1648)
void orc_dyson_timestep(int n, orc_hm *Gh, double mu, const cplx *H, orc_hm *Sh, int k, double beta,
                        double h) {
    HM G(Gh), S(Sh);
    int s1 = G.s;
    const cplx *H0 = H + G.es;
    const Integ &In = I(k);
    ORC_DISPATCH(dyson_timestep_ret_t, n, G, mu, H0, S, In, h);
    ORC_DISPATCH(dyson_timestep_tv_t, n, G, mu, H0 + (long)n * G.es, S, In, beta, h);
    ORC_DISPATCH(dyson_timestep_les_t, n, G, mu, H0, S, In, beta, h);
}

// vie2_start (cntr_vie2_impl.hpp:1338-1420)
void orc_vie2_start(orc_hm *Gh, orc_hm *Fh, orc_hm *Fcch, orc_hm *Qh, int k, double beta, double h) {
    HM G(Gh), F(Fh), Fcc(Fcch), Q(Qh);
    int s1 = G.s;
    const Integ &In = I(k);
    ORC_DISPATCH(vie2_start_ret_t, G, F, Fcc, Q, In, h);
    ORC_DISPATCH(vie2_start_tv_t, G, F, Fcc, Q, In, beta, h);
    for (int n = 0; n <= k; n++) ORC_DISPATCH(vie2_timestep_les_t, n, G, F, Fcc, Q, In, beta, h);
}

// vie2_timestep (cntr_vie2_impl.hpp:1505-1596)
void orc_vie2_timestep(int n, orc_hm *Gh, orc_hm *Fh, orc_hm *Fcch, orc_hm *Qh, int k, double beta, double h,
                       int method) {
    if (n == -1) { orc_vie2_mat(Gh, Fh, Fcch, Qh, beta, k, method); return; }
    if (n <= k) { orc_vie2_start(Gh, Fh, Fcch, Qh, n, beta, h); return; }
    HM G(Gh), F(Fh), Fcc(Fcch), Q(Qh);
    int s1 = G.s;
    const Integ &In = I(k);
    ORC_DISPATCH(vie2_timestep_ret_t, n, G, Fcc, F, Q, In, h);  // note the F/Fcc swap (:1523)
    ORC_DISPATCH(vie2_timestep_tv_t, n, G, F, Fcc, Q, In, beta, h);
    ORC_DISPATCH(vie2_timestep_les_t, n, G, F, Fcc, Q, In, beta, h);
}

// vie2_timestep_sin (cntr_vie2_impl.hpp:1779-1838): [1 + F] G = Q where F and Q carry
// instantaneous parts Fsin, Qsin (cntr::function data, (nt+2) blocks, t = -1 first).  For
// t = -1..n2: Finv(t) = (1 + Fsin(t))^-1 and Gsin(t) = Finv Qsin; the regular equation is
// [1 + Finv F] G = Finv Q - (Finv F) Gsin with Fcc -> Fcc Finv, solved by vie2_timestep
// (whose dispatch gives vie2_mat for n = -1 and a start of order n for n <= k).
void orc_vie2_timestep_sin(int n, orc_hm *Gh, cplx *Gsin, orc_hm *Fh, orc_hm *Fcch, const cplx *Fsin, orc_hm *Qh,
                           const cplx *Qsin, int k, double beta, double h) {
    const int s = Fh->size, es = s * s, nt = Fh->nt, ntau = Fh->ntau;
    const int n2 = (n <= k && n >= 0) ? k : n;
    std::vector<cplx> finv((long)(n2 + 2) * es), id(es, cplx(0)), onef(es);
    for (int i = 0; i < s; i++) id[i * s + i] = 1.0;
    auto mul = [&](cplx *z, const cplx *a, const cplx *b) {  // z = a b (s x s), z may not alias
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) {
                cplx x = 0;
                for (int l = 0; l < s; l++) x += a[i * s + l] * b[l * s + j];
                z[i * s + j] = x;
            }
    };
    for (int t = -1; t <= n2; t++) {
        const cplx *fs = Fsin + (long)(t + 1) * es;
        for (int i = 0; i < es; i++) onef[i] = fs[i] + id[i];
        cplx *fi = finv.data() + (long)(t + 1) * es;
        orc_cplx_solve(s, s, onef.data(), id.data(), fi);
        mul(Gsin + (long)(t + 1) * es, fi, Qsin + (long)(t + 1) * es);
    }
    // working copies of F, Fcc, Q
    const long nret = nt >= 0 ? (long)(nt + 1) * (nt + 2) / 2 * es : 0, ntv = (long)(nt + 1) * (ntau + 1) * es,
               nmat = (long)(ntau + 1) * es;
    auto clone = [&](orc_hm *X, std::vector<cplx> &buf) {
        buf.assign(2 * nret + ntv + nmat, cplx(0));
        if (nret) std::copy(X->ret, X->ret + nret, buf.begin());
        if (nret) std::copy(X->les, X->les + nret, buf.begin() + nret);
        if (ntv) std::copy(X->tv, X->tv + ntv, buf.begin() + 2 * nret);
        std::copy(X->mat, X->mat + nmat, buf.begin() + 2 * nret + ntv);
        orc_hm v = {nt, ntau, s, X->sig, buf.data(), buf.data() + nret, buf.data() + 2 * nret,
                    buf.data() + 2 * nret + ntv};
        return v;
    };
    std::vector<cplx> bF, bFcc, bQ, bF1, tmp(es);
    orc_hm tF = clone(Fh, bF), tFcc = clone(Fcch, bFcc), tQ = clone(Qh, bQ);
    // herm_matrix::left_multiply / right_multiply at one time step (cntr_herm_matrix_impl.hpp:
    // 2955-2995, 3206-3246): f(-1) on mat, f(t) / f(m) on the slice as the time arguments say
    auto lmul = [&](orc_hm *X, int t, const cplx *f) {
        HM x(X);
        auto fp = [&](int tt) { return f + (long)(tt + 1) * es; };
        auto app = [&](cplx *e, const cplx *fa) { mul(tmp.data(), fa, e); std::copy(tmp.begin(), tmp.end(), e); };
        if (t == -1) { for (int m = 0; m <= ntau; m++) app(x.matptr(m), fp(-1)); return; }
        for (int m = 0; m <= t; m++) app(x.retptr(t, m), fp(t));
        for (int m = 0; m <= ntau; m++) app(x.tvptr(t, m), fp(t));
        for (int m = 0; m <= t; m++) app(x.lesptr(m, t), fp(m));
    };
    auto rmul = [&](orc_hm *X, int t, const cplx *f) {
        HM x(X);
        auto fp = [&](int tt) { return f + (long)(tt + 1) * es; };
        auto app = [&](cplx *e, const cplx *fa) { mul(tmp.data(), e, fa); std::copy(tmp.begin(), tmp.end(), e); };
        if (t == -1) { for (int m = 0; m <= ntau; m++) app(x.matptr(m), fp(-1)); return; }
        for (int m = 0; m <= t; m++) app(x.retptr(t, m), fp(m));
        for (int m = 0; m <= ntau; m++) app(x.tvptr(t, m), fp(-1));
        for (int m = 0; m <= t; m++) app(x.lesptr(m, t), fp(t));
    };
    for (int t = -1; t <= n2; t++) {
        lmul(&tF, t, finv.data());
        rmul(&tFcc, t, finv.data());
        lmul(&tQ, t, finv.data());
    }
    orc_hm tF1 = clone(&tF, bF1);
    for (int t = -1; t <= n2; t++) rmul(&tF1, t, Gsin);
    // tQ(t) -= tF1(t) on the time steps -1..n2 (herm_matrix::incr_timestep)
    for (int t = -1; t <= n2; t++) {
        HM q(&tQ), f1(&tF1);
        if (t == -1) {
            for (long i = 0; i < nmat; i++) q.matptr(0)[i] -= f1.matptr(0)[i];
            continue;
        }
        for (long i = 0; i < (long)(t + 1) * es; i++) q.retptr(t, 0)[i] -= f1.retptr(t, 0)[i];
        for (long i = 0; i < (long)(ntau + 1) * es; i++) q.tvptr(t, 0)[i] -= f1.tvptr(t, 0)[i];
        for (long i = 0; i < (long)(t + 1) * es; i++) q.lesptr(0, t)[i] -= f1.lesptr(0, t)[i];
    }
    orc_vie2_timestep(n, Gh, &tF, &tFcc, &tQ, k, beta, h, 2);
}

// One component of incr_convolution (cntr_convolution_impl.hpp:4164-4760): which = 0 mat,
// 1 ret, 2 tv, 3 les; mask has ntau+1 (mat, tv) or tstp+1 (ret, les) entries (null: all set);
// ftdata = function data with F(-1) first, or null.
void orc_incr_convolution_part(int which, int tstp, const char *mask, double are, double aim, orc_hm *Ch,
                               orc_hm *Ah, orc_hm *Acch, const cplx *ftdata, orc_hm *Bh, orc_hm *Bcch, int k,
                               double beta, double h) {
    HM C(Ch), A(Ah), Acc(Acch), B(Bh), Bcc(Bcch);
    int s1 = C.s;
    cplx alpha(are, aim);
    const cplx *f0 = ftdata, *ft = ftdata ? ftdata + C.es : nullptr;
    std::vector<char> all((which == 0 || which == 2 ? C.ntau() : tstp) + 1, 1);
    const char *mk = mask ? mask : all.data();
    const Integ &In = I(k);
    if (which == 0) ORC_DISPATCH(incr_conv_mat_t, mk, alpha, C, A, f0, B, In, beta);
    else if (which == 1) ORC_DISPATCH(incr_conv_ret_t, tstp, mk, alpha, C, A, Acc, ft, B, Bcc, In, h);
    else if (which == 2) ORC_DISPATCH(incr_conv_tv_t, tstp, mk, alpha, C, A, Acc, f0, ft, B, Bcc, In, beta, h);
    else ORC_DISPATCH(incr_conv_les_t, tstp, mk, alpha, C, A, Acc, f0, ft, B, Bcc, In, beta, h);
}

// incr_convolution (:4786-4807): every element of time step tstp (tstp = -1: Matsubara)
void orc_incr_convolution(int tstp, double are, double aim, orc_hm *C, orc_hm *A, orc_hm *Acc, const cplx *ftdata,
                          orc_hm *B, orc_hm *Bcc, int k, double beta, double h) {
    if (tstp == -1) {
        orc_incr_convolution_part(0, tstp, nullptr, are, aim, C, A, Acc, ftdata, B, Bcc, k, beta, h);
    } else if (tstp >= 0) {
        for (int which = 1; which <= 3; which++)
            orc_incr_convolution_part(which, tstp, nullptr, are, aim, C, A, Acc, ftdata, B, Bcc, k, beta, h);
    }
}

// dyson_timestep_omp (cntr_dyson_omp_impl.hpp:577-605); k + 1 <= n
void orc_dyson_timestep_omp(int n, orc_hm *Gh, double mu, const cplx *H, orc_hm *Sh, int k, double beta,
                            double h) {
    HM G(Gh), S(Sh);
    int s1 = G.s;
    const cplx *H0 = H + G.es;
    const Integ &In = I(k);
    ORC_DISPATCH(dyson_timestep_ret_omp_t, n, G, mu, H0, S, In, h);
    ORC_DISPATCH(dyson_timestep_tv_omp_t, n, G, mu, H0 + (long)n * G.es, S, In, beta, h);
    ORC_DISPATCH(dyson_timestep_les_omp_t, n, G, mu, H0, S, In, beta, h);
}

// vie2_timestep_omp (cntr_vie2_impl.hpp:2125-2190): tstp = -1 vie2_mat, tstp <= k vie2_start of
// order tstp, else the element-parallel step
void orc_vie2_timestep_omp(int tstp, orc_hm *Gh, orc_hm *Fh, orc_hm *Fcch, orc_hm *Qh, int k, double beta, double h,
                           int method) {
    if (tstp == -1) { orc_vie2_mat(Gh, Fh, Fcch, Qh, beta, k, method); return; }
    if (tstp <= k) { orc_vie2_start(Gh, Fh, Fcch, Qh, tstp, beta, h); return; }
    HM G(Gh), F(Fh), Fcc(Fcch), Q(Qh);
    int s1 = G.s;
    ORC_DISPATCH(vie2_timestep_omp_t, tstp, G, F, Fcc, Q, I(k), beta, h);
}

void orc_extrapolate_timestep(int n, orc_hm *Gh, int k) {
    HM G(Gh);
    int s1 = G.s;
    ORC_DISPATCH(extrapolate_t, n, G, I(k));
}

// distance_norm2_dispatch (cntr_utilities_impl.hpp:607-650)
double orc_distance_norm2(int tstp, orc_hm *g1h, orc_hm *g2h) {
    HM g1(g1h), g2(g2h);
    int es = g1.es, ntau = g1.ntau();
    auto nrm = [&](const cplx *a, const cplx *b) {
        double r = 0;
        for (int i = 0; i < es; i++) r += std::norm(a[i] - b[i]);
        return std::sqrt(r);
    };
    double err = 0;
    if (tstp == -1) {
        for (int i = 0; i <= ntau; i++) err += nrm(g1.matptr(i), g2.matptr(i));
    } else {
        for (int i = 0; i <= tstp; i++) err += nrm(g1.retptr(tstp, i), g2.retptr(tstp, i));
        for (int i = 0; i <= ntau; i++) err += nrm(g1.tvptr(tstp, i), g2.tvptr(tstp, i));
        for (int i = 0; i <= tstp; i++) err += nrm(g1.lesptr(i, tstp), g2.lesptr(i, tstp));
    }
    return err;
}

// get_bubble_1_timestep / _mat for 1x1 functions (cntr_bubble_impl.hpp:15-75)
void orc_bubble1_scalar(int tstp, orc_hm *Ch, orc_hm *Ah, orc_hm *Acch, orc_hm *Bh, orc_hm *Bcch) {
    HM C(Ch), A(Ah), Acc(Acch), B(Bh), Bcc(Bcch);
    int ntau = C.ntau();
    if (tstp == -1) {
        double sg = -1.0 * B.sig();
        for (int m = 0; m <= ntau; m++) *C.matptr(m) = sg * *A.matptr(m) * *B.matptr(ntau - m);
        return;
    }
    cplx msigb = -1.0 * B.sig();
    for (int m = 0; m <= tstp; m++) {
        cplx bles_tt1 = -std::conj(*Bcc.lesptr(m, tstp));
        cplx bgtr_tt1 = *B.retptr(tstp, m) + bles_tt1;
        cplx bles_t1t = *B.lesptr(m, tstp);
        cplx bgtr_t1t = -std::conj(*Bcc.retptr(tstp, m)) + bles_t1t;
        cplx ales_tt1 = -std::conj(*Acc.lesptr(m, tstp));
        cplx agtr_tt1 = *A.retptr(tstp, m) + ales_tt1;
        cplx cgtr = kI * agtr_tt1 * bles_t1t;
        cplx cles = kI * ales_tt1 * bgtr_t1t;
        *C.retptr(tstp, m) = cgtr - cles;
        *C.lesptr(m, tstp) = kI * *A.lesptr(m, tstp) * bgtr_tt1;
    }
    for (int m = 0; m <= ntau; m++) {
        cplx bvt = msigb * std::conj(*Bcc.tvptr(tstp, ntau - m));
        *C.tvptr(tstp, m) = kI * *A.tvptr(tstp, m) * bvt;
    }
}

// get_bubble_2_timestep / _mat for 1x1 functions (cntr_bubble_impl.hpp:100-160)
void orc_bubble2_scalar(int tstp, orc_hm *Ch, orc_hm *Ah, orc_hm *Acch, orc_hm *Bh, orc_hm *Bcch) {
    HM C(Ch), A(Ah), Acc(Acch), B(Bh), Bcc(Bcch);
    int ntau = C.ntau();
    if (tstp == -1) {
        for (int m = 0; m <= ntau; m++) *C.matptr(m) = -*A.matptr(m) * *B.matptr(m);
        return;
    }
    for (int m = 0; m <= tstp; m++) {
        cplx bgtr = *B.retptr(tstp, m) - std::conj(*Bcc.lesptr(m, tstp));
        cplx agtr = *A.retptr(tstp, m) - std::conj(*Acc.lesptr(m, tstp));
        cplx cgtr = kI * agtr * bgtr;
        cplx cles = kI * std::conj(*Acc.lesptr(m, tstp)) * std::conj(*Bcc.lesptr(m, tstp));
        *C.retptr(tstp, m) = cgtr - cles;
        *C.lesptr(m, tstp) = kI * *A.lesptr(m, tstp) * *B.lesptr(m, tstp);
    }
    for (int m = 0; m <= ntau; m++) *C.tvptr(tstp, m) = kI * *A.tvptr(tstp, m) * *B.tvptr(tstp, m);
}

// Element-index bubbles (cntr_bubble_impl.hpp:17-130, 138-330):
//   Bubble1: C_{c1c2}(t,t') = i A_{a1a2}(t,t') B_{b2b1}(t',t)
//   Bubble2: C_{c1c2}(t,t') = i A_{a1a2}(t,t') B_{b1b2}(t,t')
// at time step tstp (tstp = -1: Matsubara, C(tau) = -sig_B A(tau) B(beta - tau) and
// -A(tau) B(tau)); the continuations to t' > t come from the partners Acc, Bcc.
void orc_bubble1(int tstp, orc_hm *Ch, int c1, int c2, orc_hm *Ah, orc_hm *Acch, int a1, int a2, orc_hm *Bh,
                 orc_hm *Bcch, int b1, int b2) {
    HM C(Ch), A(Ah), Acc(Acch), B(Bh), Bcc(Bcch);
    const int ntau = C.ntau(), c12 = c1 * C.s + c2, a12 = a1 * A.s + a2, a21 = a2 * A.s + a1;
    const int b12 = b1 * B.s + b2, b21 = b2 * B.s + b1;
    if (tstp == -1) {
        const double sg = -1.0 * B.sig();
        for (int m = 0; m <= ntau; m++) C.matptr(m)[c12] = sg * A.matptr(m)[a12] * B.matptr(ntau - m)[b21];
        return;
    }
    const cplx msigb = -1.0 * B.sig();
    for (int m = 0; m <= tstp; m++) {
        const cplx bles21_tt1 = -std::conj(Bcc.lesptr(m, tstp)[b12]);     // B^<_{21}(t, m)
        const cplx bgtr21_tt1 = B.retptr(tstp, m)[b21] + bles21_tt1;        // B^>_{21}(t, m)
        const cplx bles21_t1t = B.lesptr(m, tstp)[b21];                     // B^<_{21}(m, t)
        const cplx bgtr21_t1t = -std::conj(Bcc.retptr(tstp, m)[b12]) + bles21_t1t;
        const cplx ales12_tt1 = -std::conj(Acc.lesptr(m, tstp)[a21]);       // A^<_{12}(t, m)
        const cplx agtr12_tt1 = A.retptr(tstp, m)[a12] + ales12_tt1;
        C.retptr(tstp, m)[c12] = kI * agtr12_tt1 * bles21_t1t - kI * ales12_tt1 * bgtr21_t1t;
        C.lesptr(m, tstp)[c12] = kI * A.lesptr(m, tstp)[a12] * bgtr21_tt1;
    }
    for (int m = 0; m <= ntau; m++) {
        const cplx bvt21 = msigb * std::conj(Bcc.tvptr(tstp, ntau - m)[b12]);  // B^vt_{21}(m, t)
        C.tvptr(tstp, m)[c12] = kI * A.tvptr(tstp, m)[a12] * bvt21;
    }
}

void orc_bubble2(int tstp, orc_hm *Ch, int c1, int c2, orc_hm *Ah, orc_hm *Acch, int a1, int a2, orc_hm *Bh,
                 orc_hm *Bcch, int b1, int b2) {
    HM C(Ch), A(Ah), Acc(Acch), B(Bh), Bcc(Bcch);
    const int ntau = C.ntau(), c12 = c1 * C.s + c2, a12 = a1 * A.s + a2, a21 = a2 * A.s + a1;
    const int b12 = b1 * B.s + b2, b21 = b2 * B.s + b1;
    if (tstp == -1) {
        for (int m = 0; m <= ntau; m++) C.matptr(m)[c12] = -A.matptr(m)[a12] * B.matptr(m)[b12];
        return;
    }
    for (int m = 0; m <= tstp; m++) {
        const cplx bgtr12_tt1 = B.retptr(tstp, m)[b12] - std::conj(Bcc.lesptr(m, tstp)[b21]);
        const cplx agtr12_tt1 = A.retptr(tstp, m)[a12] - std::conj(Acc.lesptr(m, tstp)[a21]);
        const cplx cles_tt1 = kI * std::conj(Acc.lesptr(m, tstp)[a21]) * std::conj(Bcc.lesptr(m, tstp)[b21]);
        C.retptr(tstp, m)[c12] = kI * agtr12_tt1 * bgtr12_tt1 - cles_tt1;
        C.lesptr(m, tstp)[c12] = kI * A.lesptr(m, tstp)[a12] * B.lesptr(m, tstp)[b12];
    }
    for (int m = 0; m <= ntau; m++) C.tvptr(tstp, m)[c12] = kI * A.tvptr(tstp, m)[a12] * B.tvptr(tstp, m)[b12];
}

void orc_dyson_timestep_batch(int n0, int n1, int nprob, orc_hm *G, double mu, const cplx *H, long h_stride,
                              orc_hm *Sigma, int k, double beta, double h, int nthreads) {
    integ_init_all();  // integration::I is not thread-safe on first use (integration.hpp:506-514)
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int p = 0; p < nprob; p++)
        for (int n = n0; n <= n1; n++) orc_dyson_timestep(n, &G[p], mu, H + (long)p * h_stride, Sigma, k, beta, h);
    (void)nthreads;
}

// ------------------------------------------------------------------------------------
// Self-consistent lattice with a local second-order self-energy
// ------------------------------------------------------------------------------------
// Sigma_2B at one time step (examples/programs/hubbard_chain_selfen_impl.cpp:63-75):
//   Pol_ij = -Bubble1(G_ij, G_ij)              (Polarization, :25-34)
//   Pol   <- U(t) Pol U(t')                    (herm_matrix_timestep::right_multiply then
//                                               left_multiply, cntr_herm_matrix_timestep_impl.hpp:1570-1860)
//   Sigma_ij = Bubble2(G_ij, Pol_ij)           (cntr_bubble_impl.hpp:100-150)
// with Bubble1(c,a,b) = i A_{a1a2}(t,t') B_{b2b1}(t',t), Bubble2 = i A_{a1a2}(t,t') B_{b1b2}(t,t')
// (get_bubble_1_timestep / get_bubble_2_timestep, cntr_bubble_impl.hpp:33-150).  U holds (nt+2)
// s x s blocks, U(-1) first (cntr::function layout); tstp = -1 gives Sigma^mat.
void orc_sigma_2b_timestep(int tstp, orc_hm *Sh, orc_hm *Gh, const cplx *U) {
    HM S(Sh), G(Gh);
    const int s = G.s, es = G.es, ntau = G.ntau();
    const cplx ii(0.0, 1.0);
    const cplx *U0 = U;           // U(-1)
    auto Ut = [&](int t) { return U + (long)(t + 1) * es; };
    auto mm = [&](const cplx *a, const cplx *b, cplx *c) {  // c = a b (element_mult)
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++) {
                cplx x = 0;
                for (int l = 0; l < s; l++) x += a[i * s + l] * b[l * s + j];
                c[i * s + j] = x;
            }
    };
    std::vector<cplx> tmp(es);
    if (tstp == -1) {
        std::vector<cplx> pm((long)(ntau + 1) * es);
        const double sg = -1.0 * G.sig();
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++)
                for (int m = 0; m <= ntau; m++)
                    pm[(long)m * es + i * s + j] = -(sg * G.matptr(m)[i * s + j] * G.matptr(ntau - m)[j * s + i]);
        for (int m = 0; m <= ntau; m++) {
            mm(pm.data() + (long)m * es, U0, tmp.data());
            mm(U0, tmp.data(), pm.data() + (long)m * es);
        }
        for (int i = 0; i < s; i++)
            for (int j = 0; j < s; j++)
                for (int m = 0; m <= ntau; m++)
                    S.matptr(m)[i * s + j] = -G.matptr(m)[i * s + j] * pm[(long)m * es + i * s + j];
        return;
    }
    const int n = tstp;
    std::vector<cplx> pret((long)(n + 1) * es), ples((long)(n + 1) * es), ptv((long)(ntau + 1) * es);
    for (int i = 0; i < s; i++)
        for (int j = 0; j < s; j++) {
            const int a12 = i * s + j, a21 = j * s + i;
            for (int m = 0; m <= n; m++) {
                const cplx *gr = G.retptr(n, m), *gl = G.lesptr(m, n);
                cplx bles21_tt1 = -std::conj(gl[a12]);
                cplx bgtr21_tt1 = gr[a21] + bles21_tt1;
                cplx bles21_t1t = gl[a21];
                cplx bgtr21_t1t = -std::conj(gr[a12]) + bles21_t1t;
                cplx ales12_tt1 = -std::conj(gl[a21]);
                cplx agtr12_tt1 = gr[a12] + ales12_tt1;
                cplx cgtr = ii * agtr12_tt1 * bles21_t1t;
                cplx cles = ii * ales12_tt1 * bgtr21_t1t;
                pret[(long)m * es + a12] = -(cgtr - cles);
                ples[(long)m * es + a12] = -(ii * gl[a12] * bgtr21_tt1);
            }
            const cplx msigb = -1.0 * G.sig();
            for (int m = 0; m <= ntau; m++) {
                cplx bvt21 = msigb * std::conj(G.tvptr(n, ntau - m)[a12]);
                ptv[(long)m * es + a12] = -(ii * G.tvptr(n, m)[a12] * bvt21);
            }
        }
    // right_multiply(tstp, U): ret(n,m) U(m), tv U(-1), les(m,n) U(n); then left_multiply:
    // U(n) ret(n,m), U(n) tv, U(m) les(m,n)
    for (int m = 0; m <= n; m++) {
        mm(pret.data() + (long)m * es, Ut(m), tmp.data());
        mm(Ut(n), tmp.data(), pret.data() + (long)m * es);
        mm(ples.data() + (long)m * es, Ut(n), tmp.data());
        mm(Ut(m), tmp.data(), ples.data() + (long)m * es);
    }
    for (int m = 0; m <= ntau; m++) {
        mm(ptv.data() + (long)m * es, U0, tmp.data());
        mm(Ut(n), tmp.data(), ptv.data() + (long)m * es);
    }
    for (int i = 0; i < s; i++)
        for (int j = 0; j < s; j++) {
            const int a12 = i * s + j, a21 = j * s + i;
            for (int m = 0; m <= n; m++) {
                const cplx *gr = G.retptr(n, m), *gl = G.lesptr(m, n);
                const cplx *br = pret.data() + (long)m * es, *bl = ples.data() + (long)m * es;
                cplx bgtr12 = br[a12] - std::conj(bl[a21]);
                cplx agtr12 = gr[a12] - std::conj(gl[a21]);
                cplx cgtr = ii * agtr12 * bgtr12;
                cplx cles = ii * std::conj(gl[a21]) * std::conj(bl[a21]);
                S.retptr(n, m)[a12] = cgtr - cles;
                S.lesptr(m, n)[a12] = ii * gl[a12] * bl[a12];
            }
            for (int m = 0; m <= ntau; m++) S.tvptr(n, m)[a12] = ii * G.tvptr(n, m)[a12] * ptv[(long)m * es + a12];
        }
}

// G_loc(tstp) = (1/nprob) sum_p G_p(tstp): the k-average of the lattice drivers
// (examples/programs/gw_kpoints_impl.cpp:139-180 gathers the k slices and sums them).
void orc_gloc_timestep(int tstp, int nprob, orc_hm *G, orc_hm *Gloch) {
    HM L(Gloch);
    const int es = L.es, ntau = L.ntau();
    const double w = 1.0 / nprob;
    auto avg = [&](auto ptr_of) {
        cplx *dst = ptr_of(L);
        for (int e = 0; e < es; e++) {
            cplx acc = 0;
            for (int p = 0; p < nprob; p++) {
                HM Gp(&G[p]);
                acc += ptr_of(Gp)[e];
            }
            dst[e] = acc * w;
        }
    };
    if (tstp == -1) {
        for (int m = 0; m <= ntau; m++) avg([&](const HM &X) { return X.matptr(m); });
        return;
    }
    for (int m = 0; m <= tstp; m++) {
        avg([&](const HM &X) { return X.retptr(tstp, m); });
        avg([&](const HM &X) { return X.lesptr(m, tstp); });
    }
    for (int m = 0; m <= ntau; m++) avg([&](const HM &X) { return X.tvptr(tstp, m); });
}

// Bootstrap of the lattice (examples/programs/hubbard_chain_2b.cpp:245-290 with G -> G_loc):
// per iteration Sigma(0..k) = Sigma_2B[G_loc, U], dyson_start of every problem, G_loc(0..k),
// err = sum_t distance_norm2(t, G_loc, previous G_loc); stop once err < tol and iter > 2.
// Returns the number of iterations run; *err_out is the last err.
int orc_lattice2b_start(int nprob, orc_hm *G, orc_hm *Gloc, orc_hm *Sigma, const cplx *U, double mu,
                        const cplx *H, long h_stride, int k, double beta, double h, int max_iter, double tol,
                        double *err_out, int nthreads) {
    integ_init_all();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    HM L(Gloc);
    for (int t = 0; t <= k; t++) orc_gloc_timestep(t, nprob, G, Gloc);
    // previous G_loc slices 0..k, in a herm_matrix of nt = k
    std::vector<cplx> pr((long)(k + 1) * (k + 2) / 2 * L.es), pl(pr.size()), ptv((long)(k + 1) * (L.ntau() + 1) * L.es);
    orc_hm prev = {k, L.ntau(), L.s, L.sig(), pr.data(), pl.data(), ptv.data(), nullptr};
    auto save = [&]() {
        std::memcpy(pr.data(), Gloc->ret, pr.size() * sizeof(cplx));
        std::memcpy(pl.data(), Gloc->les, pl.size() * sizeof(cplx));
        std::memcpy(ptv.data(), Gloc->tv, ptv.size() * sizeof(cplx));
    };
    save();
    int iter = 0;
    double err = 0;
    for (iter = 0; iter <= max_iter; iter++) {
        for (int t = 0; t <= k; t++) orc_sigma_2b_timestep(t, Sigma, Gloc, U);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
        for (int p = 0; p < nprob; p++) orc_dyson_start(&G[p], mu, H + (long)p * h_stride, Sigma, k, beta, h);
        for (int t = 0; t <= k; t++) orc_gloc_timestep(t, nprob, G, Gloc);
        err = 0;
        for (int t = 0; t <= k; t++) err += orc_distance_norm2(t, Gloc, &prev);
        if (err < tol && iter > 2) break;
        save();
    }
    if (err_out) *err_out = err;
    (void)nthreads;
    return iter > max_iter ? max_iter + 1 : iter + 1;
}

// One time step of the lattice (examples/programs/hubbard_chain_2b.cpp:306-324 with G -> G_loc):
// predictor extrapolate_timestep(n-1) of every problem, then ncorr x [G_loc(n), Sigma_2B(n),
// dyson_timestep(n) of every problem], then G_loc(n) of the final G.
void orc_lattice2b_timestep(int n, int nprob, orc_hm *G, orc_hm *Gloc, orc_hm *Sigma, const cplx *U, double mu,
                            const cplx *H, long h_stride, int k, double beta, double h, int ncorr, int nthreads) {
    integ_init_all();
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int p = 0; p < nprob; p++) orc_extrapolate_timestep(n - 1, &G[p], k);
    for (int it = 0; it < ncorr; it++) {
        orc_gloc_timestep(n, nprob, G, Gloc);
        orc_sigma_2b_timestep(n, Sigma, Gloc, U);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
        for (int p = 0; p < nprob; p++) orc_dyson_timestep(n, &G[p], mu, H + (long)p * h_stride, Sigma, k, beta, h);
    }
    orc_gloc_timestep(n, nprob, G, Gloc);
    (void)nthreads;
}

}  // extern "C"
