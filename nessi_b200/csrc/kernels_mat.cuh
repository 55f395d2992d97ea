// dyson_mat on the device (libcntr cntr_dyson_impl.hpp:1393-1450, default CNTR_MAT_FIXPOINT):
//   G0 = green_from_H(H(-1))                        (cntr_equilibrium_impl.hpp:873-900, mat only)
//   F  = -G0 * Sigma  (convolution_matsubara)       (cntr_convolution_impl.hpp:560-582, :86-224)
//   G  = vie2_mat_fixpoint(F, Q = G0): a Fourier solve (vie2_mat_fourier_dispatch,
//        cntr_vie2_impl.hpp:305-455) and 6 corrections G -= fourier(F, F*G + G - G0) (:460-484)
//   force_matsubara_hermitian                       (cntr_utilities_impl.hpp:2077-2090)
// One CTA per problem; per-problem scratch in global memory (7 vectors of (ntau+1) s^2).
//
// The Fourier solve sums z(omega_{m + p ntau}) e^{-i omega r dtau} over the oversampling copies
// p = -pcf..pcf and the frequencies m.  Since omega_{m + p ntau} r dtau = pi (2m + 2p ntau + one) r / ntau,
// the phase depends only on q = (2(m + p ntau) + one) mod 2 ntau: contributions are first
// summed per q (exact integer arithmetic), then one DFT with twiddles e^{-i pi q r / ntau} over q.
#pragma once

__device__ __forceinline__ double d_fermi(double beta, double w) {
    const double arg = w * beta;
    if (fabs(arg) > 100.0) return arg > 0.0 ? 0.0 : 1.0;
    return 1.0 / (1.0 + exp(arg));
}
__device__ __forceinline__ double d_fermi_exp(double beta, double tau, double w) {
    if (w < 0) return exp(w * tau) * d_fermi(beta, w);
    return exp((tau - beta) * w) * d_fermi(beta, -w);
}
__device__ inline double d_bose(double beta, double w) {
    double arg = w * beta;
    double sign = 1.0, add = 0.0;
    if (arg < 0) { arg = -arg; sign = -1.0; add = -1.0; }
    double v;
    if (arg > 100.0) v = 0.0;
    else if (arg < 1e-10) v = 1.0 / arg;
    else v = 1.0 / (exp(arg) - 1.0);
    return add + sign * v;  // bose(-x) = -1 - bose(x)
}
__device__ __forceinline__ double d_bose_exp(double beta, double tau, double w) {
    if (w < 0) return exp(tau * w) * d_bose(beta, w);
    return -exp((tau - beta) * w) * d_bose(beta, -w);
}

// Hermitian eigen-decomposition A = V diag(ev) V^dagger by cyclic complex Jacobi rotations
// (one thread; S <= 8).
template <int S>
__device__ void herm_eig_dev(const double2 *A0, double *ev, double2 *V) {
    double2 A[S * S];
    for (int i = 0; i < S * S; i++) { A[i] = A0[i]; V[i] = cmk(0, 0); }
    for (int i = 0; i < S; i++) V[i * S + i] = cmk(1, 0);
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0;
        for (int p = 0; p < S; p++)
            for (int q = p + 1; q < S; q++) off += cabs2(A[p * S + q]);
        if (off < 1e-30) break;
        for (int p = 0; p < S; p++)
            for (int q = p + 1; q < S; q++) {
                const double2 apq = A[p * S + q];
                const double mag = sqrt(cabs2(apq));
                if (mag < 1e-300) continue;
                const double app = A[p * S + p].x, aqq = A[q * S + q].x;
                const double2 ph = cscale(apq, 1.0 / mag);
                const double theta = 0.5 * atan2(2.0 * mag, aqq - app);
                const double c = cos(theta), sn = sin(theta);
                const double2 rpp = cmk(c, 0), rqq = cmk(c, 0), rpq = cscale(ph, sn), rqp = cscale(cconj(ph), -sn);
                for (int i = 0; i < S; i++) {
                    const double2 aip = A[i * S + p], aiq = A[i * S + q];
                    A[i * S + p] = cadd(cmul(aip, rpp), cmul(aiq, rqp));
                    A[i * S + q] = cadd(cmul(aip, rpq), cmul(aiq, rqq));
                }
                for (int j = 0; j < S; j++) {
                    const double2 apj = A[p * S + j], aqj = A[q * S + j];
                    A[p * S + j] = cadd(cmul(cconj(rpp), apj), cmul(cconj(rqp), aqj));
                    A[q * S + j] = cadd(cmul(cconj(rpq), apj), cmul(cconj(rqq), aqj));
                }
                for (int i = 0; i < S; i++) {
                    const double2 vip = V[i * S + p], viq = V[i * S + q];
                    V[i * S + p] = cadd(cmul(vip, rpp), cmul(viq, rqp));
                    V[i * S + q] = cadd(cmul(vip, rpq), cmul(viq, rqq));
                }
            }
    }
    for (int i = 0; i < S; i++) ev[i] = A[i * S + i].x;
}

// Endpoint-corrected DFT weights of cubic order (Numerical Recipes 2nd ed., section 13.9,
// routine dftcor), the correction matsubara_ft applies (fourier.cpp:43-99).
__device__ inline void dftcorr_cubic_dev(double th, double *corfac, double2 *endcor) {
    double ar[4], ai[4];
    if (fabs(th) < 5.0e-2) {
        const double t = th, t2 = t * t, t4 = t2 * t2, t6 = t4 * t2;
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
        const double c = cos(th), s = sin(th), c2 = c * c - s * s, s2 = 2.0 * s * c;
        const double t2 = th * th, t4 = t2 * t2, tm = 3.0 - t2, sp = 6.0 + t2;
        const double sth4i = 1.0 / (6.0 * t4), tth4i = 2.0 * sth4i;
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
    for (int j = 0; j < 4; j++) endcor[j] = cmk(ar[j], ai[j]);
}

struct MatScratch {
    double2 *G0, *F, *Q, *dG, *fdft, *qdft, *Z;  // each (ntau+1) s^2, Z: 2 ntau s^2
};

// twiddle e^{i pi q / ntau} for integer q from the table tw[0..2 ntau) (shared memory)
__device__ __forceinline__ double2 twid(const double2 *tw, long q, int ntau) {
    long r = q % (2L * ntau);
    if (r < 0) r += 2L * ntau;
    return tw[r];
}

// C(m) = dtau * matsubara_integral_1(m; A, B, sig) for m = 0..ntau (conv_impl :86-224)
template <int S>
__device__ void conv_mat_dev(double2 *C, const double2 *A, const double2 *B, int k, int ntau, int sig, double dtau) {
    constexpr int s2 = S * S;
    for (int e = threadIdx.x; e < (ntau + 1) * s2; e += blockDim.x) {
        const int m = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
        auto mac = [&](double2 &acc, double w, const double2 *x, const double2 *y) {
            double2 t = cmk(0, 0);
            for (int b = 0; b < S; b++) t = cfma(x[a * S + b], y[b * S + d], t);
            acc = cfma(cmk(w, 0), t, acc);
        };
        if (m >= k) {
            for (int j = 0; j <= m; j++) mac(c1, greg_w(k, m, j), A + (long)(m - j) * s2, B + (long)j * s2);
        } else if (m > 0) {
            for (int l = 0; l <= k; l++)
                for (int j = 0; j <= k; j++) mac(c1, rcorr_w(k, m, l, j), A + (long)l * s2, B + (long)j * s2);
        }
        const int r = ntau - m;
        if (r >= k) {
            for (int j = m; j <= ntau; j++)
                mac(c2, greg_w(k, r, ntau - j), A + (long)(ntau - j + m) * s2, B + (long)j * s2);
        } else if (r > 0) {
            for (int l = 0; l <= k; l++)
                for (int j = 0; j <= k; j++)
                    mac(c2, rcorr_w(k, r, l, j), A + (long)(ntau - l) * s2, B + (long)(ntau - j) * s2);
        }
        C[e] = cscale(cadd(c1, cscale(c2, (double)sig)), dtau);
    }
}

// mdft(m) = sum_r G(r) e^{i pi (2m + one) r / ntau}, m = 0..ntau (cntr_matsubara_impl.hpp:134-160)
template <int S>
__device__ void mat_dft_dev(double2 *mdft, const double2 *G, int ntau, int one, const double2 *tw) {
    constexpr int s2 = S * S;
    for (int e = threadIdx.x; e < (ntau + 1) * s2; e += blockDim.x) {
        const int m = e / s2, ab = e % s2;
        const long step = 2 * m + one, NQ = 2L * ntau;
        double2 z = cmk(0, 0);
        long q = 0;
        for (int r = 0; r <= ntau; r++, q += step) {
            if (q >= NQ) q %= NQ;
            z = cfma(G[(long)r * s2 + ab], tw[q], z);
        }
        mdft[e] = z;
    }
}

// matsubara_ft (cntr_matsubara_impl.hpp:191-248), order 3, element ab
template <int S>
__device__ __forceinline__ void mat_ft_dev(double2 *res, int mm, const double2 *G, const double2 *mdft, int ntau, int sig,
                                           double beta, int one) {
    constexpr int s2 = S * S;
    const double dtau = beta / ntau, arg = (2.0 * mm + one) * 3.14159265358979323846 / ntau;
    double corfac;
    double2 bc[4];
    dftcorr_cubic_dev(arg, &corfac, bc);
    int m1 = mm % ntau;
    if (m1 < 0) m1 += ntau;
    for (int ab = 0; ab < s2; ab++) {
        double2 z = cmk(0, 0);
        for (int r = 0; r <= 3; r++) {
            z = cfma(G[(long)r * s2 + ab], bc[r], z);
            z = cfma(G[(long)(ntau - r) * s2 + ab], cscale(cconj(bc[r]), (double)sig), z);
        }
        res[ab] = cscale(cadd(z, cscale(mdft[(long)m1 * s2 + ab], corfac)), dtau);
    }
}

// G = vie2_mat_fourier(F, Q) with pcf oversampling copies (cntr_vie2_impl.hpp:305-455); the DFT
// of F (fdft) is given, the DFT of Q is computed into qdft.
template <int S>
__device__ void vie2_mat_fourier_dev(double2 *G, const double2 *F, const double2 *Q, const double2 *fdft, double2 *qdft,
                                     double2 *Z, double2 *qmasy, int ntau, int sig, double beta, int pcf,
                                     const double2 *tw) {
    constexpr int s2 = S * S;
    const int one = sig == -1 ? 1 : 0, m2 = ntau / 2, NQ = 2 * ntau;
    const double pi = 3.14159265358979323846, dtau = beta / ntau;
    if (threadIdx.x < s2) {
        const int ab = threadIdx.x;
        qmasy[ab] = cadd(cneg(Q[ab]), cscale(Q[(long)ntau * s2 + ab], (double)sig));
    }
    mat_dft_dev<S>(qdft, Q, ntau, one, tw);
    __syncthreads();
    // Z[q] = sum over (p, m) with (2(m + p ntau) + one) = q (mod 2 ntau) of z1(m + p ntau)
    for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
        double2 acc[s2];
        for (int ab = 0; ab < s2; ab++) acc[ab] = cmk(0, 0);
        if (((q - one) & 1) == 0) {
            const int mres = ((q - one) / 2) % ntau;  // m + p ntau = mres (mod ntau)
            for (int p = -pcf; p <= pcf; p++) {
                int m_low = 0, m_high = 0;
                if (sig == 1) { m_high = p < 0 ? 0 : 1; m_low = p > 0 ? -1 : 0; }
                const int lo = -m2 - m_low, hi = m2 - 1 + m_high;
                for (int m = lo + ((mres - lo) % ntau + ntau) % ntau; m <= hi; m += ntau) {
                    const int mm = m + p * ntau;
                    const double omn = (2.0 * mm + one) * pi / (ntau * dtau);
                    double2 fi[s2], qi[s2], z3[s2], z1[s2], z2[s2], zinv[s2];
                    mat_ft_dev<S>(fi, mm, F, fdft, ntau, sig, beta, one);
                    mat_ft_dev<S>(qi, mm, Q, qdft, ntau, sig, beta, one);
                    const double2 f3 = (sig == 1 && mm == 0) ? cmk(0, 0) : cmk(0.0, -1.0 / omn);
                    for (int ab = 0; ab < s2; ab++) {
                        z3[ab] = cmul(qmasy[ab], f3);
                        z1[ab] = fi[ab];
                        if (ab / S == ab % S) z1[ab] = cadd(z1[ab], cmk(1, 0));
                    }
                    for (int a = 0; a < S; a++)
                        for (int d = 0; d < S; d++) {
                            double2 t = cmk(0, 0);
                            for (int b = 0; b < S; b++) t = cfma(fi[a * S + b], z3[b * S + d], t);
                            z2[a * S + d] = csub(csub(qi[a * S + d], z3[a * S + d]), t);
                        }
                    small_inverse<S>(z1, zinv);
                    for (int a = 0; a < S; a++)
                        for (int d = 0; d < S; d++) {
                            double2 t = cmk(0, 0);
                            for (int b = 0; b < S; b++) t = cfma(zinv[a * S + b], z2[b * S + d], t);
                            acc[a * S + d] = cfma(cmk(1.0 / beta, 0), t, acc[a * S + d]);
                        }
                }
            }
        }
        for (int ab = 0; ab < s2; ab++) Z[(long)q * s2 + ab] = acc[ab];
    }
    __syncthreads();
    // G(r) = first-order tail + sum_q Z[q] e^{-i pi q r / ntau}
    for (int e = threadIdx.x; e < (ntau + 1) * s2; e += blockDim.x) {
        const int r = e / s2, ab = e % s2;
        double2 x = cscale(qmasy[ab], -0.5);
        if (sig == 1) x = cadd(x, cscale(qmasy[ab], (r * (beta / ntau)) / beta));
        for (int q = one; q < NQ; q += 2) x = cfma(Z[(long)q * s2 + ab], twid(tw, -(long)q * r, ntau), x);
        G[e] = x;
    }
    __syncthreads();
}

// force_matsubara_hermitian (cntr_utilities_impl.hpp:2077-2090): G(tau) = (G(tau) + G(tau)^dagger) / 2
template <int S>
__device__ void force_mat_hermitian_dev(double2 *G, double2 *tmp, int ntau) {
    constexpr int s2 = S * S;
    for (int e = threadIdx.x; e < (ntau + 1) * s2; e += blockDim.x) {
        const int m = e / s2, ab = e % s2, a = ab / S, b = ab % S;
        tmp[e] = cscale(cadd(G[e], cconj(G[(long)m * s2 + b * S + a])), 0.5);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < (ntau + 1) * s2; e += blockDim.x) G[e] = tmp[e];
    __syncthreads();
}

// G^mat by the Fourier method (dyson_mat_fourier_dispatch, cntr_dyson_impl.hpp:356-446):
//   G(tau_r) = first-order tail - 1/2 (+ tau_r / beta for bosons)
//            + (1/beta) sum_{m=-ntau/2}^{ntau/2-1} sum_{p=-10}^{10} z(mm) e^{-i omega_mm tau_r},  mm = m + p ntau,
//   z(mm) = (i omega - x)^{-1} x / (i omega),  x = H(-1) - mu + Sigma(i omega_mm)
//   (bosons at mm = 0: z = -x^{-1}); Sigma(i omega) = matsubara_ft with cubic endpoint corrections.
// The sum over (m, p) is taken per phase class q = (2 mm + one) mod 2 ntau as in vie2_mat_fourier_dev.
// hj = H(-1) - mu (shared, s^2), sdft = DFT of Sigma^mat (mat_dft_dev).
template <int S>
__device__ void dyson_mat_fourier_dev(double2 *G, const double2 *Sig, const double2 *sdft, const double2 *hj,
                                      double2 *Z, int ntau, int sig, double beta, const double2 *tw) {
    constexpr int s2 = S * S;
    const int one = sig == -1 ? 1 : 0, m2 = ntau / 2, NQ = 2 * ntau, pcf = 10;
    const double pi = 3.14159265358979323846, dtau = beta / ntau;
    for (int q = threadIdx.x; q < NQ; q += blockDim.x) {
        double2 acc[s2];
        for (int ab = 0; ab < s2; ab++) acc[ab] = cmk(0, 0);
        if (((q - one) & 1) == 0) {
            const int mres = ((q - one) / 2) % ntau;  // m + p ntau = mres (mod ntau)
            const int lo = -m2, hi = m2 - 1;
            for (int p = -pcf; p <= pcf; p++) {
                for (int m = lo + ((mres - lo) % ntau + ntau) % ntau; m <= hi; m += ntau) {
                    const int mm = m + p * ntau;
                    const double omn = (2.0 * mm + one) * pi / (ntau * dtau);
                    double2 x[s2], y[s2], yinv[s2];
                    mat_ft_dev<S>(x, mm, Sig, sdft, ntau, sig, beta, one);
                    for (int ab = 0; ab < s2; ab++) x[ab] = cadd(x[ab], hj[ab]);
                    if (sig == 1 && mm == 0) {
                        small_inverse<S>(x, yinv);
                        for (int ab = 0; ab < s2; ab++) acc[ab] = cfma(cmk(-1.0 / beta, 0), yinv[ab], acc[ab]);
                    } else {
                        for (int ab = 0; ab < s2; ab++) y[ab] = cneg(x[ab]);
                        for (int a = 0; a < S; a++) y[a * S + a] = cadd(y[a * S + a], cmk(0, omn));
                        small_inverse<S>(y, yinv);
                        // (1/beta) (1/(i omega)) yinv x
                        const double2 f = cmk(0.0, -1.0 / (omn * beta));
                        for (int a = 0; a < S; a++)
                            for (int d = 0; d < S; d++) {
                                double2 t = cmk(0, 0);
                                for (int b = 0; b < S; b++) t = cfma(yinv[a * S + b], x[b * S + d], t);
                                acc[a * S + d] = cfma(f, t, acc[a * S + d]);
                            }
                    }
                }
            }
        }
        for (int ab = 0; ab < s2; ab++) Z[(long)q * s2 + ab] = acc[ab];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < (ntau + 1) * s2; e += blockDim.x) {
        const int r = e / s2, ab = e % s2;
        const bool diag = ab / S == ab % S;
        double2 v = cmk(diag ? -0.5 : 0.0, 0);
        if (sig == 1 && diag) v = cadd(v, cmk((r * dtau) / beta, 0));
        for (int q = one; q < NQ; q += 2) v = cfma(Z[(long)q * s2 + ab], twid(tw, -(long)q * r, ntau), v);
        G[e] = v;
    }
    __syncthreads();
}

// <X, Y> = sum_r w_r sum_ab Re (X(r)^dagger Y(r))_ab, w_r the Gregory omega at both ends of the tau
// grid (the inner product of vie2_mat_steep_dispatch, cntr_vie2_impl.hpp:519-533); a fixed-order
// tree over the CTA's threads (red: blockDim.x doubles, a power of two); every thread gets the sum.
template <int S>
__device__ double mat_dot_dev(const double2 *X, const double2 *Y, int ntau, int k, double *red) {
    constexpr int s2 = S * S;
    double acc = 0.0;
    for (int r = threadIdx.x; r <= ntau; r += blockDim.x) {
        const double w = r <= k ? greg_omega(k, r) : (r >= ntau - k ? greg_omega(k, ntau - r) : 1.0);
        const double2 *x = X + (long)r * s2, *y = Y + (long)r * s2;
        double t = 0.0;
        for (int a = 0; a < S; a++)
            for (int b = 0; b < S; b++)
                for (int l = 0; l < S; l++) t += x[l * S + a].x * y[l * S + b].x + x[l * S + a].y * y[l * S + b].y;
        acc += w * t;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    const double v = red[0];
    __syncthreads();
    return v;
}

// vie2_mat by steepest descent (vie2_mat_steep_dispatch, cntr_vie2_impl.hpp:486-600): a Fourier
// solve with 3 oversampling copies as the start, then conjugate-gradient iterations on
// A X = X + (F*X + X*Fcc)/2, at most maxiter, until sqrt(<R, R>) < tol (none when <R, R> <= tol).
// fdft holds the DFT of F; qdft, Z the Fourier scratch; R, P, AP, T are (ntau+1) s^2 buffers
// (T may overlap Z: it is used after the Fourier solve).
template <int S>
__device__ void vie2_mat_steep_dev(double2 *G, const double2 *F, const double2 *Fcc, const double2 *Q,
                                   const double2 *fdft, double2 *qdft, double2 *Z, double2 *qmasy, double2 *R,
                                   double2 *P, double2 *AP, double2 *T, double *red, int k, int ntau, int sig,
                                   double beta, int maxiter, double tol, const double2 *tw) {
    constexpr int s2 = S * S;
    const int n = (ntau + 1) * s2;
    const double dtau = beta / ntau;
    vie2_mat_fourier_dev<S>(G, F, Q, fdft, qdft, Z, qmasy, ntau, sig, beta, 3, tw);
    if (maxiter <= 0) return;
    conv_mat_dev<S>(AP, F, G, k, ntau, sig, dtau);
    conv_mat_dev<S>(T, G, Fcc, k, ntau, sig, dtau);
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const double2 x = cneg(csub(cadd(cscale(cadd(AP[e], T[e]), 0.5), G[e]), Q[e]));
        R[e] = x;
        P[e] = x;
    }
    __syncthreads();
    double rsold = mat_dot_dev<S>(R, R, ntau, k, red);
    if (rsold <= tol) return;
    for (int iter = 0; iter < maxiter; iter++) {
        conv_mat_dev<S>(AP, F, P, k, ntau, sig, dtau);
        conv_mat_dev<S>(T, P, Fcc, k, ntau, sig, dtau);
        __syncthreads();
        for (int e = threadIdx.x; e < n; e += blockDim.x) AP[e] = cadd(cscale(cadd(AP[e], T[e]), 0.5), P[e]);
        __syncthreads();
        const double alpha = rsold / mat_dot_dev<S>(P, AP, ntau, k, red);
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            G[e] = cadd(G[e], cscale(P[e], alpha));
            R[e] = csub(R[e], cscale(AP[e], alpha));
        }
        __syncthreads();
        const double rsnew = mat_dot_dev<S>(R, R, ntau, k, red);
        for (int e = threadIdx.x; e < n; e += blockDim.x) P[e] = cadd(R[e], cscale(P[e], rsnew / rsold));
        __syncthreads();
        rsold = rsnew;
        if (sqrt(rsold) < tol) break;
    }
}

// Body of dyson_mat for one problem (one CTA): reads g.smat, g.k, g.ntau, g.sig, g.beta and
// p.H, p.mu; writes p.gmat; uses the scratch vectors of w.  method: 0 = Fourier
// (dyson_mat_fourier_dispatch), 1 = steepest descent (dyson_mat_steep_dispatch, cntr_dyson_impl.hpp:
// 519-540: F = -G0*Sigma, Fcc = -Sigma*G0, 40 iterations, tol 1e-12), 2 = fixpoint (the default);
// force_herm: force_matsubara_hermitian.
template <int S>
__device__ void dyson_mat_body(const GroupDev &g, const ProbDev &p, const MatScratch &w, int method = 2,
                               int force_herm = 1) {
    constexpr int s2 = S * S;
    __shared__ double ev[S];
    __shared__ double2 V[S * S], qmasy[S * S];
    extern __shared__ double2 tw[];  // 2 ntau twiddles e^{i pi q / ntau}
    const int k = g.k, ntau = g.ntau, M = ntau + 1, sig = g.sig;
    const double beta = g.beta, dtau = beta / ntau;
    for (int q = threadIdx.x; q < 2 * ntau; q += blockDim.x) {
        double sn, cs;
        sincospi((double)q / (double)ntau, &sn, &cs);
        tw[q] = cmk(cs, sn);
    }
    if (method == 0) {
        __shared__ double2 hj[S * S];
        if (threadIdx.x < s2) hj[threadIdx.x] = csub(p.H[threadIdx.x], cmk(threadIdx.x / S == threadIdx.x % S ? p.mu : 0.0, 0));
        __syncthreads();
        mat_dft_dev<S>(w.fdft, g.smat, ntau, sig == -1 ? 1 : 0, tw);
        __syncthreads();
        dyson_mat_fourier_dev<S>(p.gmat, g.smat, w.fdft, hj, w.Z, ntau, sig, beta, tw);
        if (force_herm) force_mat_hermitian_dev<S>(p.gmat, w.dG, ntau);
        return;
    }
    // G0 = green_from_H(H(-1), mu): G0(tau) = -V fexp(tau, e) V^dag (fermions), V bexp V^dag (bosons)
    if (threadIdx.x == 0) {
        double2 Hmu[S * S];
        for (int i = 0; i < s2; i++) Hmu[i] = cneg(p.H[i]);
        for (int i = 0; i < S; i++) Hmu[i * S + i] = cadd(Hmu[i * S + i], cmk(p.mu, 0));
        double e_[S];
        double2 V_[S * S];
        herm_eig_dev<S>(Hmu, e_, V_);
        for (int i = 0; i < S; i++) ev[i] = e_[i];
        for (int i = 0; i < s2; i++) V[i] = V_[i];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < M * s2; e += blockDim.x) {
        const int m = e / s2, ab = e % s2, a = ab / S, b = ab % S;
        const double tau = m * dtau;
        double2 v = cmk(0, 0);
        for (int l = 0; l < S; l++) {
            const double f = sig == -1 ? -d_fermi_exp(beta, tau, ev[l]) : d_bose_exp(beta, tau, ev[l]);
            v = cfma(cscale(V[a * S + l], f), cconj(V[b * S + l]), v);
        }
        w.G0[e] = v;
    }
    __syncthreads();
    // F = -G0 * Sigma^mat
    conv_mat_dev<S>(w.F, w.G0, g.smat, k, ntau, sig, dtau);
    __syncthreads();
    for (int e = threadIdx.x; e < M * s2; e += blockDim.x) w.F[e] = cneg(w.F[e]);
    __syncthreads();
    mat_dft_dev<S>(w.fdft, w.F, ntau, sig == -1 ? 1 : 0, tw);
    __syncthreads();
    if (method == 1) {
        __shared__ double red[256];  // blockDim.x = 256
        // Fcc = -Sigma * G0 into Q (unused by the Fourier start); after the start the Fourier
        // buffers hold the iteration: R = dG, P = fdft, AP = qdft, T = Z
        conv_mat_dev<S>(w.Q, g.smat, w.G0, k, ntau, sig, dtau);
        __syncthreads();
        for (int e = threadIdx.x; e < M * s2; e += blockDim.x) w.Q[e] = cneg(w.Q[e]);
        __syncthreads();
        vie2_mat_steep_dev<S>(p.gmat, w.F, w.Q, w.G0, w.fdft, w.qdft, w.Z, qmasy, w.dG, w.fdft, w.qdft, w.Z, red, k,
                              ntau, sig, beta, 40, 1.0e-12, tw);
        if (force_herm) force_mat_hermitian_dev<S>(p.gmat, w.dG, ntau);
        return;
    }
    const int pcf = 5;
    vie2_mat_fourier_dev<S>(p.gmat, w.F, w.G0, w.fdft, w.qdft, w.Z, qmasy, ntau, sig, beta, pcf, tw);
    for (int it = 0; it < 6; it++) {
        conv_mat_dev<S>(w.Q, w.F, p.gmat, k, ntau, sig, dtau);
        __syncthreads();
        for (int e = threadIdx.x; e < M * s2; e += blockDim.x) w.Q[e] = csub(cadd(w.Q[e], p.gmat[e]), w.G0[e]);
        __syncthreads();
        vie2_mat_fourier_dev<S>(w.dG, w.F, w.Q, w.fdft, w.qdft, w.Z, qmasy, ntau, sig, beta, pcf, tw);
        for (int e = threadIdx.x; e < M * s2; e += blockDim.x) p.gmat[e] = csub(p.gmat[e], w.dG[e]);
        __syncthreads();
    }
    if (force_herm) force_mat_hermitian_dev<S>(p.gmat, w.dG, ntau);
}

template <int S>
__global__ void __launch_bounds__(256) k_dyson_mat(GroupDev g, const ProbDev *__restrict__ probs, MatScratch *scr,
                                                   int method, int force_herm) {
    dyson_mat_body<S>(g, probs[blockIdx.x], scr[blockIdx.x], method, force_herm);
}

// vie2_mat on the device (cntr::vie2_mat with the default fixpoint method, cntr_vie2_impl.hpp:
// 460-484, 1091-1160): G^mat = vie2_mat_fourier(F, Q) (:305-455), then 6 corrections
// G -= fourier(F, F*G + G - Q).  F^mat is the group's (g.smat), Q^mat of the problem is in w.G0.
// One CTA per problem.
// method 0: the Fourier solve alone with 20 oversampling copies (vie2_mat_fourier, :1280-1336);
// method 1: steepest descent (vie2_mat_steep, :486-600, 1241-1244: 40 iterations, tol 1e-12) with
// the group's Fcc^mat.
template <int S>
__global__ void __launch_bounds__(256) k_vie2_mat(GroupDev g, const ProbDev *__restrict__ probs, MatScratch *scr,
                                                  int method) {
    constexpr int s2 = S * S;
    __shared__ double2 qmasy[S * S];
    extern __shared__ double2 tw[];  // 2 ntau twiddles e^{i pi q / ntau}
    const ProbDev p = probs[blockIdx.x];
    const MatScratch w = scr[blockIdx.x];
    const int k = g.k, ntau = g.ntau, M = ntau + 1, sig = g.sig;
    const double beta = g.beta, dtau = beta / ntau;
    for (int q = threadIdx.x; q < 2 * ntau; q += blockDim.x) {
        double sn, cs;
        sincospi((double)q / (double)ntau, &sn, &cs);
        tw[q] = cmk(cs, sn);
    }
    __syncthreads();
    mat_dft_dev<S>(w.fdft, g.smat, ntau, sig == -1 ? 1 : 0, tw);
    __syncthreads();
    if (method == 0) {
        vie2_mat_fourier_dev<S>(p.gmat, g.smat, w.G0, w.fdft, w.qdft, w.Z, qmasy, ntau, sig, beta, 20, tw);
        return;
    }
    if (method == 1) {
        __shared__ double red[256];  // blockDim.x = 256
        // after the Fourier start the Fourier buffers hold the iteration: R = dG, P = fdft, AP = qdft, T = Z
        vie2_mat_steep_dev<S>(p.gmat, g.smat, g.fccmat, w.G0, w.fdft, w.qdft, w.Z, qmasy, w.dG, w.fdft, w.qdft, w.Z,
                              red, k, ntau, sig, beta, 40, 1.0e-12, tw);
        return;
    }
    const int pcf = 5;
    vie2_mat_fourier_dev<S>(p.gmat, g.smat, w.G0, w.fdft, w.qdft, w.Z, qmasy, ntau, sig, beta, pcf, tw);
    for (int it = 0; it < 6; it++) {
        conv_mat_dev<S>(w.Q, g.smat, p.gmat, k, ntau, sig, dtau);
        __syncthreads();
        for (int e = threadIdx.x; e < M * s2; e += blockDim.x) w.Q[e] = csub(cadd(w.Q[e], p.gmat[e]), w.G0[e]);
        __syncthreads();
        vie2_mat_fourier_dev<S>(w.dG, g.smat, w.Q, w.fdft, w.qdft, w.Z, qmasy, ntau, sig, beta, pcf, tw);
        for (int e = threadIdx.x; e < M * s2; e += blockDim.x) p.gmat[e] = csub(p.gmat[e], w.dG[e]);
        __syncthreads();
    }
}
