// dyson_start on the device (libcntr cntr_dyson_impl.hpp:1502-1535): time steps 0..k of G from
// its Matsubara component, one CTA per problem.  Runs once per problem (or per bootstrap
// iteration of a self-consistent driver), in FP64.
//   ret  dyson_start_ret (:258-352): for j = 0..k-1 a (k-j)-block system in the first argument
//   tv   dyson_start_tv  (:747-888): G^tv(0,.) from G^mat, the Matsubara integral for n = 1..k,
//        then one k-block system per tau; the matrix is tau-independent, so all tau are
//        right-hand sides of one factorisation, processed in chunks
//   les  dyson_timestep_les for n = 0..k (:893-1066) with the convolutions evaluated directly
#pragma once

// shared-memory budget of k_dyson_start (double2 units)
#define NESSI_START_SMEM 6144

template <int S>
__global__ void __launch_bounds__(256) k_dyson_start(GroupDev g, const ProbDev *__restrict__ probs) {
    extern __shared__ double2 smem[];
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, s2 = S * S, tid = threadIdx.x, nth = blockDim.x;
    const int ntau = g.ntau, M = ntau + 1;
    const double h = g.h, dtau = g.beta / ntau, sg = (double)g.sig;
    const long rowstride = (long)s2 * M;  // G^tv plane layout: (t*s2 + e)*M + tau
    auto GR = [&](int t, int t1) { return p.gret + (tri(t) + t1) * s2; };
    auto SR = [&](int t, int t1) { return g.sret + (tri(t) + t1) * s2; };
    auto SL = [&](int t, int t1) { return g.sles + (tri(t1) + t) * s2; };  // Sigma^<(t,t1), t <= t1
    auto ST = [&](int t, int tau) { return g.stv + ((long)t * M + tau) * s2; };
    auto GTV = [&](int t, int e, int tau) -> double2 & { return p.gtv[(long)t * rowstride + (long)e * M + tau]; };
    int *ipiv = (int *)(smem + NESSI_START_SMEM - 1);
    int *status = ipiv + 1;

    // ---------------- ret ----------------
    for (int e = tid; e < (k + 1) * s2; e += nth) {
        const int n = e / s2, ab = e % s2;
        GR(n, n)[ab] = (ab / S == ab % S) ? cmk(0.0, -1.0) : cmk(0, 0);
    }
    __syncthreads();
    for (int j = 0; j < k; j++) {
        const int dim = k - j, KS = dim * S;
        double2 *A = smem, *R = A + KS * KS;
        // A[(pr,a),(q,b)] = mm(pr,q)[a][b]; R[(pr,a),c] = qq(pr)[a][c]; pr = n-(j+1), q = l-(j+1)
        for (int e = tid; e < KS * KS + KS * S; e += nth) {
            if (e < KS * KS) {
                const int row = e / KS, col = e % KS, pr = row / S, a = row % S, q = col / S, bb = col % S;
                const int n = pr + j + 1, l = q + j + 1;
                double2 v = cmk(0, 0);
                if (a == bb) v = cmk(0.0, poly_diff(k, n, l) / h);
                if (l == n) {
                    v = csub(v, p.H[(long)(l + 1) * s2 + a * S + bb]);
                    if (a == bb) v = cadd(v, cmk(p.mu, 0.0));
                }
                double w = h * poly_int(k, j, n, l);
                double2 st;
                if (n >= l) st = SR(n, l)[a * S + bb];
                else { st = cconj(SR(l, n)[bb * S + a]); w = -w; }
                A[e] = csub(v, cscale(st, w));
            } else {
                const int e2 = e - KS * KS, row = e2 / S, c = e2 % S, pr = row / S, a = row % S;
                const int n = pr + j + 1;
                double2 q = cmk(0, 0);
                for (int l = 0; l <= j; l++) {
                    // gtemp = -G^R(j,l)^dagger; qq += (-i/h) P(n,l) gtemp + h Pint(j,n,l) Sigma(n,l) gtemp
                    const double2 cw = cmk(0.0, -poly_diff(k, n, l) / h);
                    const double wi = h * poly_int(k, j, n, l);
                    const double2 *gjl = GR(j, l), *snl = SR(n, l);
                    double2 gt_ac = cneg(cconj(gjl[c * S + a]));
                    q = cadd(q, cmul(cw, gt_ac));
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(snl[a * S + bb], cneg(cconj(gjl[c * S + bb])), t);
                    q = cfma(cmk(wi, 0.0), t, q);
                }
                R[e2] = q;
            }
        }
        if (tid == 0) *status = 0;
        __syncthreads();
        cta_solve(A, R, KS, S, ipiv, status);
        for (int e = tid; e < dim * s2; e += nth) {
            const int pr = e / s2, ac = e % s2, a = ac / S, c = ac % S;
            GR(pr + j + 1, j)[ac] = R[(pr * S + a) * S + c];
        }
        __syncthreads();
    }

    // ---------------- tv ----------------
    // G^tv(0,tau) = sig i G^mat(ntau - tau)
    for (int e = tid; e < M * s2; e += nth) {
        const int tau = e / s2, ab = e % s2;
        GTV(0, ab, tau) = cmul(cmk(0.0, sg), p.gmat[(long)(ntau - tau) * s2 + ab]);
    }
    // G^tv(n,tau) = dtau * matsubara_integral_2(Sigma^tv(n,.), G^mat)(tau), n = 1..k
    for (int e = tid; e < k * M * s2; e += nth) {
        const int n = 1 + e / (M * s2), rem = e % (M * s2), m = rem / s2, ac = rem % s2, a = ac / S, d = ac % S;
        const double2 *A = ST(n, 0), *B = p.gmat;
        double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
        if (m == 0) {
        } else if (m < k) {
            for (int jj = 0; jj <= k; jj++)
                for (int l = 0; l <= k; l++) {
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(A[jj * s2 + a * S + bb], B[(ntau - l) * s2 + bb * S + d], t);
                    c1 = cfma(cmk(rcorr_w(k, m, l, jj), 0), t, c1);
                }
        } else {
            for (int l = 0; l <= m; l++) {
                double2 t = cmk(0, 0);
                for (int bb = 0; bb < S; bb++) t = cfma(A[(m - l) * s2 + a * S + bb], B[(ntau - l) * s2 + bb * S + d], t);
                c1 = cfma(cmk(greg_w(k, m, l), 0), t, c1);
            }
        }
        const int r = ntau - m;
        if (r == 0) {
        } else if (r < k) {
            for (int l = 0; l <= k; l++)
                for (int jj = 0; jj <= k; jj++) {
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(A[(ntau - l) * s2 + a * S + bb], B[jj * s2 + bb * S + d], t);
                    c2 = cfma(cmk(rcorr_w(k, r, l, jj), 0), t, c2);
                }
        } else {
            for (int l = 0; l <= r; l++) {
                double2 t = cmk(0, 0);
                for (int bb = 0; bb < S; bb++) t = cfma(A[(m + l) * s2 + a * S + bb], B[l * s2 + bb * S + d], t);
                c2 = cfma(cmk(greg_w(k, r, l), 0), t, c2);
            }
        }
        GTV(n, ac, m) = cscale(cadd(c2, cscale(c1, sg)), dtau);
    }
    __syncthreads();
    // k-block systems: sum_q mm(p,q) G^tv(q+1,tau) = qq(p)(tau), p = n-1
    {
        const int KS = k * S;
        const int TC = (NESSI_START_SMEM - 8 - KS * KS) / (KS * S) > 0 ? (NESSI_START_SMEM - 8 - KS * KS) / (KS * S) : 1;
        double2 *A = smem, *R = A + KS * KS;  // R: KS x (TC*S)
        for (int t0 = 0; t0 < M; t0 += TC) {
            const int tc = M - t0 < TC ? M - t0 : TC, NR = tc * S;
            for (int e = tid; e < KS * KS + KS * NR; e += nth) {
                if (e < KS * KS) {
                    const int row = e / KS, col = e % KS, pr = row / S, a = row % S, q = col / S, bb = col % S;
                    const int n = pr + 1, jj = q + 1;
                    double2 v = cmk(0, 0);
                    if (a == bb) v = cmk(0.0, poly_diff(k, n, jj) / h);
                    if (pr == q) {
                        v = csub(v, p.H[(long)(n + 1) * s2 + a * S + bb]);
                        if (a == bb) v = cadd(v, cmk(p.mu, 0.0));
                    }
                    double2 st;
                    if (n >= jj) st = SR(n, jj)[a * S + bb];
                    else st = cneg(cconj(SR(jj, n)[bb * S + a]));
                    A[e] = csub(v, cscale(st, h * greg_w(k, n, jj)));
                } else {
                    const int e2 = e - KS * KS, row = e2 / NR, col = e2 % NR, pr = row / S, a = row % S;
                    const int tt = col / S, d = col % S, tau = t0 + tt, n = pr + 1;
                    // qq = -(i/h) P(n,0) G^tv(0,tau) + h w(n,0) Sigma^R(n,0) G^tv(0,tau) + [Matsubara part]
                    double2 q = GTV(n, a * S + d, tau);
                    q = csub(q, cmul(cmk(0.0, poly_diff(k, n, 0) / h), GTV(0, a * S + d, tau)));
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(SR(n, 0)[a * S + bb], GTV(0, bb * S + d, tau), t);
                    q = cfma(cmk(h * greg_w(k, n, 0), 0.0), t, q);
                    R[e2] = q;
                }
            }
            if (tid == 0) *status = 0;
            __syncthreads();
            cta_solve(A, R, KS, NR, ipiv, status);
            for (int e = tid; e < KS * NR; e += nth) {
                const int row = e / NR, col = e % NR, pr = row / S, a = row % S, tt = col / S, d = col % S;
                GTV(pr + 1, a * S + d, t0 + tt) = R[e];
            }
            __syncthreads();
        }
    }

    // ---------------- les: dyson_timestep_les for n = 0..k ----------------
    for (int n = 0; n <= k; n++) {
        double2 *gl = smem;                 // gles(j), j = 0..k  ((k+1) s2)
        double2 *badv = gl + (k + 1) * s2;  // (k+1) s2
        double2 *scr = badv + (k + 1) * s2; // start-block workspace
        for (int e = tid; e < (k + 1) * s2; e += nth) {
            const int m = e / s2, cd = e % s2, c = cd / S, d = cd % S;
            const double w = h * greg_w(k, n, m);
            badv[e] = m <= n ? cscale(cconj(GR(n, m)[d * S + c]), w) : cscale(GR(m, n)[cd], -w);
        }
        __syncthreads();
        for (int e = tid; e < (k + 1) * s2; e += nth) {
            const int j = e / s2, ad = e % s2, a = ad / S, d = ad % S;
            double2 v = cmk(0, 0);
            // tv*vt: sum_m w(ntau,m) Sigma^tv(j,m) (-i dtau)(-sig) G^tv(n,ntau-m)^dagger
            for (int m = 0; m <= ntau; m++) {
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) t = cfma(ST(j, m)[a * S + c], cconj(GTV(n, d * S + c, ntau - m)), t);
                v = cfma(cmk(0.0, dtau * sg * greg_w(k, ntau, m)), t, v);
            }
            // les*adv: sum_m L(j,m) badv(m), L(j,m) = Sigma^<(j,m) (j<=m) or -Sigma^<(m,j)^dagger
            for (int m = 0; m <= k; m++) {
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) {
                    double2 l = m >= j ? SL(j, m)[a * S + c] : cneg(cconj(SL(m, j)[c * S + a]));
                    t = cfma(l, badv[m * s2 + c * S + d], t);
                }
                v = cadd(v, t);
            }
            gl[e] = v;
        }
        double2 *xcol = p.gles + tri(n) * s2;  // G^<(0..n, n); start block writes j = 1..k
        // x_0 = -G^tv(n,0)^dagger, kept in a k+1 window in shared memory (j > n are not stored)
        double2 *xw = scr;                     // (k+1) s2
        for (int ad = tid; ad < s2; ad += nth) {
            const int a = ad / S, d = ad % S;
            xw[ad] = cneg(cconj(GTV(n, d * S + a, 0)));
        }
        __syncthreads();
        les_start_block<S>(g, p, n, gl, S, xw, scr + (k + 1) * s2);
        for (int e = tid; e < (n + 1) * s2; e += nth) xcol[e] = xw[e];
        __syncthreads();
    }
}

// vie2_start on the device (libcntr cntr_vie2_impl.hpp:1338-1420): time steps 0..k of G for
// [1 + F] G = Q from G^mat, one CTA per problem, FP64.
//   ret  vie2_start_ret (:215-300): for j = 0..k-1 a (k-j)-block right solve in the first argument
//   tv   vie2_start_tv  (:727-842): G^tv(n,.) = -dtau matsubara_integral_2(F^tv(n,.), G^mat),
//        then one (k+1)-block system per tau (tau-independent matrix, tau chunks as right sides)
//   les  vie2_timestep_les for n = 0..k (:847-990) with the convolutions evaluated directly
template <int S>
__global__ void __launch_bounds__(256) k_vie2_start(GroupDev g, const ProbDev *__restrict__ probs) {
    extern __shared__ double2 smem[];
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, K1 = k + 1, s2 = S * S, tid = threadIdx.x, nth = blockDim.x;
    const int ntau = g.ntau, M = ntau + 1;
    const double h = g.h, dtau = g.beta / ntau, sg = (double)g.sig;
    const long rowstride = (long)s2 * M;
    auto GR = [&](int t, int t1) { return p.gret + (tri(t) + t1) * s2; };
    auto FR = [&](int t, int t1) { return g.sret + (tri(t) + t1) * s2; };    // F^R(t,t1), t >= t1
    auto FCR = [&](int t, int t1) { return g.rret + (tri(t) + t1) * s2; };   // Fcc^R(t,t1)
    auto FL = [&](int t, int t1) { return g.sles + (tri(t1) + t) * s2; };    // F^<(t,t1), t <= t1
    auto FCL = [&](int t, int t1) { return g.lcc + (tri(t1) + t) * s2; };    // Fcc^<(t,t1)
    auto FT = [&](int t, int tau) { return g.stv + ((long)t * M + tau) * s2; };
    auto QR = [&](int t, int t1) { return p.qret + (tri(t) + t1) * s2; };
    auto GTV = [&](int t, int e, int tau) -> double2 & { return p.gtv[(long)t * rowstride + (long)e * M + tau]; };
    int *ipiv = (int *)(smem + NESSI_START_SMEM - 1);
    int *status = ipiv + 1;
    // F'(n,j) = F^R(n,j) for n >= j, -Fcc^R(j,n)^dagger otherwise: element [a][b]
    auto FP = [&](int n, int j, int a, int b) {
        return n >= j ? FR(n, j)[a * S + b] : cneg(cconj(FCR(j, n)[b * S + a]));
    };

    // ---------------- ret ----------------
    for (int e = tid; e < K1 * s2; e += nth) {
        const int n = e / s2, ab = e % s2;
        GR(n, n)[ab] = QR(n, n)[ab];
    }
    __syncthreads();
    for (int j = 0; j < k; j++) {
        const int dim = k - j, KS = dim * S;
        double2 *A = smem, *R = A + KS * KS;
        // A[(pr,a),(q,b)] = mm(pr,q)[a][b]; R[(pr,a),c] = qq(pr)[a][c]; pr = n-(j+1), q = l-(j+1)
        for (int e = tid; e < KS * KS + KS * S; e += nth) {
            if (e < KS * KS) {
                const int row = e / KS, col = e % KS, pr = row / S, a = row % S, q = col / S, bb = col % S;
                const int n = pr + j + 1, l = q + j + 1;
                double2 v = (l == n && a == bb) ? cmk(1.0, 0.0) : cmk(0, 0);
                double w = -h * poly_int(k, j, n, l);
                double2 st;
                if (n >= l) st = FR(n, l)[a * S + bb];
                else { st = cconj(FCR(l, n)[bb * S + a]); w = -w; }
                A[e] = csub(v, cscale(st, w));
            } else {
                const int e2 = e - KS * KS, row = e2 / S, c = e2 % S, pr = row / S, a = row % S;
                const int n = pr + j + 1;
                double2 q = QR(n, j)[a * S + c];
                for (int l = 0; l <= j; l++) {
                    // qq += -h Pint(j,n,l) F^R(n,l) (-G^R(j,l)^dagger)
                    const double2 *gjl = GR(j, l), *fnl = FR(n, l);
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(fnl[a * S + bb], cneg(cconj(gjl[c * S + bb])), t);
                    q = cfma(cmk(-h * poly_int(k, j, n, l), 0.0), t, q);
                }
                R[e2] = q;
            }
        }
        if (tid == 0) *status = 0;
        __syncthreads();
        cta_solve(A, R, KS, S, ipiv, status);
        for (int e = tid; e < dim * s2; e += nth) {
            const int pr = e / s2, ac = e % s2, a = ac / S, c = ac % S;
            GR(pr + j + 1, j)[ac] = R[(pr * S + a) * S + c];
        }
        __syncthreads();
    }

    // ---------------- tv ----------------
    // G^tv(n,tau) = -dtau * matsubara_integral_2(F^tv(n,.), G^mat)(tau), n = 0..k
    for (int e = tid; e < K1 * M * s2; e += nth) {
        const int n = e / (M * s2), rem = e % (M * s2), m = rem / s2, ac = rem % s2, a = ac / S, d = ac % S;
        const double2 *A = FT(n, 0), *B = p.gmat;
        double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
        if (m == 0) {
        } else if (m < k) {
            for (int jj = 0; jj <= k; jj++)
                for (int l = 0; l <= k; l++) {
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(A[jj * s2 + a * S + bb], B[(ntau - l) * s2 + bb * S + d], t);
                    c1 = cfma(cmk(rcorr_w(k, m, l, jj), 0), t, c1);
                }
        } else {
            for (int l = 0; l <= m; l++) {
                double2 t = cmk(0, 0);
                for (int bb = 0; bb < S; bb++) t = cfma(A[(m - l) * s2 + a * S + bb], B[(ntau - l) * s2 + bb * S + d], t);
                c1 = cfma(cmk(greg_w(k, m, l), 0), t, c1);
            }
        }
        const int r = ntau - m;
        if (r == 0) {
        } else if (r < k) {
            for (int l = 0; l <= k; l++)
                for (int jj = 0; jj <= k; jj++) {
                    double2 t = cmk(0, 0);
                    for (int bb = 0; bb < S; bb++) t = cfma(A[(ntau - l) * s2 + a * S + bb], B[jj * s2 + bb * S + d], t);
                    c2 = cfma(cmk(rcorr_w(k, r, l, jj), 0), t, c2);
                }
        } else {
            for (int l = 0; l <= r; l++) {
                double2 t = cmk(0, 0);
                for (int bb = 0; bb < S; bb++) t = cfma(A[(m + l) * s2 + a * S + bb], B[l * s2 + bb * S + d], t);
                c2 = cfma(cmk(greg_w(k, r, l), 0), t, c2);
            }
        }
        GTV(n, ac, m) = cscale(cadd(c2, cscale(c1, sg)), -dtau);
    }
    __syncthreads();
    // (k+1)-block systems: sum_j mm(n,j) G^tv(j,tau) = G^tv(n,tau) + Q^tv(n,tau)
    {
        const int KS = K1 * S;
        const int TC = (NESSI_START_SMEM - 8 - KS * KS) / (KS * S) > 0 ? (NESSI_START_SMEM - 8 - KS * KS) / (KS * S) : 1;
        double2 *A = smem, *R = A + KS * KS;  // R: KS x (TC*S)
        for (int t0 = 0; t0 < M; t0 += TC) {
            const int tc = M - t0 < TC ? M - t0 : TC, NR = tc * S;
            for (int e = tid; e < KS * KS + KS * NR; e += nth) {
                if (e < KS * KS) {
                    const int row = e / KS, col = e % KS, n = row / S, a = row % S, jj = col / S, bb = col % S;
                    double2 v = (n == jj && a == bb) ? cmk(1.0, 0.0) : cmk(0, 0);
                    A[e] = cfma(cmk(h * greg_w(k, n, jj), 0.0), FP(n, jj, a, bb), v);
                } else {
                    const int e2 = e - KS * KS, row = e2 / NR, col = e2 % NR, n = row / S, a = row % S;
                    const int tt = col / S, d = col % S, tau = t0 + tt;
                    R[e2] = cadd(GTV(n, a * S + d, tau), p.qtv[(long)n * rowstride + (long)(a * S + d) * M + tau]);
                }
            }
            if (tid == 0) *status = 0;
            __syncthreads();
            cta_solve(A, R, KS, NR, ipiv, status);
            for (int e = tid; e < KS * NR; e += nth) {
                const int row = e / NR, col = e % NR, n = row / S, a = row % S, tt = col / S, d = col % S;
                GTV(n, a * S + d, t0 + tt) = R[e];
            }
            __syncthreads();
        }
    }

    // ---------------- les: vie2_timestep_les for n = 0..k ----------------
    for (int n = 0; n <= k; n++) {
        double2 *gl = smem;                 // gles(j), j = 0..k  ((k+1) s2)
        double2 *badv = gl + K1 * s2;       // (k+1) s2
        double2 *xw = badv + K1 * s2;       // (k+1) s2 solution window
        double2 *scr = xw + K1 * s2;        // start-block workspace
        for (int e = tid; e < K1 * s2; e += nth) {
            const int m = e / s2, cd = e % s2, c = cd / S, d = cd % S;
            const double w = h * greg_w(k, n, m);
            badv[e] = m <= n ? cscale(cconj(GR(n, m)[d * S + c]), w) : cscale(GR(m, n)[cd], -w);
        }
        __syncthreads();
        for (int e = tid; e < K1 * s2; e += nth) {
            const int j = e / s2, ad = e % s2, a = ad / S, d = ad % S;
            double2 v = cmk(0, 0);
            // tv*vt: sum_m w(ntau,m) F^tv(j,m) (-i dtau)(-sig) G^tv(n,ntau-m)^dagger
            for (int m = 0; m <= ntau; m++) {
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) t = cfma(FT(j, m)[a * S + c], cconj(GTV(n, d * S + c, ntau - m)), t);
                v = cfma(cmk(0.0, dtau * sg * greg_w(k, ntau, m)), t, v);
            }
            // les*adv: sum_m L(j,m) badv(m), L(j,m) = F^<(j,m) (j<=m) or -Fcc^<(m,j)^dagger
            for (int m = 0; m <= k; m++) {
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) {
                    double2 l = m >= j ? FL(j, m)[a * S + c] : cneg(cconj(FCL(m, j)[c * S + a]));
                    t = cfma(l, badv[m * s2 + c * S + d], t);
                }
                v = cadd(v, t);
            }
            gl[e] = cneg(v);
        }
        __syncthreads();
        les_start_block_vie<S>(g, p, n, gl, S, xw, scr);
        double2 *xcol = p.gles + tri(n) * s2;  // G^<(0..n, n)
        for (int e = tid; e < (n + 1) * s2; e += nth) xcol[e] = xw[e];
        __syncthreads();
    }
}
