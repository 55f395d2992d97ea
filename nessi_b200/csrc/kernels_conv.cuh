// cntr::convolution_timestep on device-resident herm_matrix data (libcntr
// cntr_convolution_impl.hpp:594-1803): C(n) = [A * B](n) for independent problems, each with its
// own C, A, Acc, B, Bcc in libcntr's layout (tv as ((t M + tau) s^2 + e)).  One launch covers up
// to NESSI_CONV_MAXP problems whose pointers travel in the kernel parameters, so a call needs no
// device allocation.
//   k_conv_ret   C^R(n, j)                 convolution_timestep_ret      (:741-899)
//   k_conv_tv    C^tv(n, tau)              convolution_timestep_tv       (:901-1073)
//   k_conv_les   C^<(j, n)                 convolution_timestep_les_*    (:1075-1580)
//   k_conv_mat   C^mat(tau)                convolution_matsubara         (:560-605)
// Thread per output element (j or tau, then the s x s entry); work items of a problem are
// spread over blockIdx.x, problems over blockIdx.y.
#pragma once
#include "device_common.cuh"

#define NESSI_CONV_MAXP 24  // 24 x 160 B of pointers keeps the parameters under 4 KB

struct ConvHM {
    double2 *ret, *les, *tv, *mat;
};
struct ConvProb {
    ConvHM C, A, Acc, B, Bcc;
};
struct ConvBatch {
    ConvProb p[NESSI_CONV_MAXP];
    int count, ntau, sig_a, sig_b, k;
    double h, beta;
};

__device__ __forceinline__ long ctri(long t) { return t * (t + 1) / 2; }

// element [a][b] of the s x s product X Y
template <int S>
__device__ __forceinline__ double2 emul(const double2 *X, const double2 *Y, int a, int b) {
    double2 t = cmk(0, 0);
#pragma unroll
    for (int c = 0; c < S; c++) t = cfma(X[a * S + c], Y[c * S + b], t);
    return t;
}
// element [a][b] of X Y^dagger
template <int S>
__device__ __forceinline__ double2 emul_ad(const double2 *X, const double2 *Y, int a, int b) {
    double2 t = cmk(0, 0);
#pragma unroll
    for (int c = 0; c < S; c++) t = cfma(X[a * S + c], cconj(Y[b * S + c]), t);
    return t;
}
// element [a][b] of X^dagger Y
template <int S>
__device__ __forceinline__ double2 emul_da(const double2 *X, const double2 *Y, int a, int b) {
    double2 t = cmk(0, 0);
#pragma unroll
    for (int c = 0; c < S; c++) t = cfma(cconj(X[c * S + a]), Y[c * S + b], t);
    return t;
}

// matsubara_integral_2 (conv_impl :410-540), element [a][d]: C(m) = c2 + sig c1 with
//   c1 = int_0^tau A(tau - x) B(beta - x) ..., c2 = int A(tau + x) B(x)  (rcorr near the ends)
// A and B are s x s blocks at A + t s^2 (t = 0..ntau).
template <int S>
__device__ double2 mat_int2(const double2 *A, const double2 *B, int m, int ntau, int k, double sg, int a, int d) {
    constexpr int s2 = S * S;
    double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
    if (m == 0) {
    } else if (m < k) {
        for (int jj = 0; jj <= k; jj++)
            for (int l = 0; l <= k; l++)
                c1 = cfma(cmk(rcorr_w(k, m, l, jj), 0), emul<S>(A + jj * s2, B + (long)(ntau - l) * s2, a, d), c1);
    } else {
        for (int l = 0; l <= m; l++)
            c1 = cfma(cmk(greg_w(k, m, l), 0), emul<S>(A + (long)(m - l) * s2, B + (long)(ntau - l) * s2, a, d), c1);
    }
    const int r = ntau - m;
    if (r == 0) {
    } else if (r < k) {
        for (int l = 0; l <= k; l++)
            for (int jj = 0; jj <= k; jj++)
                c2 = cfma(cmk(rcorr_w(k, r, l, jj), 0), emul<S>(A + (long)(ntau - l) * s2, B + jj * s2, a, d), c2);
    } else {
        for (int l = 0; l <= r; l++)
            c2 = cfma(cmk(greg_w(k, r, l), 0), emul<S>(A + (long)(m + l) * s2, B + (long)l * s2, a, d), c2);
    }
    return cadd(c2, cscale(c1, sg));
}

// matsubara_integral_1 (conv_impl :86-224), element [a][d]: C(m) = c1 + sig c2 with
//   c1 = int_0^tau A(tau - x) B(x), c2 = int_tau^beta A(beta + tau - x) B(x)
template <int S>
__device__ double2 mat_int1(const double2 *A, const double2 *B, int m, int ntau, int k, double sg, int a, int d) {
    constexpr int s2 = S * S;
    double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
    if (m >= k) {
        for (int j = 0; j <= m; j++)
            c1 = cfma(cmk(greg_w(k, m, j), 0), emul<S>(A + (long)(m - j) * s2, B + (long)j * s2, a, d), c1);
    } else if (m > 0) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                c1 = cfma(cmk(rcorr_w(k, m, l, j), 0), emul<S>(A + (long)l * s2, B + (long)j * s2, a, d), c1);
    }
    const int r = ntau - m;
    if (r >= k) {
        for (int j = m; j <= ntau; j++)
            c2 = cfma(cmk(greg_w(k, r, ntau - j), 0), emul<S>(A + (long)(ntau - j + m) * s2, B + (long)j * s2, a, d), c2);
    } else if (r > 0) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                c2 = cfma(cmk(rcorr_w(k, r, l, j), 0),
                          emul<S>(A + (long)(ntau - l) * s2, B + (long)(ntau - j) * s2, a, d), c2);
    }
    return cadd(c1, cscale(c2, sg));
}

// ---------------------------------------------------------------------------------------
// k_conv_ret: C^R(n,j) = h sum_m W(j,m) A^R(n,m) B^R(m,j) (convolution_timestep_ret, :741-899).
//   n >= k: m = j..n with W = gregory_weights(n-j, n-m) for m - j <= k, else 1 (m < n-k) or
//           omega(n-m); for j > n-k also m = n-k..j-1 with B^R(m,j) = -Bcc^R(j,m)^dagger.
//   n < k:  m = 0..k with polynomial weights poly_integration(j, n, m) and the continuations
//           A^R(n,m) = -Acc^R(m,n)^dagger (m > n), B^R(m,j) = -Bcc^R(j,m)^dagger (m < j).
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_conv_ret(ConvBatch cb, int n) {
    constexpr int s2 = S * S;
    const ConvProb &P = cb.p[blockIdx.y];
    const int k = cb.k;
    const double h = cb.h;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)(n + 1) * s2; e += (long)gridDim.x * blockDim.x) {
        const int j = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        double2 acc = cmk(0, 0);
        if (n >= k) {
            for (int m = n; m >= j; m--) {
                double w;
                if (m - j <= k) w = greg_w(k, n - j, n - m);
                else w = m < n - k ? 1.0 : greg_omega(k, n - m);
                acc = cfma(cmk(w, 0), emul<S>(P.A.ret + (ctri(n) + m) * s2, P.B.ret + (ctri(m) + j) * s2, a, b), acc);
            }
            for (int m = (n - k > 0 ? n - k : 0); m < j; m++) {
                const double w = greg_w(k, n - j, n - m);
                acc = cfma(cmk(-w, 0), emul_ad<S>(P.A.ret + (ctri(n) + m) * s2, P.Bcc.ret + (ctri(j) + m) * s2, a, b),
                           acc);
            }
        } else {
            for (int m = 0; m <= k; m++) {
                double w = poly_int(k, j, n, m);
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) {
                    double2 av = n >= m ? P.A.ret[(ctri(n) + m) * s2 + a * S + c] : cconj(P.Acc.ret[(ctri(m) + n) * s2 + c * S + a]);
                    double2 bv = m >= j ? P.B.ret[(ctri(m) + j) * s2 + c * S + b] : cconj(P.Bcc.ret[(ctri(j) + m) * s2 + b * S + c]);
                    t = cfma(av, bv, t);
                }
                if (n < m) w = -w;
                if (m < j) w = -w;
                acc = cfma(cmk(w, 0), t, acc);
            }
        }
        P.C.ret[(ctri(n) + j) * s2 + ab] = cscale(acc, h);
    }
}

// ---------------------------------------------------------------------------------------
// k_conv_tv: C^tv(n,tau) = dtau matsubara_integral_2(A^tv(n,.), B^mat)(tau)
//                        + h sum_{j=0}^{max(n,k)} w(n,j) A'(n,j) B^tv(j,tau)   (:901-1073)
// with A'(n,j) = A^R(n,j) (j <= n) or -Acc^R(j,n)^dagger.
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_conv_tv(ConvBatch cb, int n) {
    constexpr int s2 = S * S;
    const ConvProb &P = cb.p[blockIdx.y];
    const int k = cb.k, ntau = cb.ntau, M = ntau + 1, n1 = n > k ? n : k;
    const double h = cb.h, dtau = cb.beta / ntau;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)M * s2; e += (long)gridDim.x * blockDim.x) {
        const int m = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        double2 acc = cscale(mat_int2<S>(P.A.tv + (long)n * M * s2, P.B.mat, m, ntau, k, (double)cb.sig_b, a, b), dtau);
        for (int j = 0; j <= n1; j++) {
            const double w = h * greg_w(k, n, j);
            const double2 *bt = P.B.tv + ((long)j * M + m) * s2;
            double2 t;
            if (j <= n) t = emul<S>(P.A.ret + (ctri(n) + j) * s2, bt, a, b);
            else t = cneg(emul_da<S>(P.Acc.ret + (ctri(j) + n) * s2, bt, a, b));
            acc = cfma(cmk(w, 0), t, acc);
        }
        P.C.tv[((long)n * M + m) * s2 + ab] = acc;
    }
}

// ---------------------------------------------------------------------------------------
// k_conv_les: C^<(j,n), j = 0..n (convolution_timestep_les, :1525-1580) as the sum of
//   tv*vt   sum_m w(ntau,m) A^tv(j,m) (-i dtau)(-sig_A) Bcc^tv(n,ntau-m)^dagger      (:1075-1242)
//   les*adv sum_m L(j,m) badv(m), L = A^< or -Acc^<(m,j)^dagger (m < j),
//           badv(m) = h w(n,m) Bcc^R(n,m)^dagger (m <= n) or -h w(n,m) B^R(m,n)       (:1244-1394)
//   ret*les sum_{m<=j} w(j,m) A^R(j,m) bl(m) [- sum_{m=j+1}^{k} w(j,m) Acc^R(m,j)^dagger bl(m), j < k],
//           bl(m) = h B^<(m,n) (m <= n) or -h Bcc^<(n,m)^dagger                        (:1396-1523)
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_conv_les(ConvBatch cb, int n) {
    constexpr int s2 = S * S;
    const ConvProb &P = cb.p[blockIdx.y];
    const int k = cb.k, ntau = cb.ntau, M = ntau + 1, n1 = n > k ? n : k;
    const double h = cb.h, dtau = cb.beta / ntau;
    const double2 fvt = cmk(0.0, dtau * (double)cb.sig_a);  // (-i dtau)(-sig_A)
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)(n + 1) * s2; e += (long)gridDim.x * blockDim.x) {
        const int j = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        double2 acc = cmk(0, 0);
        // tv*vt
        for (int m = 0; m <= ntau; m++) {
            const double2 t = emul_ad<S>(P.A.tv + ((long)j * M + m) * s2, P.Bcc.tv + ((long)n * M + ntau - m) * s2, a, b);
            acc = cfma(cmul(fvt, cmk(greg_w(k, ntau, m), 0)), t, acc);
        }
        // les*adv
        for (int m = 0; m <= n1; m++) {
            const double w = h * greg_w(k, n, m);
            double2 t = cmk(0, 0);
            for (int c = 0; c < S; c++) {
                double2 lv = m >= j ? P.A.les[(ctri(m) + j) * s2 + a * S + c] : cneg(cconj(P.Acc.les[(ctri(j) + m) * s2 + c * S + a]));
                double2 bv = m <= n ? cscale(cconj(P.Bcc.ret[(ctri(n) + m) * s2 + b * S + c]), w)
                                    : cscale(P.B.ret[(ctri(m) + n) * s2 + c * S + b], -w);
                t = cfma(lv, bv, t);
            }
            acc = cadd(acc, t);
        }
        // ret*les
        for (int m = 0; m <= j; m++) {
            const double w = h * greg_w(k, j, m);
            acc = cfma(cmk(w, 0), emul<S>(P.A.ret + (ctri(j) + m) * s2, P.B.les + (ctri(n) + m) * s2, a, b), acc);
        }
        if (j < k)
            for (int m = j + 1; m <= k; m++) {
                const double w = h * greg_w(k, j, m);
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) {
                    double2 av = cconj(P.Acc.ret[(ctri(m) + j) * s2 + c * S + a]);
                    double2 bv = m <= n ? P.B.les[(ctri(n) + m) * s2 + c * S + b] : cneg(cconj(P.Bcc.les[(ctri(m) + n) * s2 + b * S + c]));
                    t = cfma(av, bv, t);
                }
                acc = cfma(cmk(-w, 0), t, acc);
            }
        P.C.les[(ctri(n) + j) * s2 + ab] = acc;
    }
}

// k_conv_mat: C^mat(tau) = dtau matsubara_integral_1(A^mat, B^mat)(tau), sig of A (:560-582)
template <int S>
__global__ void k_conv_mat(ConvBatch cb) {
    constexpr int s2 = S * S;
    const ConvProb &P = cb.p[blockIdx.y];
    const int k = cb.k, ntau = cb.ntau, M = ntau + 1;
    const double dtau = cb.beta / ntau;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)M * s2; e += (long)gridDim.x * blockDim.x) {
        const int m = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        P.C.mat[(long)m * s2 + ab] = cscale(mat_int1<S>(P.A.mat, P.B.mat, m, ntau, k, (double)cb.sig_a, a, b), dtau);
    }
}
