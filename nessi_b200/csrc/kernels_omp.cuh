// The element-parallel path of libcntr (the routines its OpenMP solvers are built from) on
// device-resident herm_matrix data in libcntr's layout:
//   k_incr_mat/ret/tv/les   incr_convolution_{mat,ret,tv,les}   cntr_convolution_impl.hpp:4164-4760
//   dyson_timestep_omp      cntr_dyson_omp_impl.hpp:37-605: k_omp_ret_start (the k x k start block),
//                           k_incr_ret + k_omp_ret_solve, k_incr_tv + k_omp_tv_solve,
//                           k_incr_les + k_omp_les_solve and k_omp_les_serial (rows n-k..n, or the
//                           serial lesser step for n < 2k+1)
//   vie2_timestep_omp       cntr_vie2_impl.hpp:1851-1980: k_incr_* with Q as the base and
//                           k_omp_vie2_solve
// Where the reference's threads each take every nomp-th output element, here a thread takes one
// element (index, s x s entry) of one problem: problems on blockIdx.y, elements grid-strided
// over blockIdx.x.  Every convolution of a component is complete before its solves (the
// reference's one-thread order); entries of time step tstp that the reference zeroes before a
// convolution reads them are skipped (skip_tstp), so the output may alias an operand.
#pragma once
#include "kernels_conv.cuh"

#define NESSI_OMP_MAXP 16

struct OmpProb {
    ConvHM C, Cin, A, Acc, B, Bcc;  // output, base added to it, operands
    const double2 *f;               // incr: function data F(-1) first, or null
    const double2 *H;               // solvers: H(-1) first, (nt+2) blocks
    double mu;
};
struct OmpBatch {
    OmpProb p[NESSI_OMP_MAXP];
    const unsigned char *mask;  // per output index of the component (null = all)
    double2 alpha;
    int count, ntau, sig_a, sig_b, k;
    int lo, hi;        // output indices [lo, hi) of the component
    int out_mode;      // 0: C += alpha conv, 1: C = Cin + alpha conv, 2: C = alpha conv
    int skip_tstp;     // entries of time step tstp read as zero (see above)
    double h, beta;
};

// element (r, c) of X (mode 0), X^dagger (1), -X^dagger (2), -X (3) for an S x S block X
template <int S>
__device__ __forceinline__ double2 blk(const double2 *X, int mode, int r, int c) {
    switch (mode) {
        case 0: return X[r * S + c];
        case 1: return cconj(X[c * S + r]);
        case 2: return cneg(cconj(X[c * S + r]));
        default: return cneg(X[r * S + c]);
    }
}

// element [a][b] of L' R' with L' = L FL (FL on the right of L) and R' = FR R (FR on the left
// of R); FL / FR null = identity
template <int S>
__device__ double2 term3(const double2 *L, int lm, const double2 *FL, const double2 *R, int rm, const double2 *FR,
                         int a, int b) {
    double2 t = cmk(0, 0);
#pragma unroll
    for (int c = 0; c < S; c++) {
        double2 l, r;
        if (FL) {
            l = cmk(0, 0);
            for (int d = 0; d < S; d++) l = cfma(blk<S>(L, lm, a, d), FL[d * S + c], l);
        } else {
            l = blk<S>(L, lm, a, c);
        }
        if (FR) {
            r = cmk(0, 0);
            for (int d = 0; d < S; d++) r = cfma(FR[c * S + d], blk<S>(R, rm, d, b), r);
        } else {
            r = blk<S>(R, rm, c, b);
        }
        t = cfma(l, r, t);
    }
    return t;
}

// Weight of point j in the reference's three-loop end-corrected sum on 0..N (the incr_* loops:
// omega(j) for j <= k, 1 for k < j < N - k, omega(N - j) for j >= N - k).  For N < 2k+1 the
// first and last loops overlap and the reference adds both terms; so does this.
__device__ __forceinline__ double omega_split(int k, int N, int j) {
    double w = 0.0;
    if (j <= k) w += greg_omega(k, j);
    if (j >= N - k) w += greg_omega(k, N - j);
    if (j > k && j < N - k) w = 1.0;
    return w;
}

// matsubara_integral_1 / _2 (conv_impl :86-224, :410-540) with a middle factor F between the
// two blocks (A(.) F B(.)); F null = identity
template <int S>
__device__ double2 mat_int1_f(const double2 *A, const double2 *F, const double2 *B, int m, int ntau, int k, double sg,
                              int a, int d) {
    constexpr int s2 = S * S;
    double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
    if (m >= k) {
        for (int j = 0; j <= m; j++)
            c1 = cfma(cmk(greg_w(k, m, j), 0), term3<S>(A + (long)(m - j) * s2, 0, F, B + (long)j * s2, 0, nullptr, a, d), c1);
    } else if (m > 0) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                c1 = cfma(cmk(rcorr_w(k, m, l, j), 0), term3<S>(A + (long)l * s2, 0, F, B + (long)j * s2, 0, nullptr, a, d), c1);
    }
    const int r = ntau - m;
    if (r >= k) {
        for (int j = m; j <= ntau; j++)
            c2 = cfma(cmk(greg_w(k, r, ntau - j), 0),
                      term3<S>(A + (long)(ntau - j + m) * s2, 0, F, B + (long)j * s2, 0, nullptr, a, d), c2);
    } else if (r > 0) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                c2 = cfma(cmk(rcorr_w(k, r, l, j), 0),
                          term3<S>(A + (long)(ntau - l) * s2, 0, F, B + (long)(ntau - j) * s2, 0, nullptr, a, d), c2);
    }
    return cadd(c1, cscale(c2, sg));
}
template <int S>
__device__ double2 mat_int2_f(const double2 *A, const double2 *F, const double2 *B, int m, int ntau, int k, double sg,
                              int a, int d) {
    constexpr int s2 = S * S;
    double2 c1 = cmk(0, 0), c2 = cmk(0, 0);
    if (m == 0) {
    } else if (m < k) {
        for (int jj = 0; jj <= k; jj++)
            for (int l = 0; l <= k; l++)
                c1 = cfma(cmk(rcorr_w(k, m, l, jj), 0),
                          term3<S>(A + jj * s2, 0, F, B + (long)(ntau - l) * s2, 0, nullptr, a, d), c1);
    } else {
        for (int l = 0; l <= m; l++)
            c1 = cfma(cmk(greg_w(k, m, l), 0),
                      term3<S>(A + (long)(m - l) * s2, 0, F, B + (long)(ntau - l) * s2, 0, nullptr, a, d), c1);
    }
    const int r = ntau - m;
    if (r == 0) {
    } else if (r < k) {
        for (int l = 0; l <= k; l++)
            for (int jj = 0; jj <= k; jj++)
                c2 = cfma(cmk(rcorr_w(k, r, l, jj), 0),
                          term3<S>(A + (long)(ntau - l) * s2, 0, F, B + jj * s2, 0, nullptr, a, d), c2);
    } else {
        for (int l = 0; l <= r; l++)
            c2 = cfma(cmk(greg_w(k, r, l), 0), term3<S>(A + (long)(m + l) * s2, 0, F, B + (long)l * s2, 0, nullptr, a, d), c2);
    }
    return cadd(c2, cscale(c1, sg));
}

__device__ __forceinline__ bool omp_take(const OmpBatch &ob, int i) { return !ob.mask || ob.mask[i]; }

__device__ __forceinline__ double2 omp_out(const OmpBatch &ob, const double2 *C, const double2 *Cin, long idx, double2 v) {
    if (ob.out_mode == 0) return cadd(C[idx], v);
    if (ob.out_mode == 1) return cadd(Cin[idx], v);
    return v;
}

// ---------------------------------------------------------------------------------------
// incr_convolution_mat (:4164-4200): C^mat(m) += alpha dtau matsubara_integral_1(A^mat, f0 B^mat)(m)
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_incr_mat(OmpBatch ob) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const double2 fac = cscale(ob.alpha, ob.beta / ob.ntau);
    for (long e = (long)ob.lo * s2 + blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)ob.hi * s2;
         e += (long)gridDim.x * blockDim.x) {
        const int m = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        if (!omp_take(ob, m)) continue;
        double2 v = cmul(fac, mat_int1_f<S>(P.A.mat, P.f, P.B.mat, m, ob.ntau, ob.k, (double)ob.sig_a, a, b));
        P.C.mat[(long)m * s2 + ab] = omp_out(ob, P.C.mat, P.Cin.mat, (long)m * s2 + ab, v);
    }
}

// ---------------------------------------------------------------------------------------
// incr_convolution_ret (:4243-4360): C^R(tstp, n) += alpha h sum_j W A'(tstp, j) F(j) B'(j, n)
//   A'(tstp, j) = A^R(tstp, j) (j <= tstp) or -Acc^R(j, tstp)^dagger, B'(j, n) = B^R(j, n)
//   (j >= n) or -Bcc^R(n, j)^dagger; W: polynomial weights (tstp < k), Gregory weights
//   w(tstp - n, l) (tstp - n <= 2k+2), else the omega split on n..tstp.
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_incr_ret(OmpBatch ob, int tstp) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k;
    const double2 *ft = P.f ? P.f + s2 : nullptr;  // F(0)
    const double2 fac = cscale(ob.alpha, ob.h);
    for (long e = (long)ob.lo * s2 + blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)ob.hi * s2;
         e += (long)gridDim.x * blockDim.x) {
        const int n = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        if (!omp_take(ob, n)) continue;
        const int n2 = tstp - n;
        double2 acc = cmk(0, 0);
        auto add = [&](double w, int j) {
            const int brow = j >= n ? j : n;  // the row of B or Bcc this term reads
            if (ob.skip_tstp && brow == tstp) return;
            const double2 *L = j <= tstp ? P.A.ret + (ctri(tstp) + j) * s2 : P.Acc.ret + (ctri(j) + tstp) * s2;
            const double2 *R = j >= n ? P.B.ret + (ctri(j) + n) * s2 : P.Bcc.ret + (ctri(n) + j) * s2;
            acc = cfma(cmk(w, 0), term3<S>(L, j <= tstp ? 0 : 2, ft ? ft + (long)j * s2 : nullptr, R, j >= n ? 0 : 2,
                                           nullptr, a, b), acc);
        };
        if (tstp < k) {
            for (int j = 0; j <= k; j++) add(poly_int(k, n, tstp, j), j);
        } else if (n2 < k) {
            for (int l = 0; l <= k; l++) add(greg_w(k, n2, l), tstp - l);
        } else if (n2 <= 2 * k + 2) {
            for (int l = 0; l <= n2; l++) add(greg_w(k, n2, l), n + l);
        } else {
            for (int j = n; j <= tstp; j++) add(omega_split(k, n2, j - n), j);
        }
        const long idx = (ctri(tstp) + n) * s2 + ab;
        P.C.ret[idx] = omp_out(ob, P.C.ret, P.Cin.ret, idx, cmul(fac, acc));
    }
}

// ---------------------------------------------------------------------------------------
// incr_convolution_tv (:4396-4500): C^tv(tstp, m) += alpha [ dtau mat_int_2(A^tv(tstp, .), f0 B^mat)(m)
//   + h sum_j W(tstp, j) A'(tstp, j) F(j) B^tv(j, m) ], W = w(tstp, j) for tstp <= 2k+2, else
//   the omega split on 0..tstp.
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_incr_tv(OmpBatch ob, int tstp) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k, ntau = ob.ntau, M = ntau + 1, n1 = tstp > k ? tstp : k;
    const double2 *ft = P.f ? P.f + s2 : nullptr;
    const double2 fmat = cscale(ob.alpha, ob.beta / ntau), fret = cscale(ob.alpha, ob.h);
    for (long e = (long)ob.lo * s2 + blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)ob.hi * s2;
         e += (long)gridDim.x * blockDim.x) {
        const int m = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        if (!omp_take(ob, m)) continue;
        double2 c1 = mat_int2_f<S>(P.A.tv + (long)tstp * M * s2, P.f, P.B.mat, m, ntau, k, (double)ob.sig_b, a, b);
        double2 c2 = cmk(0, 0);
        const int jmax = tstp <= 2 * k + 2 ? n1 : tstp;
        for (int j = 0; j <= jmax; j++) {
            if (ob.skip_tstp && j == tstp) continue;
            const double w = tstp <= 2 * k + 2 ? greg_w(k, tstp, j) : omega_split(k, tstp, j);
            const double2 *L = j <= tstp ? P.A.ret + (ctri(tstp) + j) * s2 : P.Acc.ret + (ctri(j) + tstp) * s2;
            c2 = cfma(cmk(w, 0), term3<S>(L, j <= tstp ? 0 : 2, ft ? ft + (long)j * s2 : nullptr,
                                          P.B.tv + ((long)j * M + m) * s2, 0, nullptr, a, b), c2);
        }
        const long idx = ((long)tstp * M + m) * s2 + ab;
        P.C.tv[idx] = omp_out(ob, P.C.tv, P.Cin.tv, idx, cadd(cmul(fmat, c1), cmul(fret, c2)));
    }
}

// ---------------------------------------------------------------------------------------
// incr_convolution_les (:4539-4760): C^<(n, tstp) += alpha [ h c1 + h c3 - i dtau c2 ] with
//   c1 = sum_j W A'(n, j) F(j) B'^<(j, tstp)           (ret * les; Gregory w(n, j) for n <= 2k+2,
//        A'(n, j) = -Acc^R(j, n)^dagger for j > n, B'^< = -Bcc^<(tstp, j)^dagger for j > tstp)
//   c2 = sum_m omega_split(ntau, m) A^tv(n, m) f0 (-sig_B) Bcc^tv(tstp, ntau - m)^dagger  (tv * vt)
//   c3 = sum_j W L(n, j) F(j) B'^A(j, tstp)             (les * adv; B'^A = Bcc^R(tstp, j)^dagger,
//        or -B^R(j, tstp) for j > tstp; L(n, j) = A^<(n, j), or -Acc^<(j, n)^dagger for j <= n
//        when tstp <= 2k+2 and for j < n otherwise)
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_incr_les(OmpBatch ob, int tstp) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k, ntau = ob.ntau, M = ntau + 1, n1 = tstp > k ? tstp : k;
    const double2 *ft = P.f ? P.f + s2 : nullptr;
    const double2 *f0 = P.f;
    const double2 fh = cscale(ob.alpha, ob.h), ftau = cmul(ob.alpha, cmk(0.0, -ob.beta / ntau));
    for (long e = (long)ob.lo * s2 + blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)ob.hi * s2;
         e += (long)gridDim.x * blockDim.x) {
        const int n = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        if (!omp_take(ob, n)) continue;
        // ret * les
        double2 c1 = cmk(0, 0);
        {
            const int nup = n > k ? n : k;
            const bool small = n <= 2 * k + 2;
            const int jmax = small ? nup : n;
            for (int j = 0; j <= jmax; j++) {
                const double w = small ? greg_w(k, n, j) : omega_split(k, n, j);
                const double2 *L = j <= n ? P.A.ret + (ctri(n) + j) * s2 : P.Acc.ret + (ctri(j) + n) * s2;
                const double2 *R = j <= tstp ? P.B.les + (ctri(tstp) + j) * s2 : P.Bcc.les + (ctri(j) + tstp) * s2;
                c1 = cfma(cmk(w, 0), term3<S>(L, j <= n ? 0 : 2, nullptr, R, j <= tstp ? 0 : 2,
                                              ft ? ft + (long)j * s2 : nullptr, a, b), c1);
            }
        }
        // tv * vt
        double2 c2 = cmk(0, 0);
        {
            const int vmode = ob.sig_b == -1 ? 1 : 2;
            for (int m = 0; m <= ntau; m++) {
                const double w = omega_split(k, ntau, m);
                c2 = cfma(cmk(w, 0), term3<S>(P.A.tv + ((long)n * M + m) * s2, 0, nullptr,
                                              P.Bcc.tv + ((long)tstp * M + ntau - m) * s2, vmode, f0, a, b), c2);
            }
        }
        // les * adv
        double2 c3 = cmk(0, 0);
        {
            const bool small = tstp <= 2 * k + 2;
            const int jmax = small ? n1 : tstp;
            for (int j = 0; j <= jmax; j++) {
                if (ob.skip_tstp && j == tstp) continue;  // A^<(n, tstp) or Acc^<(tstp, tstp): zero
                const double w = small ? greg_w(k, tstp, j) : omega_split(k, tstp, j);
                const bool cc = small ? j <= n : j < n;
                const double2 *L = cc ? P.Acc.les + (ctri(n) + j) * s2 : P.A.les + (ctri(j) + n) * s2;
                const double2 *R = j <= tstp ? P.Bcc.ret + (ctri(tstp) + j) * s2 : P.B.ret + (ctri(j) + tstp) * s2;
                c3 = cfma(cmk(w, 0), term3<S>(L, cc ? 2 : 0, nullptr, R, j <= tstp ? 1 : 3,
                                              ft ? ft + (long)j * s2 : nullptr, a, b), c3);
            }
        }
        const long idx = (ctri(tstp) + n) * s2 + ab;
        const double2 v = cadd(cadd(cmul(fh, c1), cmul(fh, c3)), cmul(ftau, c2));
        P.C.les[idx] = omp_out(ob, P.C.les, P.Cin.les, idx, v);
    }
}

// ---------------------------------------------------------------------------------------
// dyson_timestep_omp (cntr_dyson_omp_impl.hpp:37-414).  p.C = p.B = p.Bcc = G, p.A = p.Acc = Sigma.
// ---------------------------------------------------------------------------------------
// Retarded start (:51-129, the serial step's k x k block): row n zeroed, G^R(n, n) = -i, and
// X_q = G^R(n, n-q-1), q = 0..k-1, from sum_q X_q mm(p, q) = qq(p) (a left solve).  One CTA per
// problem; shared memory mm (k^2 s^2), qq (k s^2), the system (kS)^2 + kS S, pivot and status.
template <int S>
__global__ void k_omp_ret_start(OmpBatch ob, int n, int *status_out) {
    constexpr int s2 = S * S;
    extern __shared__ double2 smem[];
    const OmpProb &P = ob.p[blockIdx.x];
    const int k = ob.k, KS = k * S;
    const double h = ob.h;
    double2 *mm = smem, *qq = mm + k * k * s2, *A = qq + k * s2, *R = A + KS * KS;
    int *ipiv = (int *)(R + KS * S), *status = ipiv + 1;
    double2 *grow = P.C.ret + ctri(n) * s2;
    const double2 *sr = P.A.ret;
    for (long e = threadIdx.x; e < (long)(n + 1) * s2; e += blockDim.x) {
        const int ab = (int)(e % s2);
        grow[e] = (e / s2 == n && ab / S == ab % S) ? cmk(0.0, -1.0) : cmk(0, 0);
    }
    for (int e = threadIdx.x; e < k * k * s2; e += blockDim.x) mm[e] = cmk(0, 0);
    if (threadIdx.x == 0) *status = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
        const int pr = e / s2, ab = e % s2, a = ab / S, b = ab % S, j = pr + 1;
        const double2 gnn = a == b ? cmk(0.0, -1.0) : cmk(0, 0);
        double2 q = cneg(cmul(cmk(0.0, poly_diff(k, j, 0) / h), gnn));
        if (a == b)
            for (int l = 1; l <= k; l++) {
                const int idx = (pr * k + l - 1) * s2 + ab;
                mm[idx] = cadd(mm[idx], cmk(0.0, poly_diff(k, j, l) / h));
            }
        {
            double2 v = cneg(P.H[(long)(n - j + 1) * s2 + ab]);
            if (a == b) v = cadd(v, cmk(P.mu, 0.0));
            mm[(pr * k + pr) * s2 + ab] = cadd(mm[(pr * k + pr) * s2 + ab], v);
        }
        for (int l = 0; l <= k; l++) {
            double w = h * greg_w(k, j, l);
            double2 st;
            if (l <= j) st = sr[(ctri(n - l) + (n - j)) * s2 + ab];
            else { st = cconj(sr[(ctri(n - j) + (n - l)) * s2 + b * S + a]); w = -w; }
            if (l == 0) {
                q = cadd(q, cmul(cmk(0.0, -w), st));  // w G(n,n) stemp with G(n,n) = -i 1
            } else {
                const int idx = (pr * k + l - 1) * s2 + ab;
                mm[idx] = csub(mm[idx], cscale(st, w));
            }
        }
        qq[pr * s2 + ab] = q;
    }
    __syncthreads();
    // the left solve as the right solve of the block-wise adjoints
    for (int e = threadIdx.x; e < KS * KS; e += blockDim.x) {
        const int r = e / KS, c = e % KS, pr = r / S, a = r % S, q = c / S, b = c % S;
        A[e] = cconj(mm[(pr * k + q) * s2 + b * S + a]);
    }
    for (int e = threadIdx.x; e < KS * S; e += blockDim.x) {
        const int r = e / S, c = e % S, pr = r / S, a = r % S;
        R[e] = cconj(qq[pr * s2 + c * S + a]);
    }
    __syncthreads();
    cta_solve(A, R, KS, S, ipiv, status);
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
        const int q = e / s2, ac = e % s2, a = ac / S, c = ac % S;
        grow[(long)(n - q - 1) * s2 + ac] = cconj(R[(q * S + c) * S + a]);
    }
    if (threadIdx.x == 0 && *status && status_out) atomicExch(status_out, 1);
}

// X = M^-1 Q (right) or X = Q M^-1 (left) for one S x S block held by one thread
template <int S>
__device__ void omp_block_solve(const double2 *Mm, const double2 *Q, double2 *X, bool left, int *status_out) {
    double2 mi[S * S], q[S * S];
    if (small_inverse<S>(Mm, mi) && status_out) atomicExch(status_out, 1);
    for (int i = 0; i < S * S; i++) q[i] = Q[i];
    for (int a = 0; a < S; a++)
        for (int b = 0; b < S; b++) {
            double2 t = cmk(0, 0);
            for (int c = 0; c < S; c++) t = left ? cfma(q[a * S + c], mi[c * S + b], t) : cfma(mi[a * S + c], q[c * S + b], t);
            X[a * S + b] = t;
        }
}

// G^R(n, j), j in [0, n-k): qq = G^R(n, j) - sum_p d_p G^R(n-p, j) (d_p = i/h bd_p, BD(k+1)),
// [ d_0 + mu - h omega_0 Sigma^R(j, j) - H(n) ] G^R(n, j) = qq   (:160-172)
template <int S>
__global__ void k_omp_ret_solve(OmpBatch ob, int n, int *status_out) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k;
    const double h = ob.h, w0 = h * greg_omega(k, 0);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n - k; j += gridDim.x * blockDim.x) {
        double2 qq[s2], mm[s2];
        double2 *g = P.C.ret + (ctri(n) + j) * s2;
        for (int e = 0; e < s2; e++) {
            double2 q = g[e];
            for (int p = 1; p <= k + 1; p++)
                q = csub(q, cmul(cmk(0.0, bd_w(k, p) / h), P.C.ret[(ctri(n - p) + j) * s2 + e]));
            qq[e] = q;
            double2 m = cneg(P.H[(long)(n + 1) * s2 + e]);
            m = csub(m, cscale(P.A.ret[(ctri(j) + j) * s2 + e], w0));
            if (e / S == e % S) m = cadd(m, cmk(P.mu, bd_w(k, 0) / h));
            mm[e] = m;
        }
        omp_block_solve<S>(mm, qq, g, false, status_out);
    }
}

// G^tv(n, m): qq = G^tv(n, m) - sum_p d_p G^tv(n-p, m),
// [ d_0 + mu - H(n) - h w(n, 0) Sigma^R(n, n) ] G^tv(n, m) = qq   (:210-232)
template <int S>
__global__ void k_omp_tv_solve(OmpBatch ob, int n, int *status_out) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k, M = ob.ntau + 1;
    const double h = ob.h, wn = -h * greg_w(k, n, 0);
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
        double2 qq[s2], mm[s2];
        double2 *g = P.C.tv + ((long)n * M + m) * s2;
        for (int e = 0; e < s2; e++) {
            double2 q = g[e];
            for (int p = 1; p <= k + 1; p++)
                q = csub(q, cmul(cmk(0.0, bd_w(k, p) / h), P.C.tv[((long)(n - p) * M + m) * s2 + e]));
            qq[e] = q;
            double2 v = cneg(P.H[(long)(n + 1) * s2 + e]);
            v = cadd(v, cscale(P.A.ret[(ctri(n) + n) * s2 + e], wn));
            if (e / S == e % S) v = cadd(v, cmk(P.mu, bd_w(k, 0) / h));
            mm[e] = v;
        }
        omp_block_solve<S>(mm, qq, g, false, status_out);
    }
}

// G^<(j, n), j in [0, n-k): qq = G^<(j, n) + sum_p d_p G^<(j, n-p),
// G^<(j, n) [ -d_0 + mu - h omega_0 Sigma^R(j, j)^dagger - H(n) ] = qq   (:343-358)
template <int S>
__global__ void k_omp_les_solve(OmpBatch ob, int n, int *status_out) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k;
    const double h = ob.h, w0 = h * greg_omega(k, 0);
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n - k; j += gridDim.x * blockDim.x) {
        double2 qq[s2], mm[s2];
        double2 *g = P.C.les + (ctri(n) + j) * s2;
        for (int e = 0; e < s2; e++) {
            const int a = e / S, b = e % S;
            double2 q = g[e];
            for (int p = 1; p <= k + 1; p++)
                q = cadd(q, cmul(cmk(0.0, bd_w(k, p) / h), P.C.les[(ctri(n - p) + j) * s2 + e]));
            qq[e] = q;
            double2 v = cneg(P.H[(long)(n + 1) * s2 + e]);
            v = csub(v, cscale(cconj(P.A.ret[(ctri(j) + j) * s2 + b * S + a]), w0));
            if (a == b) v = cadd(v, cmk(P.mu, -bd_w(k, 0) / h));
            mm[e] = v;
        }
        omp_block_solve<S>(mm, qq, g, true, status_out);
    }
}

// The lesser rows solved in sequence, one CTA per problem (:362-410, and the serial step
// dyson_timestep_les :893-1056 for n < 2k+1).  Rows r0..n of G^<(., n): first
// gles(j) = [Sigma^tv * G^vt + Sigma^< * G^A](j, n) (convolution_timestep_les_tvvt / _lesadv,
// :1075-1394), then for the full step G^<(0, n) = -G^tv(n, 0)^dagger and the k x k right
// solve for rows 1..k; then, row by row,
//   [ d_0 + mu - H(j) - h w(j, j) Sigma^R(j, j) ] G^<(j, n) = gles(j) - sum_p d_p G^<(j-p, n)
//                                                          + h sum_{m<j} w(j, m) Sigma^R(j, m) G^<(m, n).
// Shared memory: 8 blocks of s^2, partial sums (blockDim / s^2 groups), the start system.
template <int S>
__global__ void k_omp_les_serial(OmpBatch ob, int n, int full, int *status_out) {
    constexpr int s2 = S * S;
    extern __shared__ double2 smem[];
    const OmpProb &P = ob.p[blockIdx.x];
    const int k = ob.k, ntau = ob.ntau, M = ntau + 1, n1 = n > k ? n : k;
    const double h = ob.h, dtau = ob.beta / ntau;
    const int r0 = full ? 0 : n - k;
    double2 *gcol = P.C.les + ctri(n) * s2;  // G^<(., n)
    const double2 *sret = P.A.ret, *sles = P.A.les, *stv = P.A.tv;
    const int ngrp = blockDim.x / s2;  // >= 1: blockDim.x >= s2
    double2 *part = smem;                       // ngrp * s2
    double2 *blk1 = part + (long)ngrp * s2;     // s2: qq, then X
    double2 *minv = blk1 + s2;                  // s2
    double2 *sys = minv + s2;                   // start system (full step)
    int *ipiv = (int *)(sys + (long)(k * S) * (k * S) + (long)(k * S) * S), *status = ipiv + 1;
    if (threadIdx.x == 0) *status = 0;
    // gles rows r0..n into G^<(., n)
    const double2 fvt = cmk(0.0, dtau * (double)ob.sig_a);  // (-i dtau)(-sig_Sigma)
    for (long e = threadIdx.x; e < (long)(n - r0 + 1) * s2; e += blockDim.x) {
        const int j = r0 + (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        double2 acc = cmk(0, 0);
        for (int m = 0; m <= ntau; m++)
            acc = cfma(cmul(fvt, cmk(greg_w(k, ntau, m), 0)),
                       emul_ad<S>(stv + ((long)j * M + m) * s2, P.Bcc.tv + ((long)n * M + ntau - m) * s2, a, b), acc);
        for (int m = 0; m <= n1; m++) {
            const double w = h * greg_w(k, n, m);
            double2 t = cmk(0, 0);
            for (int c = 0; c < S; c++) {
                double2 lv = m >= j ? sles[(ctri(m) + j) * s2 + a * S + c] : cneg(cconj(sles[(ctri(j) + m) * s2 + c * S + a]));
                double2 bv = m <= n ? cscale(cconj(P.Bcc.ret[(ctri(n) + m) * s2 + b * S + c]), w)
                                    : cscale(P.B.ret[(ctri(m) + n) * s2 + c * S + b], -w);
                t = cfma(lv, bv, t);
            }
            acc = cadd(acc, t);
        }
        gcol[(long)j * s2 + ab] = acc;
    }
    __syncthreads();
    int jfirst = r0;
    if (full) {
        const int KS = k * S;
        double2 *A = sys, *R = sys + (long)KS * KS;
        // G^<(0, n) = -G^tv(n, 0)^dagger
        double2 g0[s2];
        for (int e = 0; e < s2; e++) g0[e] = cneg(cconj(P.B.tv[((long)n * M) * s2 + (e % S) * S + e / S]));
        // block rows p = j - 1 of the start system: sum_q mm(p, q) X_q = qq(p)
        for (int e = threadIdx.x; e < KS * KS; e += blockDim.x) A[e] = cmk(0, 0);
        __syncthreads();
        for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
            const int p = e / s2, ab = e % s2, a = ab / S, b = ab % S, j = p + 1;
            double2 q = gcol[(long)j * s2 + ab];
            for (int m = 0; m <= k; m++) {
                const double2 cw = cmk(0.0, poly_diff(k, j, m) / h);
                if (m == 0) q = csub(q, cmul(cw, g0[ab]));
                else if (a == b) A[(p * S + a) * KS + (m - 1) * S + b] = cadd(A[(p * S + a) * KS + (m - 1) * S + b], cw);
            }
            {
                double2 v = cneg(P.H[(long)(j + 1) * s2 + ab]);
                if (a == b) v = cadd(v, cmk(P.mu, 0.0));
                A[(p * S + a) * KS + p * S + b] = cadd(A[(p * S + a) * KS + p * S + b], v);
            }
            for (int m = 0; m <= k; m++) {
                const double cw = h * greg_w(k, j, m);
                if (m == 0) {
                    double2 t = cmk(0, 0);
                    for (int c = 0; c < S; c++) t = cfma(sret[(ctri(j)) * s2 + a * S + c], g0[c * S + b], t);
                    q = cfma(cmk(cw, 0), t, q);
                } else {
                    double2 st = j >= m ? sret[(ctri(j) + m) * s2 + ab] : cneg(cconj(sret[(ctri(m) + j) * s2 + b * S + a]));
                    const long idx = (long)(p * S + a) * KS + (m - 1) * S + b;
                    A[idx] = csub(A[idx], cscale(st, cw));
                }
            }
            R[(p * S + a) * S + b] = q;
        }
        __syncthreads();
        cta_solve(A, R, KS, S, ipiv, status);
        for (int e = threadIdx.x; e < s2; e += blockDim.x) gcol[e] = g0[e];
        for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
            const int q = e / s2, ab = e % s2, a = ab / S, b = ab % S;
            gcol[(long)(q + 1) * s2 + ab] = R[(q * S + a) * S + b];
        }
        __syncthreads();
        jfirst = k + 1;
    }
    for (int j = jfirst; j <= n; j++) {
        // partial sums of h w(j, m) Sigma^R(j, m) G^<(m, n) over m < j, group g takes m = g mod ngrp
        if (threadIdx.x < ngrp * s2) {
            const int g = threadIdx.x / s2, ab = threadIdx.x % s2, a = ab / S, b = ab % S;
            double2 t = cmk(0, 0);
            for (int m = g; m < j; m += ngrp)
                t = cfma(cmk(h * greg_w(k, j, m), 0), emul<S>(sret + (ctri(j) + m) * s2, gcol + (long)m * s2, a, b), t);
            part[g * s2 + ab] = t;
        }
        __syncthreads();
        if (threadIdx.x < s2) {
            const int ab = threadIdx.x;
            double2 q = gcol[(long)j * s2 + ab];
            for (int p = 1; p <= k + 1; p++) q = csub(q, cmul(cmk(0.0, bd_w(k, p) / h), gcol[(long)(j - p) * s2 + ab]));
            for (int g = 0; g < ngrp; g++) q = cadd(q, part[g * s2 + ab]);
            blk1[ab] = q;
        }
        if (threadIdx.x == 0) {
            double2 mm[s2];
            const double wjj = -h * greg_w(k, j, j);
            for (int e = 0; e < s2; e++) {
                double2 v = cneg(P.H[(long)(j + 1) * s2 + e]);
                v = cadd(v, cscale(sret[(ctri(j) + j) * s2 + e], wjj));
                if (e / S == e % S) v = cadd(v, cmk(P.mu, bd_w(k, 0) / h));
                mm[e] = v;
            }
            if (small_inverse<S>(mm, minv)) *status = 1;
        }
        __syncthreads();
        if (threadIdx.x < s2) {
            const int a = threadIdx.x / S, b = threadIdx.x % S;
            gcol[(long)j * s2 + threadIdx.x] = emul<S>(minv, blk1, a, b);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && *status && status_out) atomicExch(status_out, 1);
}

// ---------------------------------------------------------------------------------------
// vie2_timestep_omp (cntr_vie2_impl.hpp:1911-1965): after the convolutions wrote
// Q1 = Q - F * G into G's time step (k_incr_* with Q as the base),
//   ret (which 0):  [1 + wt h F^R(tstp, tstp)] G^R(tstp, n) = Q1, wt = w(tstp - n, 0)
//                   (poly_integration(n, tstp, tstp) for tstp < k)
//   tv  (which 1):  [1 + w(tstp, tstp) h F^R(tstp, tstp)] G^tv(tstp, m) = Q1
//   les (which 2):  G^<(n, tstp) [1 + w(tstp, tstp) h F^R(tstp, tstp)]^dagger = Q1
// for indices [lo, hi).  p.A = F.
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_omp_vie2_solve(OmpBatch ob, int tstp, int which, int *status_out) {
    constexpr int s2 = S * S;
    const OmpProb &P = ob.p[blockIdx.y];
    const int k = ob.k, M = ob.ntau + 1;
    const double2 *ftt = P.A.ret + (ctri(tstp) + tstp) * s2;
    for (int i = ob.lo + blockIdx.x * blockDim.x + threadIdx.x; i < ob.hi; i += gridDim.x * blockDim.x) {
        double wt;
        double2 *g;
        if (which == 0) {
            wt = tstp < k ? poly_int(k, i, tstp, tstp) : greg_w(k, tstp - i, 0);
            g = P.C.ret + (ctri(tstp) + i) * s2;
        } else {
            wt = greg_w(k, tstp, tstp);
            g = which == 1 ? P.C.tv + ((long)tstp * M + i) * s2 : P.C.les + (ctri(tstp) + i) * s2;
        }
        double2 mm[s2];
        for (int e = 0; e < s2; e++) {
            const int a = e / S, b = e % S;
            double2 v = which == 2 ? cconj(ftt[b * S + a]) : ftt[e];
            v = cscale(v, wt * ob.h);
            if (a == b) v = cadd(v, cmk(1.0, 0.0));
            mm[e] = v;
        }
        double2 q[s2];
        for (int e = 0; e < s2; e++) q[e] = g[e];
        omp_block_solve<S>(mm, q, g, which == 2, status_out);
    }
}
