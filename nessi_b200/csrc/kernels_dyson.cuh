// Batched Dyson time step (libcntr cntr_dyson_impl.hpp:1618-1648) for many problems
// ("k-points") sharing one self-energy Sigma.  Every problem keeps libcntr's herm_matrix
// layout in device memory (cntr_herm_matrix_impl.hpp:457-477).
//
// One time step n > k runs as
//   k_prep_problem   s x s inverses of the step matrices (dyson_impl :179-213, :693-706, :983-1011)
//   k_prep_group     history coefficients for tv, dense copies of Sigma^< and Sigma^tv
//   k_ret            G^R(n, 0..n): k-block start + Volterra recursion in t'   (:80-222)
//   k_tv             G^tv(n, 0..ntau): history stream + Matsubara integral + solve (:651-741)
//   k_les_operands   right-hand operands of the Sigma-shared products
//   2 x ZGEMM        tv*vt + les*adv convolutions for all problems at once (conv_impl :1075-1394)
//   k_les            G^<(0..n, n): k-block start + Volterra recursion in t (:893-1056)
#pragma once
#include "device_common.cuh"

struct ProbDev {
    double2 *gret, *gles, *gtv, *gmat;  // this problem's G (libcntr layout)
    const double2 *H;                   // (nt+2) s^2 blocks, H(-1) first
    double2 *minv_ret, *minv_les;       // (nt+1) s^2: inverses of the ret / les+tv step matrices
    double mu;
    int nt;
    int col;                            // column of this problem in the group's GEMM operands
    int pad;
};

struct GroupDev {
    const double2 *sret, *sles, *stv, *smat;  // Sigma (libcntr layout, shared by the group)
    double2 *Ldense;   // ((ntmax+1)s) x ((ntmax+1)s) row-major: Sigma^<(j,m), full (anti-hermitian)
    double2 *Tdense;   // ((ntmax+1)s) x ((ntau+1)s) row-major: Sigma^tv(j,m) reordered (s>1)
    double2 *tvcoef;   // (ntmax+1) s^2: coefficients of the tv history sum at the current step
    double2 *badv, *btv, *gles;  // GEMM operands / result, leading dimension ldc
    int ntmax, ntau, s, sig, k;
    int ldc;           // >= nprob * s
    double h, beta;
};

__device__ __forceinline__ long tri(long t) { return t * (t + 1) / 2; }

// ---------------------------------------------------------------------------------------
// k_prep_problem: Minv_les[n] (= tv step matrix for n > k), Minv_ret[j] for j in [r0, r1]
//   tv/les:  mm = i/h bd0 + mu - H(n) - h w0 Sigma^R(n,n)        (dyson_impl :693-699, :983-1004)
//   ret:     mm = i/h bd0 + mu - H(j)^dagger - h w0 Sigma^R(j,j) (dyson_impl :188-199)
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_prep_problem(GroupDev g, const ProbDev *__restrict__ probs, int n, int les_lo, int r0, int r1) {
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, s2 = S * S;
    const double h = g.h;
    const double2 ibd0 = cmk(0.0, bd_w(k, 0) / h);
    const double w0 = h * greg_omega(k, 0);
    // rows: les indices les_lo..n then ret indices r0..r1
    int nles = n - les_lo + 1;
    int nret = r1 >= r0 ? r1 - r0 + 1 : 0;
    for (int t = threadIdx.x; t < nles + nret; t += blockDim.x) {
        bool is_ret = t >= nles;
        int j = is_ret ? r0 + (t - nles) : les_lo + t;
        if (j > p.nt) continue;
        double2 M[S * S];
        const double2 *Hj = p.H + (long)(j + 1) * s2;
        const double2 *Sjj = g.sret + (tri(j) + j) * s2;
        for (int a = 0; a < S; a++)
            for (int b = 0; b < S; b++) {
                double2 hv = is_ret ? cconj(Hj[b * S + a]) : Hj[a * S + b];
                double2 v = csub(cscale(Sjj[a * S + b], -w0), hv);
                if (a == b) v = cadd(v, cadd(ibd0, cmk(p.mu, 0.0)));
                M[a * S + b] = v;
            }
        double2 *dst = (is_ret ? p.minv_ret : p.minv_les) + (long)j * s2;
        small_inverse<S>(M, dst);
    }
}

// ---------------------------------------------------------------------------------------
// k_prep_group: tv coefficients a_j = h w(n,j) Sigma^R(n,j) - [n-k-1<=j<n] (i/h) bd(n-j) 1
// (conv_impl :942-972 with the BDF terms of dyson_impl :681-692 folded in), and the dense
// copies of Sigma^< (rows/columns d_lo..n) and Sigma^tv (rows d_lo..n).
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_prep_group(GroupDev g, int n, int d_lo) {
    const int k = g.k, s2 = S * S;
    const double h = g.h;
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nth = (long)gridDim.x * blockDim.x;
    // tv coefficients, j = 0..n-1
    for (long e = tid; e < (long)n * s2; e += nth) {
        int j = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        double2 v = cscale(g.sret[(tri(n) + j) * s2 + ab], h * greg_w(k, n, j));
        if (j >= n - k - 1 && a == b) v = csub(v, cmk(0.0, bd_w(k, n - j) / h));
        g.tvcoef[(long)j * s2 + ab] = v;
    }
    // dense Sigma^<: for every t in [d_lo, n]: column t (rows 0..t) and row t (cols 0..t-1)
    const long ldL = (long)(g.ntmax + 1) * S;
    for (int t = d_lo; t <= n; t++) {
        for (long e = tid; e < (long)(t + 1) * s2; e += nth) {
            int j = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
            // L(j,t) = Sigma^<(j,t), j <= t
            double2 v = g.sles[(tri(t) + j) * s2 + ab];
            g.Ldense[((long)j * S + a) * ldL + (long)t * S + b] = v;
            // L(t,j) = -Sigma^<(j,t)^dagger, j < t   [element (b,a) of the block]
            if (j < t) g.Ldense[((long)t * S + b) * ldL + (long)j * S + a] = cneg(cconj(v));
        }
    }
    if (S > 1) {
        const long ldT = (long)(g.ntau + 1) * S;
        for (int t = d_lo; t <= n; t++)
            for (long e = tid; e < (long)(g.ntau + 1) * s2; e += nth) {
                int m = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
                g.Tdense[((long)t * S + a) * ldT + (long)m * S + b] =
                    g.stv[((long)t * (g.ntau + 1) + m) * s2 + ab];
            }
    }
}

// ---------------------------------------------------------------------------------------
// Start blocks: the k x k block systems of dyson_timestep_ret (:112-157) and
// dyson_timestep_les (:926-982), solved by the whole CTA in shared memory.
// ---------------------------------------------------------------------------------------
// ret: unknowns X_q = G(n, n-q-1); equations sum_q X_q mm(p,q) = qq(p)  (left solve)
template <int S>
__device__ void ret_start_block(const GroupDev &g, const ProbDev &p, int n, double2 *smem) {
    const int k = g.k, s2 = S * S, KS = k * S;
    const double h = g.h;
    double2 *mm = smem;                 // k*k blocks (block (p,q) at (p*k+q)*s2)
    double2 *qq = mm + k * k * s2;      // k blocks
    double2 *A = qq + k * s2;           // (KS x KS)
    double2 *R = A + KS * KS;           // (KS x S)
    int *ipiv = (int *)(R + KS * S);
    int *status = ipiv + 1;
    double2 *grow = p.gret + tri(n) * s2;  // G(n, .)
    for (int e = threadIdx.x; e < k * k * s2; e += blockDim.x) mm[e] = cmk(0, 0);
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) qq[e] = cmk(0, 0);
    if (threadIdx.x == 0) *status = 0;
    __syncthreads();
    // thread per (row-block pr, element ab): fills block row pr of mm and qq(pr)
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
        int pr = e / s2, ab = e % s2, a = ab / S, b = ab % S;
        int j = pr + 1;
        double2 q = cmk(0, 0);
        // derivative: l == 0 -> qq -= (i/h) P(j,0) G(n,n); G(n,n) = -i 1
        {
            double2 cw = cmk(0.0, poly_diff(k, j, 0) / h);
            double2 gnn = a == b ? cmk(0.0, -1.0) : cmk(0, 0);
            q = csub(q, cmul(cw, gnn));
        }
        for (int l = 1; l <= k; l++) {
            if (a == b) mm[(pr * k + l - 1) * s2 + ab] = cadd(mm[(pr * k + l - 1) * s2 + ab], cmk(0.0, poly_diff(k, j, l) / h));
        }
        // H: mm(pr,pr) += mu - H(n-j)
        {
            double2 hv = p.H[(long)(n - j + 1) * s2 + ab];
            double2 v = cneg(hv);
            if (a == b) v = cadd(v, cmk(p.mu, 0.0));
            mm[(pr * k + pr) * s2 + ab] = cadd(mm[(pr * k + pr) * s2 + ab], v);
        }
        // integral: l = 0..k, w = h w(j,l), stemp = Sigma(n-l, n-j) or -Sigma(n-j,n-l)^dagger
        for (int l = 0; l <= k; l++) {
            double w = h * greg_w(k, j, l);
            double2 st;
            if (l <= j) st = g.sret[(tri(n - l) + (n - j)) * s2 + ab];
            else { st = cconj(g.sret[(tri(n - j) + (n - l)) * s2 + b * S + a]); w = -w; }
            if (l == 0) {
                // qq += w * G(n,n) * stemp, G(n,n) = -i 1  ->  -i w stemp
                q = cadd(q, cmul(cmk(0.0, -w), st));
            } else {
                int idx = (pr * k + l - 1) * s2 + ab;
                mm[idx] = csub(mm[idx], cscale(st, w));
            }
        }
        qq[pr * s2 + ab] = q;
    }
    __syncthreads();
    // conjugate-transpose to a right solve: A[(pr,a),(q,b)] = conj(mm(pr,q)[b][a]),
    // R[(pr,a),c] = conj(qq(pr)[c][a])
    for (int e = threadIdx.x; e < KS * KS; e += blockDim.x) {
        int r = e / KS, c = e % KS, pr = r / S, a = r % S, q = c / S, b = c % S;
        A[e] = cconj(mm[(pr * k + q) * s2 + b * S + a]);
    }
    for (int e = threadIdx.x; e < KS * S; e += blockDim.x) {
        int r = e / S, c = e % S, pr = r / S, a = r % S;
        R[e] = cconj(qq[pr * s2 + c * S + a]);
    }
    __syncthreads();
    cta_solve(A, R, KS, S, ipiv, status);
    // X_q[a][c] = conj(Y[(q,c), a]) -> G(n, n-q-1)
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
        int q = e / s2, ac = e % s2, a = ac / S, c = ac % S;
        grow[(long)(n - q - 1) * s2 + ac] = cconj(R[(q * S + c) * S + a]);
    }
    __syncthreads();
}

// les: unknowns x_j = G^<(j,n), j = 1..k; sum_q mm(p,q) x_{q+1} = qq(p)  (right solve)
template <int S>
__device__ void les_start_block(const GroupDev &g, const ProbDev &p, int n, const double2 *gl, long ldc,
                                double2 *xcol, double2 *smem) {
    const int k = g.k, s2 = S * S, KS = k * S;
    const double h = g.h;
    double2 *A = smem;           // (KS x KS)
    double2 *R = A + KS * KS;    // (KS x S)
    int *ipiv = (int *)(R + KS * S);
    int *status = ipiv + 1;
    if (threadIdx.x == 0) *status = 0;
    for (int e = threadIdx.x; e < KS * KS; e += blockDim.x) A[e] = cmk(0, 0);
    __syncthreads();
    // thread per (pr, a, d): qq(pr)[a][d] and the row (pr,a) of A
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
        int pr = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        int j = pr + 1;
        double2 q = gl[((long)j * S + a) * ldc + d];  // gles(j)
        double2 cw0 = cmk(0.0, poly_diff(k, j, 0) / h);
        q = csub(q, cmul(cw0, xcol[ad]));  // x_0 = xcol[0..s2)
        // h w(j,0) Sigma^R(j,0) x_0
        {
            double w = h * greg_w(k, j, 0);
            double2 acc = cmk(0, 0);
            for (int b = 0; b < S; b++) acc = cfma(g.sret[(tri(j) + 0) * s2 + a * S + b], xcol[b * S + d], acc);
            q = cadd(q, cscale(acc, w));
        }
        R[(pr * S + a) * S + d] = q;
        if (d == 0) {
            for (int m = 1; m <= k; m++) {
                double2 cwm = cmk(0.0, poly_diff(k, j, m) / h);
                double w = h * greg_w(k, j, m);
                for (int b = 0; b < S; b++) {
                    double2 st;
                    if (j >= m) st = g.sret[(tri(j) + m) * s2 + a * S + b];
                    else st = cneg(cconj(g.sret[(tri(m) + j) * s2 + b * S + a]));
                    double2 v = cscale(st, -w);
                    if (a == b) v = cadd(v, cwm);
                    if (m == j) {
                        double2 hv = p.H[(long)(j + 1) * s2 + a * S + b];
                        v = csub(v, hv);
                        if (a == b) v = cadd(v, cmk(p.mu, 0.0));
                    }
                    A[(pr * S + a) * KS + (m - 1) * S + b] = v;
                }
            }
        }
    }
    __syncthreads();
    cta_solve(A, R, KS, S, ipiv, status);
    for (int e = threadIdx.x; e < k * s2; e += blockDim.x) {
        int q = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        xcol[(long)(q + 1) * s2 + ad] = R[(q * S + a) * S + d];
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------------------
// k_ret: G^R(n, j), j = n-k-1 .. 0 (dyson_impl :158-213), blocked left-looking:
//   qq(j) = h sum_{m=j+1}^{n} w(n-j, n-m) G(n,m) Sigma(m,j) - sum_{p=1}^{k+1} (i/h) bd(p) G(n, j+p)
//   G(n,j) = qq(j) Minv_ret[j]
// Blocks of JB consecutive j: phase A sums all m above the block (CTA-parallel), phase B
// finishes the block sequentially on warp 0.
// ---------------------------------------------------------------------------------------
template <int S> struct RetCfg {
    static constexpr int JB = (S == 1) ? 32 : (S == 2 ? 32 : (256 / (S * S) > 1 ? 256 / (S * S) : 1));
    static constexpr int E = JB * S * S;               // entries of one block
    static constexpr int GM = (256 / E) > 0 ? 256 / E : 1;  // m-groups in phase A
};

template <int S>
__global__ void __launch_bounds__(256) k_ret(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    extern __shared__ double2 smem[];
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, s2 = S * S;
    const double h = g.h;
    constexpr int JB = RetCfg<S>::JB, E = RetCfg<S>::E, GM = RetCfg<S>::GM;
    double2 *grow = p.gret + tri(n) * s2;  // G(n, 0..n)
    // zero the row, G(n,n) = -i
    for (long e = threadIdx.x; e < (long)(n + 1) * s2; e += blockDim.x) {
        int ab = (int)(e % s2);
        grow[e] = (e / s2 == n && (ab / S == ab % S)) ? cmk(0.0, -1.0) : cmk(0, 0);
    }
    __syncthreads();
    ret_start_block<S>(g, p, n, smem);
    double2 *part = smem;            // GM * E partial sums
    double2 *acc = part + GM * E;    // E block sums
    double2 *qv = acc + E;           // s2 scratch for phase B
    const int tid = threadIdx.x;
    for (int jhi = n - k - 1; jhi >= 0; jhi -= JB) {
        const int jlo = jhi - JB + 1 < 0 ? 0 : jhi - JB + 1;
        const int nb = jhi - jlo + 1;
        // ---- phase A: acc(j) = sum_{m=jhi+1}^{n} w(n-j,n-m) G(n,m) Sigma(m,j)
        if (tid < GM * E) {
            const int gi = tid / E, e = tid % E;
            const int jj = e / s2, ad = e % s2, a = ad / S, d = ad % S;
            double2 sum = cmk(0, 0);
            if (jj < nb) {
                const int j = jhi - jj;
                for (int m = jhi + 1 + gi; m <= n; m += GM) {
                    const double2 *gm = grow + (long)m * s2 + a * S;
                    const double2 *sm = g.sret + (tri(m) + j) * s2 + d;
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int b = 0; b < S; b++) t = cfma(gm[b], sm[b * S], t);
                    sum = cfma(cmk(greg_w(k, n - j, n - m), 0.0), t, sum);
                }
            }
            part[gi * E + e] = sum;
        }
        __syncthreads();
        for (int e = tid; e < E; e += blockDim.x) {
            double2 s = part[e];
            for (int gi = 1; gi < GM; gi++) s = cadd(s, part[gi * E + e]);
            acc[e] = s;
        }
        __syncthreads();
        // ---- phase B: sequential within the block (warp 0)
        if (tid < 32) {
            const int lane = tid;
            for (int jj = 0; jj < nb; jj++) {
                const int j = jhi - jj;
                for (int ad = lane; ad < s2; ad += 32) {
                    const int a = ad / S, d = ad % S;
                    double2 sum = acc[jj * s2 + ad];
                    for (int m = j + 1; m <= jhi; m++) {
                        const double2 *gm = grow + (long)m * s2 + a * S;
                        const double2 *sm = g.sret + (tri(m) + j) * s2 + d;
                        double2 t = cmk(0, 0);
                        for (int b = 0; b < S; b++) t = cfma(gm[b], sm[b * S], t);
                        sum = cfma(cmk(greg_w(k, n - j, n - m), 0.0), t, sum);
                    }
                    double2 q = cscale(sum, h);
                    for (int pp = 1; pp <= k + 1; pp++)
                        q = csub(q, cmul(cmk(0.0, bd_w(k, pp) / h), grow[(long)(j + pp) * s2 + ad]));
                    qv[ad] = q;
                }
                __syncwarp();
                for (int ad = lane; ad < s2; ad += 32) {
                    const int a = ad / S, d = ad % S;
                    const double2 *mi = p.minv_ret + (long)j * s2;
                    double2 x = cmk(0, 0);
                    for (int b = 0; b < S; b++) x = cfma(qv[a * S + b], mi[b * S + d], x);
                    grow[(long)j * s2 + ad] = x;
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// k_tv: G^tv(n, tau) for one problem and a tile of tau (dyson_impl :651-741):
//   Q(tau) = sum_{j<n} a_j G^tv(j,tau) + dtau * matsubara_integral_2(Sigma^tv(n,.), G^mat)(tau)
//   G^tv(n,tau) = Minv_les[n] Q(tau)
// Thread per (tau, column d); the history G^tv(0..n-1, tile) is streamed once.
// ---------------------------------------------------------------------------------------
template <int S>
__device__ __forceinline__ void acc_col(double2 *acc, const double2 *A, const double2 *B, int d, double w) {
    // acc[a] += w * sum_b A[a][b] B[b][d]
#pragma unroll
    for (int a = 0; a < S; a++) {
        double2 t = cmk(0, 0);
#pragma unroll
        for (int b = 0; b < S; b++) t = cfma(A[a * S + b], B[b * S + d], t);
        acc[a] = cfma(cmk(w, 0.0), t, acc[a]);
    }
}

template <int S, int TT>
__global__ void __launch_bounds__(TT * S) k_tv(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    constexpr int s2 = S * S, CH = (s2 <= 32) ? 64 : 2048 / s2;  // coefficient chunk (j) staged in shared memory
    __shared__ double2 coef[CH * s2];
    const ProbDev p = probs[blockIdx.y];
    const int k = g.k, ntau = g.ntau, M = ntau + 1;
    const int tl = threadIdx.x / S, d = threadIdx.x % S;
    const int tau = blockIdx.x * TT + tl;
    const bool live = tau <= ntau;
    double2 acc[S];
#pragma unroll
    for (int a = 0; a < S; a++) acc[a] = cmk(0, 0);
    // history: j = 0..n-1 (G^tv(n,.) itself is zero at this point in the reference)
    for (int j0 = 0; j0 < n; j0 += CH) {
        const int nj = n - j0 < CH ? n - j0 : CH;
        __syncthreads();
        for (int e = threadIdx.x; e < nj * s2; e += blockDim.x) coef[e] = g.tvcoef[(long)j0 * s2 + e];
        __syncthreads();
        if (live) {
            const double2 *gcol = p.gtv + ((long)j0 * M + tau) * s2 + d;
#pragma unroll 4
            for (int jj = 0; jj < nj; jj++) {
                const double2 *gj = gcol + (long)jj * M * s2;
                double2 bv[S];
#pragma unroll
                for (int b = 0; b < S; b++) bv[b] = __ldg(gj + b * S);
#pragma unroll
                for (int a = 0; a < S; a++) {
                    double2 t = acc[a];
#pragma unroll
                    for (int b = 0; b < S; b++) t = cfma(coef[jj * s2 + a * S + b], bv[b], t);
                    acc[a] = t;
                }
            }
        }
    }
    if (!live) return;
    // Matsubara part: dtau * [c2 + sig c1] (conv_impl :410-540), A = Sigma^tv(n,.), B = G^mat
    const double2 *A = g.stv + (long)n * M * s2;
    const double2 *B = p.gmat;
    const int m = tau;
    double2 c1[S], c2[S];
#pragma unroll
    for (int a = 0; a < S; a++) { c1[a] = cmk(0, 0); c2[a] = cmk(0, 0); }
    if (m == 0) {
    } else if (m < k) {
        for (int j = 0; j <= k; j++)
            for (int l = 0; l <= k; l++)
                acc_col<S>(c1, A + (long)j * s2, B + (long)(ntau - l) * s2, d, rcorr_w(k, m, l, j));
    } else {
        for (int l = 0; l <= m; l++)
            acc_col<S>(c1, A + (long)(m - l) * s2, B + (long)(ntau - l) * s2, d, greg_w(k, m, l));
    }
    const int r = ntau - m;
    if (r == 0) {
    } else if (r < k) {
        for (int l = 0; l <= k; l++)
            for (int j = 0; j <= k; j++)
                acc_col<S>(c2, A + (long)(ntau - l) * s2, B + (long)j * s2, d, rcorr_w(k, r, l, j));
    } else {
        for (int l = 0; l <= r; l++)
            acc_col<S>(c2, A + (long)(m + l) * s2, B + (long)l * s2, d, greg_w(k, r, l));
    }
    const double dtau = g.beta / ntau, sg = (double)g.sig;
    double2 q[S];
#pragma unroll
    for (int a = 0; a < S; a++) q[a] = cadd(acc[a], cscale(cadd(c2[a], cscale(c1[a], sg)), dtau));
    // solve: G^tv(n,tau)[a][d] = sum_b Minv[a][b] Q[b][d]
    const double2 *mi = p.minv_les + (long)n * s2;
    double2 *out = p.gtv + ((long)n * M + tau) * s2;
#pragma unroll
    for (int a = 0; a < S; a++) {
        double2 x = cmk(0, 0);
#pragma unroll
        for (int b = 0; b < S; b++) x = cfma(mi[a * S + b], q[b], x);
        out[a * S + d] = x;
    }
}

// ---------------------------------------------------------------------------------------
// k_les_operands: right-hand operands of the Sigma-shared products (conv_impl :1075-1394)
//   badv[(m,c)][(col,d)] = h w(n,m) G^R(n,m)^dagger[c][d],                 m = 0..n
//   btv [(m,c)][(col,d)] = w(ntau,m) (-i dtau)(-sig) G^tv(n,ntau-m)^dagger[c][d]
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void k_les_operands(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    const ProbDev p = probs[blockIdx.y];
    const int k = g.k, s2 = S * S, ntau = g.ntau;
    const double h = g.h, dtau = g.beta / ntau;
    const long ldc = g.ldc;
    const int rows = (n + 1) + (ntau + 1);
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)rows * s2; e += (long)gridDim.x * blockDim.x) {
        int r = (int)(e / s2), cd = (int)(e % s2), c = cd / S, d = cd % S;
        if (r <= n) {
            const int m = r;
            double2 v = cconj(p.gret[(tri(n) + m) * s2 + d * S + c]);
            g.badv[((long)m * S + c) * ldc + (long)p.col * S + d] = cscale(v, h * greg_w(k, n, m));
        } else {
            const int m = r - (n + 1);
            double2 v = cconj(p.gtv[((long)n * (ntau + 1) + (ntau - m)) * s2 + d * S + c]);
            // (-i dtau)(-sig) v * w
            double2 f = cmk(0.0, dtau * (double)g.sig * greg_w(k, ntau, m));
            g.btv[((long)m * S + c) * ldc + (long)p.col * S + d] = cmul(f, v);
        }
    }
}

// ---------------------------------------------------------------------------------------
// k_les: G^<(j, n), j = 0..n (dyson_impl :893-1056):
//   x_0 = -G^tv(n,0)^dagger; x_1..x_k from the k-block start system;
//   qq(j) = gles(j) - sum_{p=1}^{k+1} (i/h) bd(p) x_{j-p} + h sum_{m<j} w(j,m) Sigma^R(j,m) x_m
//   x_j = Minv_les[j] qq(j)
// Blocked left-looking as k_ret; phase A rows are Sigma^R(j, 0..jlo-1) (contiguous).
// ---------------------------------------------------------------------------------------
template <int S>
__global__ void __launch_bounds__(256) k_les(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    extern __shared__ double2 smem[];
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, s2 = S * S, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double h = g.h;
    const long ldc = g.ldc;
    constexpr int JB = RetCfg<S>::JB;
    const double2 *gl = g.gles + (long)p.col * S;   // gles(j)[a][d] at gl[(j*S+a)*ldc + d]
    double2 *xcol = p.gles + tri(n) * s2;           // G^<(0..n, n)
    // x_0
    for (int ad = tid; ad < s2; ad += blockDim.x) {
        int a = ad / S, d = ad % S;
        xcol[ad] = cneg(cconj(p.gtv[((long)n * (g.ntau + 1) + 0) * s2 + d * S + a]));
    }
    __syncthreads();
    les_start_block<S>(g, p, n, gl, ldc, xcol, smem);
    double2 *acc = smem;            // JB * s2
    double2 *qv = acc + JB * s2;    // s2
    const int nwarps = blockDim.x >> 5;
    for (int jlo = k + 1; jlo <= n; jlo += JB) {
        const int jhi = jlo + JB - 1 > n ? n : jlo + JB - 1;
        const int nb = jhi - jlo + 1;
        // ---- phase A: acc(j)[a][d] = sum_{m<jlo} w(j,m) Sigma^R(j,m)[a][b] x_m[b][d]
        // warp per row j; lane = (m-group, d)
        constexpr int LPG = S;                        // lanes per m-group
        constexpr int NG = 32 / LPG;                  // m-groups per warp
        for (int jj = warp; jj < nb; jj += nwarps) {
            const int j = jlo + jj;
            const int mg = lane / LPG, dd = lane % LPG;
            double2 a_[S];
#pragma unroll
            for (int a = 0; a < S; a++) a_[a] = cmk(0, 0);
            if (mg < NG) {
                const double2 *srow = g.sret + tri(j) * s2;
                for (int m = mg; m < jlo; m += NG) {
                    const double w = greg_w(k, j, m);
                    const double2 *sm = srow + (long)m * s2;
                    const double2 *xm = xcol + (long)m * s2;
#pragma unroll
                    for (int a = 0; a < S; a++) {
                        double2 t = cmk(0, 0);
#pragma unroll
                        for (int b = 0; b < S; b++) t = cfma(sm[a * S + b], xm[b * S + dd], t);
                        a_[a] = cfma(cmk(w, 0.0), t, a_[a]);
                    }
                }
            }
            // reduce over m-groups (lanes with equal dd)
            if constexpr ((S & (S - 1)) == 0) {
#pragma unroll
                for (int a = 0; a < S; a++) {
                    double2 v = a_[a];
                    for (int off = LPG; off < 32; off <<= 1) {
                        v.x += __shfl_xor_sync(0xffffffffu, v.x, off);
                        v.y += __shfl_xor_sync(0xffffffffu, v.y, off);
                    }
                    a_[a] = v;
                }
                if (mg == 0)
                    for (int a = 0; a < S; a++) acc[jj * s2 + a * S + dd] = a_[a];
            } else {
                double2 *red = qv + s2 + warp * 32 * S;
                for (int a = 0; a < S; a++) red[lane * S + a] = (mg < NG) ? a_[a] : cmk(0, 0);
                __syncwarp();
                if (lane < S) {
                    for (int a = 0; a < S; a++) {
                        double2 v = cmk(0, 0);
                        for (int g2 = 0; g2 < NG; g2++) v = cadd(v, red[(g2 * S + lane) * S + a]);
                        acc[jj * s2 + a * S + lane] = v;
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // ---- phase B on warp 0
        if (tid < 32) {
            for (int jj = 0; jj < nb; jj++) {
                const int j = jlo + jj;
                for (int ad = lane; ad < s2; ad += 32) {
                    const int a = ad / S, d = ad % S;
                    double2 sum = acc[jj * s2 + ad];
                    const double2 *srow = g.sret + tri(j) * s2;
                    for (int m = jlo; m < j; m++) {
                        double2 t = cmk(0, 0);
                        for (int b = 0; b < S; b++) t = cfma(srow[(long)m * s2 + a * S + b], xcol[(long)m * s2 + b * S + d], t);
                        sum = cfma(cmk(greg_w(k, j, m), 0.0), t, sum);
                    }
                    double2 q = gl[((long)j * S + a) * ldc + d];
                    for (int pp = 1; pp <= k + 1; pp++)
                        q = csub(q, cmul(cmk(0.0, bd_w(k, pp) / h), xcol[(long)(j - pp) * s2 + ad]));
                    q = cfma(cmk(h, 0.0), sum, q);
                    qv[ad] = q;
                }
                __syncwarp();
                for (int ad = lane; ad < s2; ad += 32) {
                    const int a = ad / S, d = ad % S;
                    const double2 *mi = p.minv_les + (long)j * s2;
                    double2 x = cmk(0, 0);
                    for (int b = 0; b < S; b++) x = cfma(mi[a * S + b], qv[b * S + d], x);
                    xcol[(long)j * s2 + ad] = x;
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
}
