// Batched Dyson time step (libcntr cntr_dyson_impl.hpp:1618-1648) for many problems
// ("k-points") sharing one self-energy Sigma.  Every problem keeps libcntr's herm_matrix
// layout in device memory (cntr_herm_matrix_impl.hpp:457-477).
//
// One time step n > k runs as
//   k_prep_problem   s x s inverses of the step matrices (dyson_impl :179-213, :693-706, :983-1011)
//   k_prep_group     history coefficients for tv, dense copies of Sigma^< and Sigma^tv
//   k_ret            G^R(n, 0..n): k-block start + Volterra recursion in t'   (:80-222)
//   k_tv             G^tv(n, 0..ntau): history stream + Matsubara integral + solve (:651-741)
//   k_les_operands_t right-hand operands of the Sigma-shared products
//   2 x k_zgemm      tv*vt + les*adv convolutions for all problems at once (conv_impl :1075-1394)
//   k_les            G^<(0..n, n): k-block start + Volterra recursion in t (:893-1056)
// The Volterra recursions also run group-wide (k_ret_start / k_les_start + k_volterra_cl).
#pragma once
#include "device_common.cuh"

struct ProbDev {
    double2 *gret, *gles, *gtv, *gmat;  // this problem's G (libcntr layout)
    const double2 *qret, *qles, *qtv;   // VIE2: the source term Q (tv in plane layout); else null
    const double2 *H;                   // (nt+2) s^2 blocks, H(-1) first
    double2 *minv_ret, *minv_les;       // (nt+1) s^2: inverses of the ret / les+tv step matrices
    float2 *gtv32;                      // mixed precision: FP32 copy of G^tv (plane layout) or null
    double mu;
    int nt;
    int col;                            // column of this problem in the group's GEMM operands
    int pad;
};

struct GroupDev {
    const double2 *sret, *sles, *stv, *smat;  // Sigma, or F of a VIE2 group (libcntr layout, shared)
    const double2 *rret;  // triangle of the retarded recursion: Sigma^R, or Fcc^R for VIE2
    const double2 *lcc;   // lesser triangle for t' < t of the les*adv operand: Sigma^<, or Fcc^<
    double2 *Ldense;   // ((ntmax+1)s) x ((ntmax+1)s) row-major: Sigma^<(j,m), full (anti-hermitian)
    double2 *Tdense;   // ((ntmax+1)s) x ((ntau+1)s) row-major: Sigma^tv(j,m) reordered (s>1)
    double2 *tvcoef;   // (ntmax+1) s^2: coefficients of the tv history sum at the current step
    double2 *badv, *btv, *gles;  // GEMM operands / result, leading dimension ldc
    double2 *Kmat;     // ((ntau+1)s) x ((ntau+1)s) row-major: Matsubara operator of the step
    double2 *Gmat_all; // ((ntau+1)s) x ldc: every problem's G^mat as columns
    double2 *Cmat;     // ((ntau+1)s) x ldc: Matsubara part of the tv right-hand side
    const double2 *fccmat;  // Fcc^mat of a VIE2 group (steepest-descent vie2_mat), or null
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
// VIE2 ([1 + F] G = Q, cntr_vie2_impl.hpp:60-140, 645-725, 847-990): the step matrices are
//   tv/les:  mm = 1 + h w0 F^R(j,j);   ret: mm = 1 + h w0 Fcc^R(j,j)
template <int S, bool VIE = false>
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
        if (VIE) {
            const double2 *Fjj = (is_ret ? g.rret : g.sret) + (tri(j) + j) * s2;
            for (int e = 0; e < s2; e++) M[e] = cadd(cscale(Fjj[e], w0), cmk(e / S == e % S ? 1.0 : 0.0, 0.0));
        } else {
            const double2 *Hj = p.H + (long)(j + 1) * s2;
            const double2 *Sjj = g.sret + (tri(j) + j) * s2;
            for (int a = 0; a < S; a++)
                for (int b = 0; b < S; b++) {
                    double2 hv = is_ret ? cconj(Hj[b * S + a]) : Hj[a * S + b];
                    double2 v = csub(cscale(Sjj[a * S + b], -w0), hv);
                    if (a == b) v = cadd(v, cadd(ibd0, cmk(p.mu, 0.0)));
                    M[a * S + b] = v;
                }
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
// VIE2: a_j = -h w(n,j) F^R(n,j) (conv_tv with A = F, moved to the right-hand side).
template <int S, bool VIE = false>
__global__ void k_prep_group(GroupDev g, int n, int d_lo) {
    const int k = g.k, s2 = S * S;
    const double h = g.h;
    const long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nth = (long)gridDim.x * blockDim.x;
    // tv coefficients, j = 0..n-1
    for (long e = tid; e < (long)n * s2; e += nth) {
        int j = (int)(e / s2), ab = (int)(e % s2), a = ab / S, b = ab % S;
        (void)a; (void)b;
        double2 v = cscale(g.sret[(tri(n) + j) * s2 + ab], (VIE ? -h : h) * greg_w(k, n, j));
        if (!VIE && j >= n - k - 1 && a == b) v = csub(v, cmk(0.0, bd_w(k, n - j) / h));
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
            // L(t,j) = -Sigma^<(j,t)^dagger (-Fcc^<(j,t)^dagger for VIE2), j < t  [element (b,a)]
            if (j < t) g.Ldense[((long)t * S + b) * ldL + (long)j * S + a] = cneg(cconj(g.lcc[(tri(t) + j) * s2 + ab]));
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
template <int S, class X = CtaExec>
__device__ void ret_start_block(const GroupDev &g, const ProbDev &p, int n, double2 *smem, const X &x = X()) {
    const int k = g.k, s2 = S * S, KS = k * S;
    const double h = g.h;
    double2 *mm = smem;                 // k*k blocks (block (p,q) at (p*k+q)*s2)
    double2 *qq = mm + k * k * s2;      // k blocks
    double2 *A = qq + k * s2;           // (KS x KS)
    double2 *R = A + KS * KS;           // (KS x S)
    int *ipiv = (int *)(R + KS * S);
    int *status = ipiv + 1;
    double2 *grow = p.gret + tri(n) * s2;  // G(n, .)
    for (int e = x.t(); e < k * k * s2; e += x.n()) mm[e] = cmk(0, 0);
    for (int e = x.t(); e < k * s2; e += x.n()) qq[e] = cmk(0, 0);
    if (x.t() == 0) *status = 0;
    x.sync();
    // thread per (row-block pr, element ab): fills block row pr of mm and qq(pr)
    for (int e = x.t(); e < k * s2; e += x.n()) {
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
    x.sync();
    // conjugate-transpose to a right solve: A[(pr,a),(q,b)] = conj(mm(pr,q)[b][a]),
    // R[(pr,a),c] = conj(qq(pr)[c][a])
    for (int e = x.t(); e < KS * KS; e += x.n()) {
        int r = e / KS, c = e % KS, pr = r / S, a = r % S, q = c / S, b = c % S;
        A[e] = cconj(mm[(pr * k + q) * s2 + b * S + a]);
    }
    for (int e = x.t(); e < KS * S; e += x.n()) {
        int r = e / S, c = e % S, pr = r / S, a = r % S;
        R[e] = cconj(qq[pr * s2 + c * S + a]);
    }
    x.sync();
    grp_solve(x, A, R, KS, S, ipiv, status);
    // X_q[a][c] = conj(Y[(q,c), a]) -> G(n, n-q-1)
    for (int e = x.t(); e < k * s2; e += x.n()) {
        int q = e / s2, ac = e % s2, a = ac / S, c = ac % S;
        grow[(long)(n - q - 1) * s2 + ac] = cconj(R[(q * S + c) * S + a]);
    }
    x.sync();
}

// VIE2 ret (vie2_timestep_ret, cntr_vie2_impl.hpp:60-140, called with F and Fcc swapped):
// unknowns X_q = G(n, n-q-1), q = 0..k-1, with G(n,n) = Q(n,n) set;
//   sum_q X_q mm(p,q) = qq(p),  mm(p,q) = 1 delta_pq + h w(j,l) F'(n-l, n-j) [l = q+1]
//   qq(p) = Q(n, n-j) - h w(j,0) G(n,n) F'(n, n-j),  j = p+1,
// F'(t,t') = Fcc^R(t,t') for t >= t' and F^R(t',t)^dagger otherwise (sign folded into w).
template <int S, class X = CtaExec>
__device__ void ret_start_block_vie(const GroupDev &g, const ProbDev &p, int n, double2 *smem, const X &x = X()) {
    const int k = g.k, s2 = S * S, KS = k * S;
    const double h = g.h;
    double2 *mm = smem;
    double2 *qq = mm + k * k * s2;
    double2 *A = qq + k * s2;
    double2 *R = A + KS * KS;
    int *ipiv = (int *)(R + KS * S);
    int *status = ipiv + 1;
    double2 *grow = p.gret + tri(n) * s2;
    for (int e = x.t(); e < k * k * s2; e += x.n()) mm[e] = cmk(0, 0);
    if (x.t() == 0) *status = 0;
    x.sync();
    for (int e = x.t(); e < k * s2; e += x.n()) {
        const int pr = e / s2, ab = e % s2, a = ab / S, b = ab % S, j = pr + 1;
        double2 q = p.qret[(tri(n) + n - j) * s2 + ab];
        if (a == b) mm[(pr * k + pr) * s2 + ab] = cadd(mm[(pr * k + pr) * s2 + ab], cmk(1.0, 0.0));
        for (int l = 0; l <= k; l++) {
            double w = -h * greg_w(k, j, l);
            if (l == 0) {
                // qq += w G(n,n) F'(n, n-j)
                const double2 *fr = g.rret + (tri(n) + n - j) * s2;
                double2 t = cmk(0, 0);
                for (int c = 0; c < S; c++) t = cfma(grow[(long)n * s2 + a * S + c], fr[c * S + b], t);
                q = cfma(cmk(w, 0.0), t, q);
            } else {
                double2 st;
                if (l <= j) st = g.rret[(tri(n - l) + n - j) * s2 + ab];
                else { st = cconj(g.sret[(tri(n - j) + n - l) * s2 + b * S + a]); w = -w; }
                const int idx = (pr * k + l - 1) * s2 + ab;
                mm[idx] = csub(mm[idx], cscale(st, w));
            }
        }
        qq[pr * s2 + ab] = q;
    }
    x.sync();
    for (int e = x.t(); e < KS * KS; e += x.n()) {
        int r = e / KS, c = e % KS, pr = r / S, a = r % S, q = c / S, b = c % S;
        A[e] = cconj(mm[(pr * k + q) * s2 + b * S + a]);
    }
    for (int e = x.t(); e < KS * S; e += x.n()) {
        int r = e / S, c = e % S, pr = r / S, a = r % S;
        R[e] = cconj(qq[pr * s2 + c * S + a]);
    }
    x.sync();
    grp_solve(x, A, R, KS, S, ipiv, status);
    for (int e = x.t(); e < k * s2; e += x.n()) {
        int q = e / s2, ac = e % s2, a = ac / S, c = ac % S;
        grow[(long)(n - q - 1) * s2 + ac] = cconj(R[(q * S + c) * S + a]);
    }
    x.sync();
}

// VIE2 les (vie2_timestep_les, cntr_vie2_impl.hpp:847-990): unknowns x_j = G^<(j,n), j = 0..k;
//   sum_m mm(j,m) x_m = gl(j) + Q^<(j,n),  mm(j,m) = 1 delta_jm + h w(j,m) F'(j,m),
// F'(j,m) = F^R(j,m) for j >= m and -Fcc^R(m,j)^dagger otherwise (right solve).
template <int S, class X = CtaExec>
__device__ void les_start_block_vie(const GroupDev &g, const ProbDev &p, int n, const double2 *gl, long ldc,
                                    double2 *xcol, double2 *smem, const X &x = X()) {
    const int k = g.k, K1 = k + 1, s2 = S * S, KS = K1 * S;
    const double h = g.h;
    double2 *A = smem;
    double2 *R = A + KS * KS;
    int *ipiv = (int *)(R + KS * S);
    int *status = ipiv + 1;
    if (x.t() == 0) *status = 0;
    for (int e = x.t(); e < K1 * s2; e += x.n()) {
        const int j = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        double2 q = gl[((long)j * S + a) * ldc + d];
        q = cadd(q, j <= n ? p.qles[(tri(n) + j) * s2 + ad] : cneg(cconj(p.qles[(tri(j) + n) * s2 + d * S + a])));
        R[(j * S + a) * S + d] = q;
        if (d == 0) {
            for (int m = 0; m <= k; m++) {
                const double w = h * greg_w(k, j, m);
                for (int b = 0; b < S; b++) {
                    double2 st = j >= m ? g.sret[(tri(j) + m) * s2 + a * S + b]
                                        : cneg(cconj(g.rret[(tri(m) + j) * s2 + b * S + a]));
                    double2 v = cscale(st, w);
                    if (m == j && a == b) v = cadd(v, cmk(1.0, 0.0));
                    A[(j * S + a) * KS + m * S + b] = v;
                }
            }
        }
    }
    x.sync();
    grp_solve(x, A, R, KS, S, ipiv, status);
    for (int e = x.t(); e < K1 * s2; e += x.n()) {
        const int j = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        xcol[(long)j * s2 + ad] = R[(j * S + a) * S + d];
    }
    x.sync();
}

// les: unknowns x_j = G^<(j,n), j = 1..k; sum_q mm(p,q) x_{q+1} = qq(p)  (right solve)
template <int S, class X = CtaExec>
__device__ void les_start_block(const GroupDev &g, const ProbDev &p, int n, const double2 *gl, long ldc,
                                double2 *xcol, double2 *smem, const X &x = X()) {
    const int k = g.k, s2 = S * S, KS = k * S;
    const double h = g.h;
    double2 *A = smem;           // (KS x KS)
    double2 *R = A + KS * KS;    // (KS x S)
    int *ipiv = (int *)(R + KS * S);
    int *status = ipiv + 1;
    if (x.t() == 0) *status = 0;
    for (int e = x.t(); e < KS * KS; e += x.n()) A[e] = cmk(0, 0);
    x.sync();
    // thread per (pr, a, d): qq(pr)[a][d] and the row (pr,a) of A
    for (int e = x.t(); e < k * s2; e += x.n()) {
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
    x.sync();
    grp_solve(x, A, R, KS, S, ipiv, status);
    for (int e = x.t(); e < k * s2; e += x.n()) {
        int q = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        xcol[(long)(q + 1) * s2 + ad] = R[(q * S + a) * S + d];
    }
    x.sync();
}

// ---------------------------------------------------------------------------------------
// k_tv: G^tv(n, tau) for one problem and a tile of tau (dyson_impl :651-741):
//   Q(tau) = sum_{j<n} a_j G^tv(j,tau) + dtau * matsubara_integral_2(Sigma^tv(n,.), G^mat)(tau)
//   G^tv(n,tau) = Minv_les[n] Q(tau)
// The Matsubara integral is linear in G^mat with an operator K_n built from Sigma^tv(n,.)
// alone (k_mat_operator), so for a group sharing Sigma it is one GEMM over all problems
// (Cmat = K_n Gmat_all); this kernel streams the history and adds Cmat.
// Thread per (tau, column d); the history G^tv(0..n-1, tile) is streamed once.
// ---------------------------------------------------------------------------------------
// k_tv works on the device layout of G^tv: element planes, (t*s^2 + e)*(ntau+1) + tau, so a
// warp reading 32 consecutive tau of one plane issues one contiguous 512-byte access.
template <int S> struct TvCfg {
    static constexpr int DCH = S <= 2 ? S : (S <= 4 ? 2 : 1);  // block columns per pass
    static constexpr int NW = 8;                // warps per CTA, splitting the history sum over j
};

// MIXED: history rows j < n-k-1 are read from the FP32 copy (half the bytes); the k+1 rows
// that carry the backward-difference terms, and all sums, stay in FP64.
// VIE2 (vie2_timestep_tv, cntr_vie2_impl.hpp:645-725): a_j and Cmat carry the minus sign of
// the convolution and Q^tv(n, tau) is added before the solve with (1 + h w0 F^R(n,n))^-1.
template <int S, bool MIXED, bool VIE = false>
__global__ void __launch_bounds__(256) k_tv(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    constexpr int s2 = S * S, DCH = TvCfg<S>::DCH, NW = TvCfg<S>::NW;
    __shared__ double2 red[NW * 32 * S * DCH];
    const ProbDev p = probs[blockIdx.y];
    const int ntau = g.ntau, M = ntau + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tau = blockIdx.x * 32 + lane;
    const bool live = tau <= ntau;
    const long rowstride = (long)s2 * M;
    for (int c0 = 0; c0 < S; c0 += DCH) {
        double2 acc[S][DCH];
#pragma unroll
        for (int a = 0; a < S; a++)
#pragma unroll
            for (int c = 0; c < DCH; c++) acc[a][c] = cmk(0, 0);
        if (live) {
            const double2 *gb = p.gtv + tau;
            const double2 *cf = g.tvcoef;
            const int j64 = MIXED ? (n - g.k - 1 > 0 ? n - g.k - 1 : 0) : 0;  // first FP64 row
            if (MIXED) {
                const float2 *gb32 = p.gtv32 + tau;
                // 8-byte loads: twice the rows in flight of the FP64 loop keep as many bytes in flight
#pragma unroll 8
                for (int j = warp; j < j64; j += NW) {
                    const float2 *gj = gb32 + (long)j * rowstride;
                    double2 bv[S][DCH];
#pragma unroll
                    for (int b = 0; b < S; b++)
#pragma unroll
                        for (int c = 0; c < DCH; c++) {
                            float2 f = (c0 + c < S) ? __ldg(gj + (long)(b * S + c0 + c) * M) : make_float2(0.f, 0.f);
                            bv[b][c] = cmk((double)f.x, (double)f.y);
                        }
                    const double2 *cj = cf + (long)j * s2;
#pragma unroll
                    for (int a = 0; a < S; a++)
#pragma unroll
                        for (int b = 0; b < S; b++) {
                            const double2 cab = __ldg(cj + a * S + b);
#pragma unroll
                            for (int c = 0; c < DCH; c++) acc[a][c] = cfma(cab, bv[b][c], acc[a][c]);
                        }
                }
            }
            const int jfirst = j64 + ((warp - j64 % NW) + NW) % NW;  // keep j = warp (mod NW)
#pragma unroll 4
            for (int j = jfirst; j < n; j += NW) {
                const double2 *gj = gb + (long)j * rowstride;
                double2 bv[S][DCH];
#pragma unroll
                for (int b = 0; b < S; b++)
#pragma unroll
                    for (int c = 0; c < DCH; c++)
                        bv[b][c] = (c0 + c < S) ? __ldg(gj + (long)(b * S + c0 + c) * M) : cmk(0, 0);
                const double2 *cj = cf + (long)j * s2;
#pragma unroll
                for (int a = 0; a < S; a++)
#pragma unroll
                    for (int b = 0; b < S; b++) {
                        const double2 cab = __ldg(cj + a * S + b);
#pragma unroll
                        for (int c = 0; c < DCH; c++) acc[a][c] = cfma(cab, bv[b][c], acc[a][c]);
                    }
            }
        }
#pragma unroll
        for (int a = 0; a < S; a++)
#pragma unroll
            for (int c = 0; c < DCH; c++) red[((warp * 32 + lane) * S + a) * DCH + c] = acc[a][c];
        __syncthreads();
        if (warp == 0 && live) {
#pragma unroll
            for (int a = 0; a < S; a++)
#pragma unroll
                for (int c = 0; c < DCH; c++) {
                    double2 v = red[(lane * S + a) * DCH + c];
                    for (int w = 1; w < NW; w++) v = cadd(v, red[((w * 32 + lane) * S + a) * DCH + c]);
                    acc[a][c] = v;
                }
            // Matsubara part dtau*[c2 + sig c1] from the group GEMM (k_mat_operator)
            const double2 *cm = g.Cmat + (long)tau * S * g.ldc + (long)p.col * S + c0;
#pragma unroll
            for (int a = 0; a < S; a++)
#pragma unroll
                for (int c = 0; c < DCH; c++)
                    if (c0 + c < S) acc[a][c] = cadd(acc[a][c], cm[(long)a * g.ldc + c]);
            if (VIE) {
                const double2 *qt = p.qtv + (long)n * rowstride + tau;
#pragma unroll
                for (int a = 0; a < S; a++)
#pragma unroll
                    for (int c = 0; c < DCH; c++)
                        if (c0 + c < S) acc[a][c] = cadd(acc[a][c], qt[(long)(a * S + c0 + c) * M]);
            }
            // solve: G^tv(n,tau)[a][d] = sum_b Minv[a][b] Q[b][d]
            const double2 *mi = p.minv_les + (long)n * s2;
            double2 *out = p.gtv + (long)n * rowstride + tau;
#pragma unroll
            for (int a = 0; a < S; a++)
#pragma unroll
                for (int c = 0; c < DCH; c++) {
                    if (c0 + c >= S) continue;
                    double2 x = cmk(0, 0);
#pragma unroll
                    for (int b = 0; b < S; b++) x = cfma(mi[a * S + b], acc[b][c], x);
                    out[(long)(a * S + c0 + c) * M] = x;
                    if (MIXED) p.gtv32[(long)n * rowstride + tau + (long)(a * S + c0 + c) * M] =
                        make_float2((float)x.x, (float)x.y);
                }
        }
        __syncthreads();
    }
}

// k_tv_to32: FP32 copy of G^tv rows [t0, t0+rows) (plane layout, same indexing)
__global__ void k_tv_to32(float2 *__restrict__ dst, const double2 *__restrict__ src, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

// k_tv_relayout: G^tv between libcntr's layout ((t*M + tau)*s^2 + e) and the element-plane
// layout ((t*s^2 + e)*M + tau) used on the device; rows t = 0..rows-1.
__global__ void k_tv_relayout(double2 *__restrict__ dst, const double2 *__restrict__ src, long rows, int M, int s2,
                              int to_planes) {
    const long total = rows * M * s2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
        // i indexes the plane layout: t, e, tau
        const long t = i / ((long)s2 * M);
        const int rem = (int)(i % ((long)s2 * M)), e = rem / M, tau = rem % M;
        const long j = (t * M + tau) * s2 + e;  // libcntr index
        if (to_planes) dst[i] = src[j]; else dst[j] = src[i];
    }
}

// ---------------------------------------------------------------------------------------
// k_mat_operator: K_n[(m,a),(x,c)] such that dtau * matsubara_integral_2(Sigma^tv(n,.), B)(m)
// = sum_x K_n[m,x] B(x) for every B (conv_impl :410-540 read as a linear map of B):
//   c2 = sum_{l=0}^{r} w(r,l) A(m+l) B(l)           (r = ntau-m >= k; rcorr for 0<r<k)
//   c1 = sum_{l=0}^{m} w(m,l) A(m-l) B(ntau-l)      (m >= k; rcorr for 0<m<k),  C = c2 + sig c1
// ---------------------------------------------------------------------------------------
// sgn = -1 for VIE2, whose Matsubara convolution enters the right-hand side with a minus sign.
template <int S>
__global__ void k_mat_operator(GroupDev g, int n, double sgn) {
    const int k = g.k, s2 = S * S, ntau = g.ntau, M = ntau + 1;
    const long KS = (long)M * S;
    const double2 *A = g.stv + (long)n * M * s2;
    const double dtau = g.beta / ntau, sg = (double)g.sig;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)M * M * s2; e += (long)gridDim.x * blockDim.x) {
        const int m = (int)(e / ((long)M * s2));
        const int rem = (int)(e % ((long)M * s2));
        const int x = rem / s2, ac = rem % s2, a = ac / S, c = ac % S;
        const int r = ntau - m;
        double2 v = cmk(0, 0);
        if (r >= k) {
            if (x <= r) v = cfma(cmk(greg_w(k, r, x), 0), A[(long)(m + x) * s2 + ac], v);
        } else if (r > 0 && x <= k) {
            for (int l = 0; l <= k; l++) v = cfma(cmk(rcorr_w(k, r, l, x), 0), A[(long)(ntau - l) * s2 + ac], v);
        }
        const int l = ntau - x;
        if (m >= k) {
            if (l >= 0 && l <= m) v = cfma(cmk(sg * greg_w(k, m, l), 0), A[(long)(m - l) * s2 + ac], v);
        } else if (m > 0 && l >= 0 && l <= k) {
            for (int jj = 0; jj <= k; jj++) v = cfma(cmk(sg * rcorr_w(k, m, l, jj), 0), A[(long)jj * s2 + ac], v);
        }
        g.Kmat[((long)m * S + a) * KS + (long)x * S + c] = cscale(v, dtau * sgn);
    }
}

// k_gmat_stack: Gmat_all[(x,c)][(col,d)] = G^mat_col(x)[c][d]
template <int S>
__global__ void k_gmat_stack(GroupDev g, const ProbDev *__restrict__ probs) {
    const ProbDev p = probs[blockIdx.y];
    const int s2 = S * S, M = g.ntau + 1;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < M * s2; e += gridDim.x * blockDim.x) {
        const int x = e / s2, cd = e % s2, c = cd / S, d = cd % S;
        g.Gmat_all[((long)x * S + c) * g.ldc + (long)p.col * S + d] = p.gmat[e];
    }
}

// ---------------------------------------------------------------------------------------
// k_les_operands_t: right-hand operands of the Sigma-shared products (conv_impl :1075-1394)
//   badv[(m,c)][(col,d)] = h w(n,m) G^R(n,m)^dagger[c][d],                 m = 0..n
//   btv [(m,c)][(col,d)] = w(ntau,m) (-i dtau)(-sig) G^tv(n,ntau-m)^dagger[c][d]
// badv / btv are row-major with the problems side by side in a row, so one problem's column is
// a strided write; a CTA takes a tile of LOT problems x LOR time indices, reads each problem's
// contiguous slice into shared memory and writes whole row segments (coalesced).
//   which = 1: badv rows m = 0..n (from G^R(n, m)); which = 2: btv rows m = 0..ntau (from G^tv(n, .))
// ---------------------------------------------------------------------------------------
#define LOT 32
template <int S> struct LoCfg {
    static constexpr int LOR = S == 1 ? 32 : (S == 2 ? 16 : (S <= 4 ? 4 : 1));  // time indices per tile
};

template <int S>
__global__ void __launch_bounds__(256) k_les_operands_t(GroupDev g, const ProbDev *__restrict__ probs, int n,
                                                        int which, int nact) {
    constexpr int s2 = S * S, LOR = LoCfg<S>::LOR;
    __shared__ double2 buf[LOT * LOR * s2 + LOT];
    __shared__ const double2 *src[LOT];
    __shared__ int colid[LOT];
    const int k = g.k, ntau = g.ntau, M = ntau + 1;
    const double h = g.h, dtau = g.beta / ntau;
    const long ldc = g.ldc;
    const int q0 = blockIdx.y * LOT, nq = min(LOT, nact - q0);
    const int m0 = blockIdx.x * LOR, rows = which == 1 ? n + 1 : M, nm = min(LOR, rows - m0);
    if (threadIdx.x < LOT) {
        const int q = threadIdx.x;
        src[q] = q < nq ? (which == 1 ? probs[q0 + q].gret + tri(n) * s2 : probs[q0 + q].gtv + (long)n * s2 * M)
                        : nullptr;
        colid[q] = q < nq ? probs[q0 + q].col : 0;
    }
    __syncthreads();
    // gather: buf[(q*LOR + mm)*s2 + e] = G element e of problem q at time index m0+mm
    for (int i = threadIdx.x; i < nq * nm * s2; i += blockDim.x) {
        if (which == 1) {
            const int q = i / (nm * s2), rem = i % (nm * s2), mm = rem / s2, e = rem % s2;
            buf[(q * LOR + mm) * s2 + e] = src[q][(long)(m0 + mm) * s2 + e];     // ret row n, contiguous
        } else {
            const int q = i / (nm * s2), rem = i % (nm * s2), e = rem / nm, mm = rem % nm;
            buf[(q * LOR + mm) * s2 + e] = src[q][(long)e * M + (ntau - (m0 + mm))];  // tv planes
        }
    }
    __syncthreads();
    // scatter: row (m, c), columns (col, d) of this tile
    for (int i = threadIdx.x; i < nm * S * nq * S; i += blockDim.x) {
        const int r = i / (nq * S), cc = i % (nq * S), mm = r / S, c = r % S, q = cc / S, d = cc % S;
        const int m = m0 + mm;
        const double2 v = cconj(buf[(q * LOR + mm) * s2 + d * S + c]);
        const long dst = ((long)m * S + c) * ldc + (long)colid[q] * S + d;
        if (which == 1) g.badv[dst] = cscale(v, h * greg_w(k, n, m));
        else g.btv[dst] = cmul(cmk(0.0, dtau * (double)g.sig * greg_w(k, ntau, m)), v);
    }
}

#include "kernels_volterra.cuh"
#include "kernels_volterra_mp.cuh"
#include "kernels_volterra_cl.cuh"
