// Volterra recursions of one Dyson / VIE2 time step for a whole Sigma group, as a blocked
// right-looking triangular solve run by thread-block clusters.
//
//   ret  G^R(n, j), j = n-k-1 .. 0     dyson_impl :158-213, vie2_impl :60-140
//        x(j) M_j = h sum_{m>j} w(n-j, n-m) x(m) Sigma^R(m, j) - bdf(j)        (Dyson)
//        x(j) M_j = Q(n, j) - h sum_{m>j} w(n-j, n-m) x(m) Fcc^R(m, j)          (VIE2)
//   les  G^<(j, n), j = k+1 .. n       dyson_impl :983-1011, vie2_impl :847-990
//        M_j x(j) = gl(j) + h sum_{m<j} w(j, m) Sigma^R(j, m) x(m) - bdf(j)     (Dyson)
//        M_j x(j) = gl(j) + Q^<(j, n) - h sum_{m<j} w(j, m) F^R(j, m) x(m)      (VIE2)
//
// For rows j > k the Gregory weight is w(N, i) = a_i + a_{N-i} - 1 with a_i = omega_i (i <= k)
// or 1 (integration.hpp:382-390, and the overlap rows k < N < 2k+2 below it), so for |m - j| > k
// it depends on m alone: c_m = a_{n-m} (ret) or a_m (les).  The unknowns are solved in blocks of
// JB rows.  After a block is solved, its rows m enter the sums of every later row j as ONE
// complex GEMM over the problems of the group (columns (p, .)) with the column weight c_m (the
// "trailing update"); the <= k rows next to a block are corrected to the exact weight when the
// next block is solved, and the block's own pairs use exact weights in the in-block chain.  The
// first block takes the start rows with exact weights directly.
//
// One cluster of CL CTAs owns PT problems (their GEMM columns) for the whole recursion:
//   phase D  warp per problem: exact start / near terms + accumulated far sum -> in-block chain,
//            writes x into G and the block's rows, times their column weight, into the panel
//   cluster barrier
//   phase G  the cluster's 2 CL tile groups run the trailing GEMM tiles over the remaining rows
//   cluster barrier
// Data written by another CTA of the cluster (panel, accumulators) are read with ld.global.cg.
#pragma once
#include "kernels_gemm.cuh"

template <int S> struct ClCfg {
    static constexpr int JB = S <= 2 ? 32 : (S <= 4 ? 16 : 8);  // rows per block (>= k+1)
    static constexpr int s2 = S * S;
    static constexpr int TRI = JB * (JB - 1) / 2;     // packed strictly-lower block triangle
    static constexpr int DWMAX = S <= 2 ? 8 : 2;      // chain warps (problems) per CTA
    // per-warp state of the element-parallel chain (S >= 3): A, MI, GV (JB s2 each), X window
    // ((JB + K1MAX) s2), Q (s2)
    static constexpr int WS = (3 * JB + NESSI_K1MAX + 1) * s2;
    static constexpr int PANEL_ROWS = JB + NESSI_K1MAX;  // rows of the largest panel (block 0)
};

__device__ __forceinline__ void cl_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ unsigned cl_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cl_nrank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ double2 ldcg2(const double2 *p) { return __ldcg(p); }
__device__ __forceinline__ unsigned long long global_ns_cl() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- trailing-update operands -------------------------------------------------------------
// ret: A(r = (j, d), kk = (i, b)) = T(m = mlo + i, j)[b][d] (triangle rows m, contiguous in j)
template <int S> struct LdRetTri {
    static constexpr bool KC = false;
    const double2 *tri_;
    int mlo, M, K;
    __device__ __forceinline__ double2 get(int r, int kk) const {
        if (r >= M || kk >= K) return cmk(0, 0);
        const int j = r / S, d = r % S, m = mlo + kk / S, b = kk % S;
        return __ldg(tri_ + (tri(m) + j) * (S * S) + b * S + d);
    }
};
// les: A(r = (j, a), kk = (i, b)) = T(j = j0 + r/S, m = mlo + i)[a][b] (triangle row j, contiguous in m)
template <int S> struct LdLesTri {
    static constexpr bool KC = true;
    const double2 *tri_;
    int j0, mlo, M, K;
    __device__ __forceinline__ double2 get(int r, int kk) const {
        if (r >= M || kk >= K) return cmk(0, 0);
        const int j = j0 + r / S, a = r % S, m = mlo + kk / S, b = kk % S;
        return __ldg(tri_ + (tri(j) + m) * (S * S) + a * S + b);
    }
};
// B(kk, c) = panel[kk * ld + c] for columns c < cmax (written by other CTAs of the cluster)
struct LdPanel {
    static constexpr bool KC = false;
    const double2 *p;
    long ld;
    int cmax, K;
    __device__ __forceinline__ double2 get(int c, int kk) const {
        return (c < cmax && kk < K) ? ldcg2(p + (long)kk * ld + c) : cmk(0, 0);
    }
};
// C[r][c] (+)= v for r < M, c < cmax (the accumulators, read back through L2)
struct StCl {
    double2 *p;
    long ld;
    int M, cmax, accumulate;
    __device__ __forceinline__ bool accumulates() const { return accumulate != 0; }
    __device__ __forceinline__ double2 load(int r, int c) const {
        return (r < M && c < cmax) ? ldcg2(p + (long)r * ld + c) : cmk(0, 0);
    }
    __device__ __forceinline__ double2 combine(double2 old, double2 v) const { return cadd(old, v); }
    __device__ __forceinline__ void store(int r, int c, double2 x) const {
        if (r < M && c < cmax) p[(long)r * ld + c] = x;
    }
};

// ---- phase D, size1 <= 2: lane r owns block row r (register chains) -------------------------
// lesser chain of one block (as mp_les_chain; gl read through L2)
template <int S, bool VIE>
__device__ void cl_les_chain(double2 *a_, const double2 *sig, const double *wb, const ProbDev &p, const double2 *gl,
                             long ldc, double2 *xcol, int n, int jlo, int nb, int K1, const double2 *ibd, double h,
                             int lane) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
    double2 bd[s2], mi[s2], gv[s2];
#pragma unroll
    for (int e = 0; e < s2; e++) {
        const int a = e / S, d = e % S;
        mi[e] = own ? p.minv_les[(long)(jlo + r) * s2 + e] : cmk(0, 0);
        gv[e] = own ? ldcg2(gl + ((long)(jlo + r) * S + a) * ldc + d) : cmk(0, 0);
        if (VIE && own) gv[e] = cadd(gv[e], p.qles[(tri(n) + jlo + r) * s2 + e]);
        bd[e] = cmk(0, 0);
    }
    if (own && !VIE)
        for (int pp = 1; pp <= K1; pp++)
            if (r - pp < 0)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[pp], xcol[(long)(jlo + r - pp) * s2 + e], bd[e]);
    for (int rr = 0; rr < nb; rr++) {
        double2 x[s2];
        if (r == rr) {
            double2 q[s2];
#pragma unroll
            for (int e = 0; e < s2; e++)
                q[e] = VIE ? cfma(cmk(-h, 0.0), a_[e], gv[e]) : csub(cfma(cmk(h, 0.0), a_[e], gv[e]), bd[e]);
#pragma unroll
            for (int aa = 0; aa < S; aa++)
#pragma unroll
                for (int d = 0; d < S; d++) {
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) t = cfma(mi[aa * S + bb], q[bb * S + d], t);
                    x[aa * S + d] = t;
                }
        }
        shfl_blk<S>(x, rr);
        if (r == rr)
#pragma unroll
            for (int e = 0; e < s2; e++) xcol[(long)(jlo + rr) * s2 + e] = x[e];
        if (r > rr && own) {
            const int q = pk(r, rr);
            const double w = wb[q];
            const double2 *sg = sig + q * s2;
#pragma unroll
            for (int aa = 0; aa < S; aa++)
#pragma unroll
                for (int d = 0; d < S; d++) {
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) t = cfma(sg[aa * S + bb], x[bb * S + d], t);
                    a_[aa * S + d] = cfma(cmk(w, 0.0), t, a_[aa * S + d]);
                }
            if (!VIE && r - rr <= K1)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[r - rr], x[e], bd[e]);
        }
    }
}

// ret block (size1 <= 2): far sum from the accumulators (or, for block 0, the exact terms of the
// start rows), near corrections, chain, panel rows c_m x(m)[a][b] at [(i, b)][(col, a)]
template <int S, bool VIE>
__device__ void cl_ret_diag_small(const GroupDev &g, const ProbDev &p, int n, int b, int jlo, int jhi, int nb,
                                  const double2 *accr, const double2 *sig, const double *wb, const double2 *ibd,
                                  double2 *panel, int lane) {
    constexpr int s2 = S * S;
    const int k = g.k, K1 = k + 1;
    const long ldc = g.ldc;
    double2 *grow = p.gret + tri(n) * s2;
    const int r = lane, j = jlo + r;
    double2 a_[s2];
#pragma unroll
    for (int e = 0; e < s2; e++) a_[e] = cmk(0, 0);
    if (r < nb) {
        int mhi;
        if (b == 0) {
            mhi = n;  // all rows above the first block, exact weights
        } else {
#pragma unroll
            for (int e = 0; e < s2; e++) {
                const int a = e / S, d = e % S;
                a_[e] = ldcg2(accr + ((long)j * S + d) * ldc + (long)p.col * S + a);
            }
            mhi = min(jhi + k, n);  // near rows of the block above: weight minus c_m = 1
        }
        for (int m = jhi + 1; m <= mhi; m++) {
            if (b > 0 && m - j > k) continue;
            const double w = greg_w(k, n - j, n - m) - (b > 0 ? 1.0 : 0.0);
            const double2 *gm = grow + (long)m * s2, *sm = g.rret + (tri(m) + j) * s2;
#pragma unroll
            for (int aa = 0; aa < S; aa++)
#pragma unroll
                for (int d = 0; d < S; d++) {
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) t = cfma(gm[aa * S + bb], sm[bb * S + d], t);
                    a_[aa * S + d] = cfma(cmk(w, 0.0), t, a_[aa * S + d]);
                }
        }
    }
    mp_ret_chain<S, VIE>(a_, sig, wb, p, grow, n, jlo, nb, K1, ibd, g.h, lane);
    __syncwarp();
    const int rows = b == 0 ? n - jlo + 1 : nb;
    for (int i = lane; i < rows; i += 32) {
        const int m = jlo + i;
        const double cm = n - m <= k ? greg_omega(k, n - m) : 1.0;
#pragma unroll
        for (int e = 0; e < s2; e++) {
            const int a = e / S, bb = e % S;
            panel[((long)i * S + bb) * ldc + (long)p.col * S + a] = cscale(grow[(long)m * s2 + e], cm);
        }
    }
}

// les block (size1 <= 2): far sum from the accumulators (block 0: exact terms of the start rows),
// near corrections, chain, panel rows c'_m x(m)[b][d] at [(i, b)][(col, d)]
template <int S, bool VIE>
__device__ void cl_les_diag_small(const GroupDev &g, const ProbDev &p, int n, int b, int jlo, int jhi, int nb,
                                  const double2 *accl, const double2 *sig, const double *wb, const double2 *ibd,
                                  double2 *panel, int lane) {
    constexpr int s2 = S * S;
    const int k = g.k, K1 = k + 1;
    const long ldc = g.ldc;
    double2 *xcol = p.gles + tri(n) * s2;
    const int r = lane, j = jlo + r;
    double2 a_[s2];
#pragma unroll
    for (int e = 0; e < s2; e++) a_[e] = cmk(0, 0);
    if (r < nb) {
        int mlo;
        if (b == 0) {
            mlo = 0;  // the start rows 0..k, exact weights
        } else {
#pragma unroll
            for (int e = 0; e < s2; e++) {
                const int a = e / S, d = e % S;
                a_[e] = ldcg2(accl + ((long)j * S + a) * ldc + (long)p.col * S + d);
            }
            mlo = max(0, jlo - k);  // near rows of the block below: weight minus c'_m = 1
        }
        for (int m = mlo; m < jlo; m++) {
            if (b > 0 && j - m > k) continue;
            const double w = greg_w(k, j, m) - (b > 0 ? 1.0 : 0.0);
            const double2 *sm = g.sret + (tri(j) + m) * s2, *xm = xcol + (long)m * s2;
#pragma unroll
            for (int aa = 0; aa < S; aa++)
#pragma unroll
                for (int d = 0; d < S; d++) {
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) t = cfma(sm[aa * S + bb], xm[bb * S + d], t);
                    a_[aa * S + d] = cfma(cmk(w, 0.0), t, a_[aa * S + d]);
                }
        }
    }
    cl_les_chain<S, VIE>(a_, sig, wb, p, g.gles + (long)p.col * S, ldc, xcol, n, jlo, nb, K1, ibd, g.h, lane);
    __syncwarp();
    const int m0 = b == 0 ? 0 : jlo, rows = jhi - m0 + 1;
    for (int i = lane; i < rows; i += 32) {
        const int m = m0 + i;
        const double cm = m <= k ? greg_omega(k, m) : 1.0;
#pragma unroll
        for (int e = 0; e < s2; e++) {
            const int bb = e / S, d = e % S;
            panel[((long)i * S + bb) * ldc + (long)p.col * S + d] = cscale(xcol[(long)m * s2 + e], cm);
        }
    }
}

// ---- phase D, size1 >= 3: lanes over the s x s elements, rows in sequence ------------------
template <int S, bool VIE>
__device__ void cl_ret_diag_big(const GroupDev &g, const ProbDev &p, int n, int b, int jlo, int jhi, int nb,
                                const double2 *accr, const double2 *sig, const double *wb, const double2 *ibd,
                                double2 *panel, double2 *ws, int lane) {
    constexpr int s2 = S * S, JB = ClCfg<S>::JB;
    const int k = g.k, K1 = k + 1;
    const long ldc = g.ldc;
    const double h = g.h;
    double2 *A = ws, *MI = A + JB * s2, *X = MI + 2 * JB * s2, *Q = X + (JB + NESSI_K1MAX) * s2;
    double2 *grow = p.gret + tri(n) * s2;
    for (int idx = lane; idx < nb * s2; idx += 32) {
        const int r = idx / s2, e = idx % s2, a = e / S, d = e % S, j = jlo + r;
        double2 v = b == 0 ? cmk(0, 0) : ldcg2(accr + ((long)j * S + d) * ldc + (long)p.col * S + a);
        const int mhi = b == 0 ? n : min(jhi + k, n);
        for (int m = jhi + 1; m <= mhi; m++) {
            if (b > 0 && m - j > k) continue;
            const double w = greg_w(k, n - j, n - m) - (b > 0 ? 1.0 : 0.0);
            double2 t = cmk(0, 0);
#pragma unroll
            for (int bb = 0; bb < S; bb++)
                t = cfma(grow[(long)m * s2 + a * S + bb], g.rret[(tri(m) + j) * s2 + bb * S + d], t);
            v = cfma(cmk(w, 0.0), t, v);
        }
        A[idx] = v;
        MI[idx] = p.minv_ret[(long)j * s2 + e];
    }
    for (int idx = lane; idx < K1 * s2; idx += 32) X[nb * s2 + idx] = grow[(long)(jhi + 1) * s2 + idx];
    __syncwarp();
    for (int r = nb - 1; r >= 0; r--) {
        const int j = jlo + r;
        for (int e = lane; e < s2; e += 32) {
            double2 q;
            if (VIE) {
                q = csub(p.qret[(tri(n) + j) * s2 + e], cscale(A[r * s2 + e], h));
            } else {
                q = cscale(A[r * s2 + e], h);
                for (int pp = 1; pp <= K1; pp++) q = csub(q, cmul(ibd[pp], X[(r + pp) * s2 + e]));
            }
            Q[e] = q;
        }
        __syncwarp();
        for (int e = lane; e < s2; e += 32) {
            const int a = e / S, d = e % S;
            double2 x = cmk(0, 0);
#pragma unroll
            for (int bb = 0; bb < S; bb++) x = cfma(Q[a * S + bb], MI[r * s2 + bb * S + d], x);
            X[r * s2 + e] = x;
            grow[(long)j * s2 + e] = x;
        }
        __syncwarp();
        for (int idx = lane; idx < r * s2; idx += 32) {
            const int r2 = idx / s2, e = idx % s2, a = e / S, d = e % S, q = pk(r, r2);
            double2 t = cmk(0, 0);
#pragma unroll
            for (int bb = 0; bb < S; bb++) t = cfma(X[r * s2 + a * S + bb], sig[q * s2 + bb * S + d], t);
            A[idx] = cfma(cmk(wb[q], 0.0), t, A[idx]);
        }
        __syncwarp();
    }
    const int rows = b == 0 ? n - jlo + 1 : nb;
    for (int idx = lane; idx < rows * s2; idx += 32) {
        const int i = idx / s2, e = idx % s2, a = e / S, bb = e % S, m = jlo + i;
        const double cm = n - m <= k ? greg_omega(k, n - m) : 1.0;
        panel[((long)i * S + bb) * ldc + (long)p.col * S + a] = cscale(grow[(long)m * s2 + e], cm);
    }
}

template <int S, bool VIE>
__device__ void cl_les_diag_big(const GroupDev &g, const ProbDev &p, int n, int b, int jlo, int jhi, int nb,
                                const double2 *accl, const double2 *sig, const double *wb, const double2 *ibd,
                                double2 *panel, double2 *ws, int lane) {
    constexpr int s2 = S * S, JB = ClCfg<S>::JB;
    const int k = g.k, K1 = k + 1;
    const long ldc = g.ldc;
    const double h = g.h;
    double2 *A = ws, *MI = A + JB * s2, *GV = MI + JB * s2, *X = GV + JB * s2, *Q = X + (JB + NESSI_K1MAX) * s2;
    double2 *xcol = p.gles + tri(n) * s2;
    const double2 *gl = g.gles + (long)p.col * S;
    for (int idx = lane; idx < nb * s2; idx += 32) {
        const int r = idx / s2, e = idx % s2, a = e / S, d = e % S, j = jlo + r;
        double2 v = b == 0 ? cmk(0, 0) : ldcg2(accl + ((long)j * S + a) * ldc + (long)p.col * S + d);
        const int mlo = b == 0 ? 0 : max(0, jlo - k);
        for (int m = mlo; m < jlo; m++) {
            if (b > 0 && j - m > k) continue;
            const double w = greg_w(k, j, m) - (b > 0 ? 1.0 : 0.0);
            double2 t = cmk(0, 0);
#pragma unroll
            for (int bb = 0; bb < S; bb++)
                t = cfma(g.sret[(tri(j) + m) * s2 + a * S + bb], xcol[(long)m * s2 + bb * S + d], t);
            v = cfma(cmk(w, 0.0), t, v);
        }
        A[idx] = v;
        MI[idx] = p.minv_les[(long)j * s2 + e];
        double2 gv = ldcg2(gl + ((long)j * S + a) * ldc + d);
        if (VIE) gv = cadd(gv, p.qles[(tri(n) + j) * s2 + e]);
        GV[idx] = gv;
    }
    for (int idx = lane; idx < K1 * s2; idx += 32) X[idx] = xcol[(long)(jlo - K1) * s2 + idx];
    __syncwarp();
    for (int r = 0; r < nb; r++) {
        const int j = jlo + r;
        for (int e = lane; e < s2; e += 32) {
            double2 q = cfma(cmk(VIE ? -h : h, 0.0), A[r * s2 + e], GV[r * s2 + e]);
            if (!VIE)
                for (int pp = 1; pp <= K1; pp++) q = csub(q, cmul(ibd[pp], X[(K1 + r - pp) * s2 + e]));
            Q[e] = q;
        }
        __syncwarp();
        for (int e = lane; e < s2; e += 32) {
            const int a = e / S, d = e % S;
            double2 x = cmk(0, 0);
#pragma unroll
            for (int bb = 0; bb < S; bb++) x = cfma(MI[r * s2 + a * S + bb], Q[bb * S + d], x);
            X[(K1 + r) * s2 + e] = x;
            xcol[(long)j * s2 + e] = x;
        }
        __syncwarp();
        for (int idx = lane; idx < (nb - 1 - r) * s2; idx += 32) {
            const int r2 = r + 1 + idx / s2, e = idx % s2, a = e / S, d = e % S, q = pk(r2, r);
            double2 t = cmk(0, 0);
#pragma unroll
            for (int bb = 0; bb < S; bb++) t = cfma(sig[q * s2 + a * S + bb], X[(K1 + r) * s2 + bb * S + d], t);
            A[r2 * s2 + e] = cfma(cmk(wb[q], 0.0), t, A[r2 * s2 + e]);
        }
        __syncwarp();
    }
    const int m0 = b == 0 ? 0 : jlo, rows = jhi - m0 + 1;
    for (int idx = lane; idx < rows * s2; idx += 32) {
        const int i = idx / s2, e = idx % s2, bb = e / S, d = e % S, m = m0 + i;
        const double cm = m <= k ? greg_omega(k, m) : 1.0;
        panel[((long)i * S + bb) * ldc + (long)p.col * S + d] = cscale(xcol[(long)m * s2 + e], cm);
    }
}

// ---- the cluster kernel ----------------------------------------------------------------------
// Dynamic shared memory: max(GEMM stages of the two tile groups, block triangle + weights +
// per-warp chain state).
template <int S> struct ClSmem {
    static constexpr int sig = 0;                                        // TRI s2
    static constexpr int wb = sig + ClCfg<S>::TRI * S * S;               // TRI doubles
    static constexpr int ws = wb + ClCfg<S>::TRI / 2 + 1;                // per-warp state (S >= 3)
    static constexpr int diag = ws + (S <= 2 ? 0 : ClCfg<S>::DWMAX * ClCfg<S>::WS);
};
template <int BN> struct ClGemm {
    static constexpr int BM = BN == 64 ? 64 : 128;
    static constexpr int smem = 2 * zg::Smem<BM, BN>::total;  // two tile groups
};

// The block loop of one group of CTAs (a cluster, or the whole grid of a cooperative launch)
// owning the problems p0 .. p0+np-1 of the group (group order = descending nt, so the active
// problems are a prefix); PT >= np sets the chain warps per CTA.  acc: far-sum accumulators, rows
// (t, .) x columns (p, .), leading dimension ldc (ret: [(j, d)][(p, a)], les: [(j, a)][(p, d)]);
// panel: the solved block's weighted rows.  Every CTA runs the same block loop, so all reach every
// barrier; SY provides rank(), nrank() and sync() (false: a bounded wait gave up, leave the loop).
template <int S, bool VIE, bool RET, int BN, class SY>
__device__ __forceinline__ void volterra_blocked(const GroupDev &g, const ProbDev *__restrict__ probs, int n, int p0,
                                                 int np, int PT, double2 *acc, double2 *panel, const SY &sy) {
    extern __shared__ double2 smem[];
    constexpr int s2 = S * S, JB = ClCfg<S>::JB, BM = ClGemm<BN>::BM;
    constexpr int DW = ClCfg<S>::DWMAX;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rank = sy.rank(), CL = sy.nrank();
    const int cmax = (p0 + np) * S, c0 = p0 * S;  // GEMM columns of the group of CTAs
    const int k = g.k, K1 = k + 1;
    const double h = g.h;
    const long ldc = g.ldc;
    double2 *sig = smem + ClSmem<S>::sig;
    double *wb = (double *)(smem + ClSmem<S>::wb);
    __shared__ double2 ibd[NESSI_K1MAX + 1];
    if (tid <= NESSI_K1MAX) ibd[tid] = cmk(0.0, tid <= K1 ? bd_w(k, tid) / h : 0.0);
    // problem of this warp in phase D
    const int dwarps = (PT + CL - 1) / CL;  // <= DW by the host's choice of PT
    const int lp = rank * dwarps + warp;
    const bool owner = warp < dwarps && warp < DW && lp < np;
    ProbDev p;
    if (owner) p = probs[p0 + lp];
    const int nrows = n - k;  // unknowns: ret j = 0..n-k-1, les j = k+1..n
    const int nblk = (nrows + JB - 1) / JB;
    for (int b = 0; b < nblk; b++) {
        int jlo, jhi;
        if (RET) { jhi = n - k - 1 - b * JB; jlo = max(0, jhi - JB + 1); }
        else { jlo = K1 + b * JB; jhi = min(n, jlo + JB - 1); }
        const int nb = jhi - jlo + 1;
        // block triangle of Sigma and its exact weights, shared by the CTA's chains
        for (int e = tid; e < ClCfg<S>::TRI * s2; e += 256) {
            const int q = e / s2, ab = e % s2;
            int r, r2;
            pk_inv(q, r, r2);
            if (r < nb) {
                if (RET) {
                    sig[e] = g.rret[(tri(jlo + r) + jlo + r2) * s2 + ab];
                    if (ab == 0) wb[q] = greg_w(k, n - (jlo + r2), n - (jlo + r));
                } else {
                    sig[e] = g.sret[(tri(jlo + r) + jlo + r2) * s2 + ab];
                    if (ab == 0) wb[q] = greg_w(k, jlo + r, jlo + r2);
                }
            }
        }
        __syncthreads();
        if (owner) {
            if constexpr (S <= 2) {
                if (RET) cl_ret_diag_small<S, VIE>(g, p, n, b, jlo, jhi, nb, acc, sig, wb, ibd, panel, lane);
                else cl_les_diag_small<S, VIE>(g, p, n, b, jlo, jhi, nb, acc, sig, wb, ibd, panel, lane);
            } else {
                double2 *ws = smem + ClSmem<S>::ws + warp * ClCfg<S>::WS;
                if (RET) cl_ret_diag_big<S, VIE>(g, p, n, b, jlo, jhi, nb, acc, sig, wb, ibd, panel, ws, lane);
                else cl_les_diag_big<S, VIE>(g, p, n, b, jlo, jhi, nb, acc, sig, wb, ibd, panel, ws, lane);
            }
        }
        if (!sy.sync()) return;
        if (b + 1 == nblk) break;
        // phase G: trailing update of every row still to be solved
        {
            const int grp = warp >> 2, t = tid & 127;
            const int kpan = RET ? (b == 0 ? n - jlo + 1 : nb) : (b == 0 ? jhi + 1 : nb);
            const int M = (RET ? jlo : n - jhi) * S, K = kpan * S;
            const int ntn = (cmax - c0 + BN - 1) / BN, ntm = (M + BM - 1) / BM;
            LdPanel lb{panel, ldc, cmax, K};
            double2 *gsm = smem + grp * zg::Smem<BM, BN>::total;
            for (int tile = rank * 2 + grp; tile < ntm * ntn; tile += 2 * CL) {
                const int tm = tile / ntn, tn = tile % ntn;
                if (RET) {
                    LdRetTri<S> la{g.rret, jlo, M, K};
                    StCl st{acc, ldc, M, cmax, b > 0};
                    zgemm_tile<BM, BN>(la, lb, st, tm * BM, c0 + tn * BN, K, gsm, t, grp);
                } else {
                    LdLesTri<S> la{g.sret, jhi + 1, b == 0 ? 0 : jlo, M, K};
                    StCl st{acc + (long)(jhi + 1) * S * ldc, ldc, M, cmax, b > 0};
                    zgemm_tile<BM, BN>(la, lb, st, tm * BM, c0 + tn * BN, K, gsm, t, grp);
                }
            }
        }
        if (!sy.sync()) return;
    }
}

struct ClusterSync {
    __device__ __forceinline__ int rank() const { return (int)cl_rank(); }
    __device__ __forceinline__ int nrank() const { return (int)cl_nrank(); }
    __device__ __forceinline__ bool sync() const {
        cl_sync();
        return true;
    }
};

// Grid: CL x nclusters CTAs of 256 threads (cluster dimension CL along x); cluster c owns the
// problems c*PT .. min(nact, (c+1)*PT)-1 of the group.
template <int S, bool VIE, bool RET, int BN>
__global__ void __launch_bounds__(256, 1) k_volterra_cl(GroupDev g, const ProbDev *__restrict__ probs, int n,
                                                        int nact, int PT, double2 *acc, double2 *panel) {
    const int p0 = (int)(blockIdx.x / cl_nrank()) * PT;
    volterra_blocked<S, VIE, RET, BN>(g, probs, n, p0, min(PT, nact - p0), PT, acc, panel, ClusterSync{});
}

// Barrier of all CTAs of a cooperative launch (all resident at once): an arrival counter and a
// generation word in global memory; thread 0 of each CTA arrives and waits, bounded by limit_ns of
// %globaltimer.  A wait that gives up sets *err = NESSI_ERR_TIMEOUT and *abort = 1; a waiter that
// sees *abort gives up too, and the kernel returns from its block loop.  count and abort are zero
// at launch (the host clears them before every launch).  Data written before the barrier by other
// CTAs are read after it through L2 (ld.global.cg), as in the cluster form.
struct GridSync {
    unsigned *count, *gen;
    int *abort, *err;
    long long limit_ns;
    __device__ __forceinline__ int rank() const { return (int)blockIdx.x; }
    __device__ __forceinline__ int nrank() const { return (int)gridDim.x; }
    __device__ bool sync() const {
        __shared__ int s_ok;
        __syncthreads();
        if (threadIdx.x == 0) {
            int ok = 1;
            const unsigned g0 = *(volatile unsigned *)gen;
            __threadfence();
            if (atomicAdd(count, 1u) == gridDim.x - 1) {
                atomicExch(count, 0u);
                __threadfence();
                atomicAdd(gen, 1u);
            } else {
                const unsigned long long t0 = global_ns_cl();
                while (*(volatile unsigned *)gen == g0) {
                    if (*(volatile int *)abort) { ok = 0; break; }
                    if ((long long)(global_ns_cl() - t0) > limit_ns) {
                        atomicExch(err, 5);  // NESSI_ERR_TIMEOUT
                        atomicExch(abort, 1);
                        ok = 0;
                        break;
                    }
                    __nanosleep(32);
                }
            }
            __threadfence();
            if (*(volatile int *)abort) ok = 0;
            s_ok = ok;
        }
        __syncthreads();
        return s_ok != 0;
    }
};

// The whole grid (one cooperative launch, one CTA per SM) owns the problems p0 .. p0+np-1: the
// trailing GEMM of every block is spread over all SMs, which suits groups of few problems with
// long histories (size1 >= 3), where a cluster's 8 SMs would hold the whole group.
template <int S, bool VIE, bool RET, int BN>
__global__ void __launch_bounds__(256, 1) k_volterra_grid(GroupDev g, const ProbDev *__restrict__ probs, int n,
                                                          int p0, int np, double2 *acc, double2 *panel, GridSync gs) {
    volterra_blocked<S, VIE, RET, BN>(g, probs, n, p0, np, np, acc, panel, gs);
}

// ---- start blocks of the cluster path (one CTA per problem) ---------------------------------
// ret: G(n, n) = -i (Dyson) or Q(n, n) (VIE2), then the k-block start G(n, n-1..n-k)
// (dyson_impl :112-157, vie2_impl :60-100); the recursion below it is k_volterra_cl.
template <int S, bool VIE>
__global__ void __launch_bounds__(256) k_ret_start(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    extern __shared__ double2 smem[];
    constexpr int s2 = S * S;
    const ProbDev p = probs[blockIdx.x];
    double2 *grow = p.gret + tri(n) * s2;
    for (int e = threadIdx.x; e < s2; e += blockDim.x)
        grow[(long)n * s2 + e] = VIE ? p.qret[(tri(n) + n) * s2 + e] : (e / S == e % S ? cmk(0.0, -1.0) : cmk(0, 0));
    __syncthreads();
    if (VIE) ret_start_block_vie<S>(g, p, n, smem);
    else ret_start_block<S>(g, p, n, smem);
}

// les: G^<(0, n) = -G^tv(n, 0)^dagger and the k-block start G^<(1..k, n) (dyson_impl :926-982), or
// the VIE2 start G^<(0..k, n) (vie2_impl :847-900); gl = the Sigma-shared products in g.gles.
template <int S, bool VIE>
__global__ void __launch_bounds__(256) k_les_start(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    extern __shared__ double2 smem[];
    constexpr int s2 = S * S;
    const ProbDev p = probs[blockIdx.x];
    const long ldc = g.ldc;
    const double2 *gl = g.gles + (long)p.col * S;
    double2 *xcol = p.gles + tri(n) * s2;
    if (VIE) {
        les_start_block_vie<S>(g, p, n, gl, ldc, xcol, smem);
    } else {
        for (int ad = threadIdx.x; ad < s2; ad += blockDim.x) {
            const int a = ad / S, d = ad % S;
            xcol[ad] = cneg(cconj(p.gtv[((long)n * s2 + d * S + a) * (g.ntau + 1) + 0]));
        }
        __syncthreads();
        les_start_block<S>(g, p, n, gl, ldc, xcol, smem);
    }
}
