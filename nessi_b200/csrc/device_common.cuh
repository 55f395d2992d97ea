// Device helpers shared by the Kadanoff-Baym kernels: complex arithmetic on double2,
// the integration tables in constant memory, Gregory weight lookup and a CTA-wide
// dense complex solver for the (k*s) x (k*s) start blocks.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "cntr_tables.inc"

#define NESSI_MAXS 8        // largest orbital size with a compiled kernel
#define NESSI_K1MAX (CNTR_KMAX + 1)
#define NESSI_K2MAX (2 * NESSI_K1MAX)

// ---- complex arithmetic (double2 = re, im) -----------------------------------------
__host__ __device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// c + a*b
__host__ __device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {
    return cmk(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return cmk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return cmk(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cneg(double2 a) { return cmk(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return cmk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.x * r + b.y;
        return cmk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// ---- integration tables (one order k per launch; indexed [k]) ----------------------
struct IntegTables {
    double greg[NESSI_K1MAX][NESSI_K2MAX * NESSI_K2MAX];
    double omega[NESSI_K1MAX][NESSI_K1MAX];
    double poly_int[NESSI_K1MAX][NESSI_K1MAX * NESSI_K1MAX * NESSI_K1MAX];
    double poly_diff[NESSI_K1MAX][NESSI_K1MAX * NESSI_K1MAX];
    double poly_interp[NESSI_K1MAX][NESSI_K1MAX * NESSI_K1MAX];
    double bd[NESSI_K1MAX][NESSI_K1MAX + 1];
    double rcorr[NESSI_K1MAX][(NESSI_K1MAX - 2) * NESSI_K1MAX * NESSI_K1MAX];
};
__constant__ IntegTables c_tab;  // single translation unit (nessi_gpu.cu)

// Integrator::gregory_weights(n, j) (integration.hpp:382-390) for order k.
__device__ __forceinline__ double greg_w(int k, int n, int j) {
    const int k1 = k + 1, k2 = 2 * k1;
    if (n >= k2) {
        if (j > k && j < n - k) return 1.0;
        if (j < k1) return c_tab.omega[k][j];
        return c_tab.omega[k][n - j];
    }
    return c_tab.greg[k][n * NESSI_K2MAX + j];
}
__device__ __forceinline__ double greg_omega(int k, int j) { return c_tab.omega[k][j]; }
__device__ __forceinline__ double poly_diff(int k, int i, int l) { return c_tab.poly_diff[k][i * NESSI_K1MAX + l]; }
__device__ __forceinline__ double poly_int(int k, int i, int j, int l) {
    return c_tab.poly_int[k][(i * NESSI_K1MAX + j) * NESSI_K1MAX + l];
}
__device__ __forceinline__ double bd_w(int k, int l) { return c_tab.bd[k][l]; }
__device__ __forceinline__ double rcorr_w(int k, int m, int j, int l) {
    if (k < 2) return 0.0;
    return c_tab.rcorr[k][((m - 1) * NESSI_K1MAX + j) * NESSI_K1MAX + l];
}

// ---- execution groups for the small dense block solves --------------------------------------
// CtaExec: all threads of the block; WarpExec: the 32 lanes of one warp.
struct CtaExec {
    __device__ __forceinline__ int t() const { return threadIdx.x; }
    __device__ __forceinline__ int n() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct WarpExec {
    int lane;
    __device__ __forceinline__ int t() const { return lane; }
    __device__ __forceinline__ int n() const { return 32; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
};

// ---- dense solve A X = B (n x n, nrhs columns), partial pivoting, by an execution group ------
// A (n x n, row-major, lda = n) and B (n x nrhs, row-major) live in shared memory and
// are overwritten; on return B holds X.  Every member of the group must call it.
// Returns nonzero in *status (shared) if a zero pivot was met.
template <class X>
__device__ inline void grp_solve(const X &x, double2 *A, double2 *B, int n, int nrhs, int *s_piv, int *status) {
    const int tid = x.t(), nth = x.n();
    for (int c = 0; c < n; c++) {
        if (tid == 0) {
            int p = c;
            double best = cabs2(A[c * n + c]);
            for (int i = c + 1; i < n; i++) {
                double a = cabs2(A[i * n + c]);
                if (a > best) { best = a; p = i; }
            }
            *s_piv = p;
            if (best == 0.0) *status = 1;
        }
        x.sync();
        int p = *s_piv;
        if (p != c) {
            for (int j = tid; j < n + nrhs; j += nth) {
                if (j < n) {
                    double2 t = A[c * n + j]; A[c * n + j] = A[p * n + j]; A[p * n + j] = t;
                } else {
                    int jj = j - n;
                    double2 t = B[c * nrhs + jj]; B[c * nrhs + jj] = B[p * nrhs + jj]; B[p * nrhs + jj] = t;
                }
            }
        }
        x.sync();
        double2 piv = A[c * n + c];
        if (piv.x == 0.0 && piv.y == 0.0) piv = cmk(1.0, 0.0);  // status already flagged
        // eliminate rows below c
        const int w = n - c - 1 + nrhs;  // columns c+1..n-1 and rhs
        for (int idx = tid; idx < (n - c - 1) * w; idx += nth) {
            int i = c + 1 + idx / w, j = idx % w;
            double2 f = cdiv(A[i * n + c], piv);
            if (j < n - c - 1) {
                int jj = c + 1 + j;
                A[i * n + jj] = csub(A[i * n + jj], cmul(f, A[c * n + jj]));
            } else {
                int jj = j - (n - c - 1);
                B[i * nrhs + jj] = csub(B[i * nrhs + jj], cmul(f, B[c * nrhs + jj]));
            }
        }
        x.sync();
        // column c below the pivot is no longer needed (implicit zeros)
    }
    // back substitution, one rhs column per thread
    for (int i = n - 1; i >= 0; i--) {
        for (int j = tid; j < nrhs; j += nth) {
            double2 acc = B[i * nrhs + j];
            for (int l = i + 1; l < n; l++) acc = csub(acc, cmul(A[i * n + l], B[l * nrhs + j]));
            B[i * nrhs + j] = cdiv(acc, A[i * n + i].x == 0.0 && A[i * n + i].y == 0.0 ? cmk(1, 0) : A[i * n + i]);
        }
        x.sync();
    }
}

__device__ inline void cta_solve(double2 *A, double2 *B, int n, int nrhs, int *s_piv, int *status) {
    grp_solve(CtaExec{}, A, B, n, nrhs, s_piv, status);
}

// Invert an s x s complex matrix held by one thread (Gauss-Jordan, partial pivoting).
template <int S>
__device__ inline int small_inverse(const double2 *M, double2 *Minv) {
    double2 a[S][2 * S];
    for (int i = 0; i < S; i++)
        for (int j = 0; j < S; j++) {
            a[i][j] = M[i * S + j];
            a[i][S + j] = cmk(i == j ? 1.0 : 0.0, 0.0);
        }
    int bad = 0;
    for (int c = 0; c < S; c++) {
        int p = c;
        double best = cabs2(a[c][c]);
        for (int i = c + 1; i < S; i++)
            if (cabs2(a[i][c]) > best) { best = cabs2(a[i][c]); p = i; }
        if (best == 0.0) { bad = 1; continue; }
        if (p != c)
            for (int j = 0; j < 2 * S; j++) { double2 t = a[c][j]; a[c][j] = a[p][j]; a[p][j] = t; }
        double2 inv = cdiv(cmk(1, 0), a[c][c]);
        for (int j = 0; j < 2 * S; j++) a[c][j] = cmul(a[c][j], inv);
        for (int i = 0; i < S; i++) {
            if (i == c) continue;
            double2 f = a[i][c];
            for (int j = 0; j < 2 * S; j++) a[i][j] = csub(a[i][j], cmul(f, a[c][j]));
        }
    }
    for (int i = 0; i < S; i++)
        for (int j = 0; j < S; j++) Minv[i * S + j] = a[i][S + j];
    return bad;
}
