// Volterra recursions of one Dyson / VIE2 time step for size1 <= 2, several problems per CTA.
//
// The retarded row G^R(n, j), j = n-k-1 .. 0 (dyson_impl :158-213, vie2_impl :60-140) and the
// lesser column G^<(j, n), j = k+1 .. n (dyson_impl :983-1011, vie2_impl :847-990) are solved in
// blocks of 32 rows.  For a block, the sum over every row solved before it ("phase A") is
//   ret:  acc(j) = sum_{m > jhi} w(n-j, n-m) G(n,m) Sigma^R(m,j)
//   les:  acc(j) = sum_{m < jlo} w(j,m) Sigma^R(j,m) G^<(m,n)
// Sigma (F / Fcc for VIE2) is shared by all problems of a group, so a CTA takes PP <= 8 problems
// and computes phase A for all of them at once as one complex GEMM on the FP64 tensor cores
// (mma.sync m8n8k4 .f64, four real MMAs per complex 8x8x4 tile): each Sigma element is read once
// per CTA instead of once per problem.  The fragments are loaded from global memory (L2) eight
// k-steps ahead of their MMAs.  Away from the diagonal (|m - j| > k) the Gregory weight depends
// on m alone (c_m: omega at the n / 0 end, else 1), so it is a column scale of the GEMM; the <= k
// terms next to the block are corrected to the exact weight afterwards.  Warp q then solves the
// block's rows of problem q with each lane owning one row in registers (as in the one-problem
// kernels), and the next block starts.  PP is chosen per group by the autotuner on the host.
#pragma once

#define MP_JB 32  // rows per block (lane = row)
#define MP_NW 16  // warps per CTA: warps 0..PP-1 own a problem's chain, all of them share phase A
// Registers per thread of the multi-problem kernels: 128 (the most a 512-thread CTA can have).
// Capping size1 = 1 at 96, so that a k_tv_stream CTA fits beside, cost ~100-270 bytes of spills
// per thread and made the lesser recursion 20 % slower in the config-4 step, while the tv stream
// gained nothing from the company; so both kernels keep their own SMs' registers.
#define MP_MAXREG(S) 128

template <int S> struct MpCfg {
    static constexpr int s2 = S * S;
    static constexpr int TRI = MP_JB * (MP_JB - 1) / 2;    // packed strictly-lower block triangle
    static constexpr int WSW = 2 * NESSI_K1MAX * NESSI_K1MAX * s2 + 2 * NESSI_K1MAX * s2 + 2;  // start work/warp
    static constexpr int acc = 0;                           // 8 problems x 32 rows x s2: phase-A sums
    static constexpr int red = acc + 8 * MP_JB * s2;        // MP_NW warps x 32 lanes x 2 double2: partial tiles
    static constexpr int sig = red + MP_NW * 32 * 2;        // 2 x TRI x s2 (block triangle, double-buffered)
    static constexpr int wb = sig + 2 * TRI * s2;           // 2 x TRI doubles
    static constexpr int WBN = TRI / 2 + 1;                 // double2 units of one weight buffer
    static constexpr int total = wb + 2 * WBN;
    static_assert(sig + 2 * TRI * s2 >= 8 * WSW, "start workspaces must fit below the weights");
};

// D += A B on the FP64 tensor cores, one 8x8x4 tile: lane holds A[lane/4][lane%4],
// B[lane%4][lane/4] and D[lane/4][2(lane%4) + {0,1}] (mma.m8n8k4 .f64 fragment layout).
__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Complex 8x8 tile (mt, nt) of C = A B over the k-steps ks0, ks0 + kstride, ... of K (4 per step):
// c[0..1] real and c[2..3] imaginary parts of D[lane/4][2(lane%4) + {0,1}].  fa(r, kk) and fb(kk, cc)
// return the operands (zero outside the matrices, in particular for kk >= K).  The fragments of
// MMA_U k-steps are loaded first and multiplied afterwards, so that 2 MMA_U loads are in flight.
#define MMA_U 8
template <class FA, class FB>
__device__ __forceinline__ void ztile884(const FA &fa, const FB &fb, int mt, int nt, int K, int ks0, int kstride,
                                         int lane, double *c) {
    const int ar = mt * 8 + (lane >> 2), bc = nt * 8 + (lane >> 2), kq = lane & 3;
    for (int ks = ks0; ks * 4 < K; ks += MMA_U * kstride) {
        double2 a[MMA_U], b[MMA_U];
#pragma unroll
        for (int u = 0; u < MMA_U; u++) {
            const int kk = (ks + u * kstride) * 4 + kq;
            a[u] = fa(ar, kk);
            b[u] = fb(kk, bc);
        }
#pragma unroll
        for (int u = 0; u < MMA_U; u++) {
            dmma884(c[0], c[1], a[u].x, b[u].x);
            dmma884(c[0], c[1], -a[u].y, b[u].y);
            dmma884(c[2], c[3], a[u].x, b[u].y);
            dmma884(c[2], c[3], a[u].y, b[u].x);
        }
    }
}

// Phase A of one block as a complex GEMM C (R x N) = A (R x K) B (K x N) on the tensor cores, the
// MP_NW warps sharing the tiles (and the k-steps when there are fewer than MP_NW tiles, summed in
// warp order).  put(r, c, value) stores an element of C.
template <class FA, class FB, class PUT>
__device__ void zgemm_cta(const FA &fa, const FB &fb, const PUT &put, int R, int N, int K, double2 *red, int warp,
                          int lane) {
    const int MT = (R + 7) / 8, NT = (N + 7) / 8, tiles = MT * NT;
    const int r0 = lane >> 2, c0 = 2 * (lane & 3);
    if (tiles >= MP_NW) {
        for (int t = warp; t < tiles; t += MP_NW) {
            double c[4] = {0, 0, 0, 0};
            ztile884(fa, fb, t / NT, t % NT, K, 0, 1, lane, c);
            const int r = (t / NT) * 8 + r0, cc = (t % NT) * 8 + c0;
            put(r, cc, cmk(c[0], c[2]));
            put(r, cc + 1, cmk(c[1], c[3]));
        }
        __syncthreads();
        return;
    }
    const int ksplit = MP_NW / tiles, t = warp % tiles, ks0 = warp / tiles;
    double c[4] = {0, 0, 0, 0};
    if (ks0 < ksplit) ztile884(fa, fb, t / NT, t % NT, K, ks0, ksplit, lane, c);
    red[(warp * 32 + lane) * 2] = cmk(c[0], c[2]);
    red[(warp * 32 + lane) * 2 + 1] = cmk(c[1], c[3]);
    __syncthreads();
    if (warp < tiles) {
        double2 v0 = cmk(0, 0), v1 = cmk(0, 0);
        for (int q = 0; q < ksplit; q++) {
            v0 = cadd(v0, red[((q * tiles + warp) * 32 + lane) * 2]);
            v1 = cadd(v1, red[((q * tiles + warp) * 32 + lane) * 2 + 1]);
        }
        const int r = (warp / NT) * 8 + r0, cc = (warp % NT) * 8 + c0;
        put(r, cc, v0);
        put(r, cc + 1, v1);
    }
    __syncthreads();
}

// far-field column weight of the retarded sum: w(n-j, n-m) for m - j > k
__device__ __forceinline__ double ret_cw(int k, int n, int m) { return n - m <= k ? greg_omega(k, n - m) : 1.0; }
// far-field column weight of the lesser sum: w(j, m) for j - m > k
__device__ __forceinline__ double les_cw(int k, int m) { return m <= k ? greg_omega(k, m) : 1.0; }

// Register chain of the retarded rows of one block (lane r = row jlo + r, solved from r = nb-1 down):
//   Dyson x_r = (h acc_r - bdf_r) Minv_r,   VIE2 x_r = (Q_r - h acc_r) Minv_r   (left solves)
// Rows above the block (for the backward differences) are read from grow.
// operands of a lane's row that do not depend on the block's sums: the step inverse and the
// backward-difference part from rows above the block (VIE2: Q(n, j))
template <int S, bool VIE>
__device__ __forceinline__ void mp_ret_operands(const ProbDev &p, const double2 *grow, int n, int jlo, int nb, int K1,
                                                const double2 *ibd, int lane, double2 *mi, double2 *bd) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
#pragma unroll
    for (int e = 0; e < s2; e++) {
        mi[e] = own ? p.minv_ret[(long)(jlo + r) * s2 + e] : cmk(0, 0);
        bd[e] = (VIE && own) ? p.qret[(tri(n) + jlo + r) * s2 + e] : cmk(0, 0);
    }
    if (own && !VIE)
        for (int pp = 1; pp <= K1; pp++)
            if (r + pp >= nb)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[pp], grow[(long)(jlo + r + pp) * s2 + e], bd[e]);
}

template <int S, bool VIE>
__device__ __forceinline__ void mp_ret_chain_core(double2 *a_, double2 *mi, double2 *bd, const double2 *sig, const double *wb,
                                  const double2 *grow, int jlo, int nb, int K1, const double2 *ibd, double h, int lane);

template <int S, bool VIE>
__device__ void mp_ret_chain(double2 *a_, const double2 *sig, const double *wb, const ProbDev &p, const double2 *grow,
                             int n, int jlo, int nb, int K1, const double2 *ibd, double h, int lane) {
    constexpr int s2 = S * S;
    double2 bd[s2], mi[s2];
    mp_ret_operands<S, VIE>(p, grow, n, jlo, nb, K1, ibd, lane, mi, bd);
    mp_ret_chain_core<S, VIE>(a_, mi, bd, sig, wb, grow, jlo, nb, K1, ibd, h, lane);
}

template <int S, bool VIE>
__device__ __forceinline__ void mp_ret_chain_core(double2 *a_, double2 *mi, double2 *bd, const double2 *sig, const double *wb,
                                  const double2 *grow, int jlo, int nb, int K1, const double2 *ibd, double h, int lane) {
    constexpr int s2 = S * S;
    const int r = lane;
    double2 *gout = (double2 *)grow + (long)jlo * s2;
    for (int rr = nb - 1; rr >= 0; rr--) {
        double2 x[s2];
        if (r == rr) {
            double2 q[s2];
#pragma unroll
            for (int e = 0; e < s2; e++) q[e] = VIE ? csub(bd[e], cscale(a_[e], h)) : csub(cscale(a_[e], h), bd[e]);
#pragma unroll
            for (int aa = 0; aa < S; aa++)
#pragma unroll
                for (int d = 0; d < S; d++) {
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) t = cfma(q[aa * S + bb], mi[bb * S + d], t);
                    x[aa * S + d] = t;
                }
        }
        shfl_blk<S>(x, rr);
        if (r == rr)
#pragma unroll
            for (int e = 0; e < s2; e++) gout[(long)rr * s2 + e] = x[e];
        if (r < rr) {
            const int q = pk(rr, r);
            const double w = wb[q];
            const double2 *sg = sig + q * s2;
#pragma unroll
            for (int aa = 0; aa < S; aa++)
#pragma unroll
                for (int d = 0; d < S; d++) {
                    double2 t = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) t = cfma(x[aa * S + bb], sg[bb * S + d], t);
                    a_[aa * S + d] = cfma(cmk(w, 0.0), t, a_[aa * S + d]);
                }
            if (!VIE && rr - r <= K1)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[rr - r], x[e], bd[e]);
        }
    }
}

// Register chain of the lesser rows of one block (lane r = row jlo + r, solved from r = 0 up):
//   Dyson x_r = Minv_r (gl_r + h acc_r - bdf_r),   VIE2 x_r = Minv_r (gl_r + Q_r - h acc_r)
// Rows below the block (for the backward differences) are read from xcol.
// operands of a lane's row that do not depend on the block's sums: the step inverse, the
// Sigma-shared products (+ Q^<(j, n) for VIE2) and the backward-difference part from rows below
template <int S, bool VIE>
__device__ __forceinline__ void mp_les_operands(const ProbDev &p, const double2 *gl, long ldc, const double2 *xcol, int n,
                                                int jlo, int nb, int K1, const double2 *ibd, int lane, double2 *mi,
                                                double2 *gv, double2 *bd) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
#pragma unroll
    for (int e = 0; e < s2; e++) {
        const int a = e / S, d = e % S;
        mi[e] = own ? p.minv_les[(long)(jlo + r) * s2 + e] : cmk(0, 0);
        gv[e] = own ? gl[((long)(jlo + r) * S + a) * ldc + d] : cmk(0, 0);
        if (VIE && own) gv[e] = cadd(gv[e], p.qles[(tri(n) + jlo + r) * s2 + e]);
        bd[e] = cmk(0, 0);
    }
    if (own && !VIE)
        for (int pp = 1; pp <= K1; pp++)
            if (r - pp < 0)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[pp], xcol[(long)(jlo + r - pp) * s2 + e], bd[e]);
}

template <int S, bool VIE>
__device__ __forceinline__ void mp_les_chain_core(double2 *a_, double2 *mi, double2 *gv, double2 *bd, const double2 *sig,
                                  const double *wb, double2 *xcol, int jlo, int nb, int K1, const double2 *ibd, double h,
                                  int lane);

template <int S, bool VIE>
__device__ void mp_les_chain(double2 *a_, const double2 *sig, const double *wb, const ProbDev &p, const double2 *gl,
                             long ldc, double2 *xcol, int n, int jlo, int nb, int K1, const double2 *ibd, double h,
                             int lane) {
    constexpr int s2 = S * S;
    double2 bd[s2], mi[s2], gv[s2];
    mp_les_operands<S, VIE>(p, gl, ldc, xcol, n, jlo, nb, K1, ibd, lane, mi, gv, bd);
    mp_les_chain_core<S, VIE>(a_, mi, gv, bd, sig, wb, xcol, jlo, nb, K1, ibd, h, lane);
}

template <int S, bool VIE>
__device__ __forceinline__ void mp_les_chain_core(double2 *a_, double2 *mi, double2 *gv, double2 *bd, const double2 *sig,
                                  const double *wb, double2 *xcol, int jlo, int nb, int K1, const double2 *ibd, double h,
                                  int lane) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
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

// Block triangle of the recursion's matrix and its exact weights into shared memory, by threads
// t = 0..nthr-1: ret T(jlo+r, jlo+r2) with w(n - (jlo+r2), n - (jlo+r)); les T(jlo+r, jlo+r2)
// with w(jlo+r, jlo+r2), r2 < r < nb.
template <int S, bool RET>
__device__ __forceinline__ void mp_stage(const double2 *T, int k, int n, int jlo, int nb, double2 *sig, double *wb,
                                         int t, int nthr) {
    constexpr int s2 = S * S;
    for (int e = t; e < MpCfg<S>::TRI * s2; e += nthr) {
        const int q = e / s2, ab = e % s2;
        int r, r2;
        pk_inv(q, r, r2);
        if (r < nb) {
            sig[e] = T[(tri(jlo + r) + jlo + r2) * s2 + ab];
            if (ab == 0) wb[q] = RET ? greg_w(k, n - (jlo + r2), n - (jlo + r)) : greg_w(k, jlo + r, jlo + r2);
        }
    }
}

// ======================================================================================
// retarded component
// ======================================================================================
// Per block: the owner warps first gather the operands of their rows that do not depend on the
// block's sums (step inverses, backward-difference parts, the exact-weight corrections of the k
// rows next to the block), so those loads are in flight during phase A; after phase A the owners
// run their chains while the other warps stage the next block's triangle into the second buffer.
// Phase A of block [jlo, jhi] for the CTA's problems q as C[(q,a)][(jj,d)] =
//   sum_{(m,b)} c_m G_q(n,m)[a][b] Sigma^R(m, jlo+jj)[b][d],  m = jhi+1 .. n.
template <int S, bool VIE>
__global__ void __maxnreg__(MP_MAXREG(S)) k_ret_mp(GroupDev g, const ProbDev *__restrict__ probs, int n, int nact,
                                                int PP) {
    extern __shared__ double2 smem[];
    using C = MpCfg<S>;
    constexpr int s2 = S * S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int np = min(PP, nact - (int)blockIdx.x * PP);  // problems of this CTA; warp q < np owns problem q
    const bool owner = warp < np;
    const int k = g.k, K1 = k + 1;
    const double h = g.h;
    __shared__ double2 ibd[NESSI_K1MAX + 1];
    __shared__ double2 *rows[8];  // G^R(n, .) of the CTA's problems
    if (tid <= NESSI_K1MAX) ibd[tid] = cmk(0.0, tid <= K1 ? bd_w(k, tid) / h : 0.0);
    if (tid < 8) rows[tid] = tid < np ? probs[blockIdx.x * PP + tid].gret + tri(n) * s2 : nullptr;
    ProbDev p;
    if (owner) p = probs[blockIdx.x * PP + warp];
    __syncthreads();
    // row n: zero, G(n,n) = -i (Dyson) or Q(n,n) (VIE2); then the k-block start
    if (owner) {
        double2 *grow = rows[warp];
        for (long e = lane; e < (long)(n + 1) * s2; e += 32) {
            const int ab = (int)(e % s2);
            if (VIE) grow[e] = e / s2 == n ? p.qret[(tri(n) + n) * s2 + ab] : cmk(0, 0);
            else grow[e] = (e / s2 == n && ab / S == ab % S) ? cmk(0.0, -1.0) : cmk(0, 0);
        }
        __syncwarp();
        double2 *ws = smem + warp * C::WSW;
        if (VIE) ret_start_block_vie<S, WarpExec>(g, p, n, ws, WarpExec{lane});
        else ret_start_block<S, WarpExec>(g, p, n, ws, WarpExec{lane});
    }
    __syncthreads();
    double2 *acc_s = smem + C::acc, *red = smem + C::red;
    auto SIG = [&](int bf) { return smem + C::sig + bf * C::TRI * s2; };
    auto WB = [&](int bf) { return (double *)(smem + C::wb + bf * C::WBN); };
    const int jtop = n - k - 1;
    {
        const int jlo0 = jtop - MP_JB + 1 < 0 ? 0 : jtop - MP_JB + 1;
        mp_stage<S, true>(g.rret, k, n, jlo0, jtop - jlo0 + 1, SIG(0), WB(0), tid, MP_NW * 32);
    }
    __syncthreads();
    int cur = 0;
    for (int jhi = jtop; jhi >= 0; jhi -= MP_JB, cur ^= 1) {
        const int jlo = jhi - MP_JB + 1 < 0 ? 0 : jhi - MP_JB + 1, nb = jhi - jlo + 1;
        // owners: the operands of their rows that do not depend on phase A
        double2 corr[s2], mi[s2], bd[s2];
#pragma unroll
        for (int e = 0; e < s2; e++) corr[e] = cmk(0, 0);
        if (owner) {
            const double2 *grow = rows[warp];
            const int j = jlo + lane;
            mp_ret_operands<S, VIE>(p, grow, n, jlo, nb, K1, ibd, lane, mi, bd);
            if (lane < nb) {
                // exact weights for the rows m - j <= k just above the block
                for (int m = jhi + 1; m <= min(jhi + k, n); m++) {
                    if (m - j > k) continue;
                    const double dw = greg_w(k, n - j, n - m) - ret_cw(k, n, m);
                    const double2 *gm = grow + (long)m * s2, *sm = g.rret + (tri(m) + j) * s2;
#pragma unroll
                    for (int aa = 0; aa < S; aa++)
#pragma unroll
                        for (int d = 0; d < S; d++) {
                            double2 t = cmk(0, 0);
#pragma unroll
                            for (int bb = 0; bb < S; bb++) t = cfma(gm[aa * S + bb], sm[bb * S + d], t);
                            corr[aa * S + d] = cfma(cmk(dw, 0.0), t, corr[aa * S + d]);
                        }
                }
            }
        }
        const int mb = jhi + 1;
        auto fa = [&](int r, int kk) -> double2 {
            const int q = r / S, a = r % S, m = mb + kk / S, b = kk % S;
            if (q >= np || m > n) return cmk(0, 0);
            return cscale(rows[q][(long)m * s2 + a * S + b], ret_cw(k, n, m));
        };
        auto fb = [&](int kk, int cc) -> double2 {
            const int m = mb + kk / S, b = kk % S, jj = cc / S, d = cc % S;
            if (m > n || jj >= nb) return cmk(0, 0);
            return g.rret[(tri(m) + jlo + jj) * s2 + b * S + d];
        };
        auto put = [&](int r, int cc, double2 v) {
            const int q = r / S, a = r % S, jj = cc / S, d = cc % S;
            if (q < np && jj < MP_JB) acc_s[(q * MP_JB + jj) * s2 + a * S + d] = v;
        };
        zgemm_cta(fa, fb, put, np * S, MP_JB * S, (n - jhi) * S, red, warp, lane);
        if (owner) {
            double2 acc[s2];
#pragma unroll
            for (int e = 0; e < s2; e++)
                acc[e] = lane < nb ? cadd(acc_s[(warp * MP_JB + lane) * s2 + e], corr[e]) : cmk(0, 0);
            mp_ret_chain_core<S, VIE>(acc, mi, bd, SIG(cur), WB(cur), rows[warp], jlo, nb, K1, ibd, h, lane);
        } else if (warp >= 8 && jlo > 0) {
            // the next block's triangle, while the owners solve this one
            const int jhi2 = jlo - 1, jlo2 = jhi2 - MP_JB + 1 < 0 ? 0 : jhi2 - MP_JB + 1;
            mp_stage<S, true>(g.rret, k, n, jlo2, jhi2 - jlo2 + 1, SIG(cur ^ 1), WB(cur ^ 1), tid - 256,
                              MP_NW * 32 - 256);
        }
        __syncthreads();
    }
}

// ======================================================================================
// lesser component
// ======================================================================================
// Phase A of block [jlo, jhi] as C[(jj,a)][(q,d)] =
//   sum_{(m,b)} Sigma^R(jlo+jj, m)[a][b] c'_m G^<_q(m,n)[b][d],  m = 0 .. jlo-1.
template <int S, bool VIE>
__global__ void __maxnreg__(MP_MAXREG(S)) k_les_mp(GroupDev g, const ProbDev *__restrict__ probs, int n, int nact,
                                                int PP) {
    extern __shared__ double2 smem[];
    using C = MpCfg<S>;
    constexpr int s2 = S * S;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int np = min(PP, nact - (int)blockIdx.x * PP);
    const bool owner = warp < np;
    const int k = g.k, K1 = k + 1;
    const double h = g.h;
    const long ldc = g.ldc;
    __shared__ double2 ibd[NESSI_K1MAX + 1];
    __shared__ double2 *cols[8];  // G^<(., n) of the CTA's problems
    if (tid <= NESSI_K1MAX) ibd[tid] = cmk(0.0, tid <= K1 ? bd_w(k, tid) / h : 0.0);
    if (tid < 8) cols[tid] = tid < np ? probs[blockIdx.x * PP + tid].gles + tri(n) * s2 : nullptr;
    ProbDev p;
    if (owner) p = probs[blockIdx.x * PP + warp];
    __syncthreads();
    const double2 *gl = owner ? g.gles + (long)p.col * S : nullptr;  // gles(j)[a][d] at gl[(j*S+a)*ldc + d]
    if (owner) {
        double2 *xcol = cols[warp];
        double2 *ws = smem + warp * C::WSW;
        if (VIE) {
            les_start_block_vie<S, WarpExec>(g, p, n, gl, ldc, xcol, ws, WarpExec{lane});
        } else {
            for (int ad = lane; ad < s2; ad += 32) {
                const int a = ad / S, d = ad % S;
                xcol[ad] = cneg(cconj(p.gtv[((long)n * s2 + d * S + a) * (g.ntau + 1) + 0]));
            }
            __syncwarp();
            les_start_block<S, WarpExec>(g, p, n, gl, ldc, xcol, ws, WarpExec{lane});
        }
    }
    __syncthreads();
    if (n <= k) return;
    double2 *acc_s = smem + C::acc, *red = smem + C::red;
    auto SIG = [&](int bf) { return smem + C::sig + bf * C::TRI * s2; };
    auto WB = [&](int bf) { return (double *)(smem + C::wb + bf * C::WBN); };
    mp_stage<S, false>(g.sret, k, n, K1, min(n, K1 + MP_JB - 1) - K1 + 1, SIG(0), WB(0), tid, MP_NW * 32);
    __syncthreads();
    int cur = 0;
    for (int jlo = K1; jlo <= n; jlo += MP_JB, cur ^= 1) {
        const int jhi = jlo + MP_JB - 1 > n ? n : jlo + MP_JB - 1, nb = jhi - jlo + 1;
        // owners: the operands of their rows that do not depend on phase A
        double2 corr[s2], mi[s2], gv[s2], bd[s2];
#pragma unroll
        for (int e = 0; e < s2; e++) corr[e] = cmk(0, 0);
        if (owner) {
            const double2 *xcol = cols[warp];
            const int j = jlo + lane;
            mp_les_operands<S, VIE>(p, gl, ldc, xcol, n, jlo, nb, K1, ibd, lane, mi, gv, bd);
            if (lane < nb) {
                // exact weights for the columns j - m <= k just below the block
                for (int m = max(0, jlo - k); m < jlo; m++) {
                    if (j - m > k) continue;
                    const double dw = greg_w(k, j, m) - les_cw(k, m);
                    const double2 *sm = g.sret + (tri(j) + m) * s2, *xm = xcol + (long)m * s2;
#pragma unroll
                    for (int aa = 0; aa < S; aa++)
#pragma unroll
                        for (int d = 0; d < S; d++) {
                            double2 t = cmk(0, 0);
#pragma unroll
                            for (int bb = 0; bb < S; bb++) t = cfma(sm[aa * S + bb], xm[bb * S + d], t);
                            corr[aa * S + d] = cfma(cmk(dw, 0.0), t, corr[aa * S + d]);
                        }
                }
            }
        }
        auto fa = [&](int r, int kk) -> double2 {
            const int jj = r / S, a = r % S, m = kk / S, b = kk % S;
            if (jj >= nb || m >= jlo) return cmk(0, 0);
            return g.sret[(tri(jlo + jj) + m) * s2 + a * S + b];
        };
        auto fb = [&](int kk, int cc) -> double2 {
            const int m = kk / S, b = kk % S, q = cc / S, d = cc % S;
            if (q >= np || m >= jlo) return cmk(0, 0);
            return cscale(cols[q][(long)m * s2 + b * S + d], les_cw(k, m));
        };
        auto put = [&](int r, int cc, double2 v) {
            const int jj = r / S, a = r % S, q = cc / S, d = cc % S;
            if (q < np && jj < MP_JB) acc_s[(q * MP_JB + jj) * s2 + a * S + d] = v;
        };
        zgemm_cta(fa, fb, put, MP_JB * S, np * S, jlo * S, red, warp, lane);
        if (owner) {
            double2 acc[s2];
#pragma unroll
            for (int e = 0; e < s2; e++)
                acc[e] = lane < nb ? cadd(acc_s[(warp * MP_JB + lane) * s2 + e], corr[e]) : cmk(0, 0);
            mp_les_chain_core<S, VIE>(acc, mi, gv, bd, SIG(cur), WB(cur), cols[warp], jlo, nb, K1, ibd, h, lane);
        } else if (warp >= 8 && jhi < n) {
            // the next block's triangle, while the owners solve this one
            const int jlo2 = jhi + 1, jhi2 = jlo2 + MP_JB - 1 > n ? n : jlo2 + MP_JB - 1;
            mp_stage<S, false>(g.sret, k, n, jlo2, jhi2 - jlo2 + 1, SIG(cur ^ 1), WB(cur ^ 1), tid - 256,
                               MP_NW * 32 - 256);
        }
        __syncthreads();
    }
}
