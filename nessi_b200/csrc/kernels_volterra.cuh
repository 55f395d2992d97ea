// Volterra recursions of one Dyson time step, one CTA per problem:
//   k_ret  G^R(n, j), j = n-k-1 .. 0       (right equation in t', dyson_impl :158-213)
//   k_les  G^<(j, n), j = k+1 .. n         (left equation in t, dyson_impl :983-1011)
// Both are triangular solves whose matrix is the shared Sigma^R triangle.  The unknowns are
// processed in blocks of JB rows.  For each block the sum over all unknowns outside the block
// ("phase A") is a CTA-parallel reduction; the rows of the block are then solved one after
// the other by warp 0 ("phase B"), entirely from shared memory, updating the remaining rows
// of the block after every solved row.  While warp 0 solves block b, warps 1-7 already
// compute phase A of block b+1 over everything above (ret) / below (les) block b and stage
// its data; after a barrier all warps add block b's own contribution ("phase C").
#pragma once

template <int S> struct RetCfg {
    static constexpr int JB = (S <= 2) ? 32 : (256 / (S * S) > 1 ? 256 / (S * S) : 1);
    static constexpr int E = JB * S * S;               // entries of one block
    static constexpr int TRI = JB * (JB - 1) / 2;      // packed strictly-lower block triangle
};

// shared-memory layout (units of double2); acc/sig/w/minv/gl/xs are double-buffered
template <int S> struct VolLayout {
    static constexpr int JB = RetCfg<S>::JB, s2 = S * S, TRI = RetCfg<S>::TRI;
    static constexpr int XS = JB + NESSI_K1MAX;        // rows of the solved-value window
    static constexpr int WB = TRI / 2 + 1;             // TRI doubles
    static constexpr int part = 0;                     // 1024 partial sums
    static constexpr int acc = part + 1024;            // 2 x JB*s2
    static constexpr int qv = acc + 2 * JB * s2;       // s2
    static constexpr int sig = qv + s2;                // 2 x TRI*s2
    static constexpr int w = sig + 2 * TRI * s2;       // 2 x WB
    static constexpr int minv = w + 2 * WB;            // 2 x JB*s2
    static constexpr int gl = minv + 2 * JB * s2;      // 2 x JB*s2 (les only)
    static constexpr int xs = gl + 2 * JB * s2;        // 2 x XS*s2
    static constexpr int red = xs + 2 * XS * s2;       // 8*32*S (les phase A reduction)
    static constexpr int total = red + 8 * 32 * S;
};

__device__ __forceinline__ int pk(int r, int r2) { return r * (r - 1) / 2 + r2; }  // r2 < r
__device__ __forceinline__ void pk_inv(int q, int &r, int &r2) {
    r = (int)((1.0 + sqrt(1.0 + 8.0 * q)) * 0.5);
    while (pk(r, 0) > q) r--;
    while (pk(r + 1, 0) <= q) r++;
    r2 = q - pk(r, 0);
}
// barrier of warps 1..7 (224 threads); barrier 0 is __syncthreads
__device__ __forceinline__ void helper_sync() { asm volatile("bar.sync 1, 224;" ::: "memory"); }

// =======================================================================================
// retarded component
// =======================================================================================
// acc[r] = sum_{m=mlo}^{n} w(n-j, n-m) G(n,m) Sigma(m,j), j = jlo + r, by threads t..t+nthr-1.
// A work item is (m-group gi, row r, RA rows of the s x s block); U terms of m in flight.
template <int S> struct PhaseACfg {
    static constexpr int RA = (S <= 2) ? S : 1, NA = S / RA;
    static constexpr int EA = RetCfg<S>::JB * NA;
    static constexpr int U = S == 1 ? 4 : (S == 2 ? 2 : 1);
    static constexpr int GMAX = 1024 / (RetCfg<S>::JB * S * S);
};

template <int S, bool HELPERS>
__device__ void ret_phaseA(const GroupDev &g, const double2 *grow, int n, int jlo, int nb, int mlo, double2 *part,
                           double2 *acc, int t, int nthr) {
    constexpr int s2 = S * S, JB = RetCfg<S>::JB, RA = PhaseACfg<S>::RA, NA = PhaseACfg<S>::NA;
    constexpr int EA = PhaseACfg<S>::EA, U = PhaseACfg<S>::U;
    const int k = g.k;
    int G = nthr / EA;
    if (G > PhaseACfg<S>::GMAX) G = PhaseACfg<S>::GMAX;
    if (G < 1) G = 1;
    for (int idx = t; idx < G * EA; idx += nthr) {
        const int gi = idx / EA, e = idx % EA, r = e / NA, a0 = (e % NA) * RA;
        double2 sum[RA][S];
#pragma unroll
        for (int i = 0; i < RA; i++)
#pragma unroll
            for (int d = 0; d < S; d++) sum[i][d] = cmk(0, 0);
        if (r < nb) {
            const int j = jlo + r;
            const double2 *sj = g.rret + (long)j * s2;  // Sigma(m,j) at sj + tri(m) s2
            const double2 *ga = grow + a0 * S;          // G(n,m)[a0+i][b] at ga + m s2 + i S + b
            int m = mlo + gi;
            for (; m + (U - 1) * G <= n; m += U * G) {
                double2 gv[U][RA * S], sv[U][s2];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const long mu = m + u * G;
#pragma unroll
                    for (int i = 0; i < RA * S; i++) gv[u][i] = ga[mu * s2 + i];
#pragma unroll
                    for (int i = 0; i < s2; i++) sv[u][i] = sj[tri(mu) * s2 + i];
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const double w = greg_w(k, n - j, n - (m + u * G));
#pragma unroll
                    for (int i = 0; i < RA; i++)
#pragma unroll
                        for (int d = 0; d < S; d++) {
                            double2 tt = cmk(0, 0);
#pragma unroll
                            for (int bb = 0; bb < S; bb++) tt = cfma(gv[u][i * S + bb], sv[u][bb * S + d], tt);
                            sum[i][d] = cfma(cmk(w, 0.0), tt, sum[i][d]);
                        }
                }
            }
            for (; m <= n; m += G) {
                const double w = greg_w(k, n - j, n - m);
#pragma unroll
                for (int i = 0; i < RA; i++)
#pragma unroll
                    for (int d = 0; d < S; d++) {
                        double2 tt = cmk(0, 0);
#pragma unroll
                        for (int bb = 0; bb < S; bb++)
                            tt = cfma(ga[(long)m * s2 + i * S + bb], sj[tri(m) * s2 + bb * S + d], tt);
                        sum[i][d] = cfma(cmk(w, 0.0), tt, sum[i][d]);
                    }
            }
        }
#pragma unroll
        for (int i = 0; i < RA; i++)
#pragma unroll
            for (int d = 0; d < S; d++) part[(gi * JB + r) * s2 + (a0 + i) * S + d] = sum[i][d];
    }
    if (HELPERS) helper_sync(); else __syncthreads();
    for (int e = t; e < JB * s2; e += nthr) {
        double2 v = part[e];
        for (int gi = 1; gi < G; gi++) v = cadd(v, part[gi * JB * s2 + e]);
        acc[e] = v;
    }
}

template <int S, bool VIE>
__device__ void ret_stage(const GroupDev &g, const ProbDev &p, int n, int jlo, int nb, double2 *sig, double *wb,
                          double2 *minv, double2 *qb, int t, int nthr) {
    constexpr int s2 = S * S;
    const int k = g.k;
    for (int e = t; e < RetCfg<S>::TRI * s2; e += nthr) {
        const int q = e / s2, ab = e % s2;
        int r, r2;
        pk_inv(q, r, r2);
        if (r < nb) {
            sig[e] = g.rret[(tri(jlo + r) + jlo + r2) * s2 + ab];
            if (ab == 0) wb[q] = greg_w(k, n - (jlo + r2), n - (jlo + r));
        }
    }
    for (int e = t; e < nb * s2; e += nthr) {
        minv[e] = p.minv_ret[(long)jlo * s2 + e];
        if (VIE) qb[e] = p.qret[(tri(n) + jlo) * s2 + e];  // Q(n, jlo + r)
    }
}

// Register-resident solve of one block for S <= 2 (warp 0): lane r owns block row r and keeps
// its sum (acc), its backward-difference partial sum and its step inverse in registers.  After
// row rr is solved its value is broadcast with warp shuffles and every lane folds it into its
// own sums, so the sequential path per row is a handful of dependent FP64 operations and one
// shuffle.  ibd[p] = (i/h) bd(p) in shared memory.
template <int S>
__device__ __forceinline__ void shfl_blk(double2 *x, int src) {
#pragma unroll
    for (int e = 0; e < S * S; e++) {
        x[e].x = __shfl_sync(0xffffffffu, x[e].x, src);
        x[e].y = __shfl_sync(0xffffffffu, x[e].y, src);
    }
}

// ret: rows solved from r = nb-1 down to 0; x_r = (h acc_r - bdf_r) Minv_r (left solve);
// VIE2: x_r = (Q_r - h acc_r) Minv_r
template <int S, bool VIE>
__device__ void ret_chain(const double2 *acc, const double2 *sig, const double *wb, const double2 *minv,
                          const double2 *qb, double2 *xs, double2 *gout, int nb, int K1, const double2 *ibd, double h,
                          int lane) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
    double2 a_[s2], bd[s2], mi[s2];
#pragma unroll
    for (int e = 0; e < s2; e++) {
        a_[e] = own ? acc[r * s2 + e] : cmk(0, 0);
        mi[e] = own ? minv[r * s2 + e] : cmk(0, 0);
        bd[e] = (VIE && own) ? qb[r * s2 + e] : cmk(0, 0);  // VIE2: bd holds Q_r
    }
    if (own && !VIE)
        for (int pp = 1; pp <= K1; pp++)
            if (r + pp >= nb)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[pp], xs[(r + pp) * s2 + e], bd[e]);
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
        if (r == rr) {
#pragma unroll
            for (int e = 0; e < s2; e++) { xs[rr * s2 + e] = x[e]; gout[(long)rr * s2 + e] = x[e]; }
        }
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

// les: rows solved from r = 0 up; x_r = Minv_r (gl_r + h acc_r - bdf_r) (right solve);
// VIE2: x_r = Minv_r (gl_r - h acc_r) with gl_r including Q^<(j,n).
// xs holds x(jlo - K1 + i) at index i
template <int S, bool VIE>
__device__ void les_chain(const double2 *acc, const double2 *sig, const double *wb, const double2 *minv,
                          const double2 *glb, double2 *xs, double2 *gout, int nb, int K1, const double2 *ibd, double h,
                          int lane) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
    double2 a_[s2], bd[s2], mi[s2], gv[s2];
#pragma unroll
    for (int e = 0; e < s2; e++) {
        a_[e] = own ? acc[r * s2 + e] : cmk(0, 0);
        mi[e] = own ? minv[r * s2 + e] : cmk(0, 0);
        gv[e] = own ? glb[r * s2 + e] : cmk(0, 0);
        bd[e] = cmk(0, 0);
    }
    if (own && !VIE)
        for (int pp = 1; pp <= K1; pp++)
            if (r - pp < 0)
#pragma unroll
                for (int e = 0; e < s2; e++) bd[e] = cfma(ibd[pp], xs[(r - pp + K1) * s2 + e], bd[e]);
    for (int rr = 0; rr < nb; rr++) {
        double2 x[s2];
        if (r == rr) {
            double2 q[s2];
#pragma unroll
            for (int e = 0; e < s2; e++) q[e] = VIE ? cfma(cmk(-h, 0.0), a_[e], gv[e]) : csub(cfma(cmk(h, 0.0), a_[e], gv[e]), bd[e]);
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
        if (r == rr) {
#pragma unroll
            for (int e = 0; e < s2; e++) { xs[(rr + K1) * s2 + e] = x[e]; gout[(long)rr * s2 + e] = x[e]; }
        }
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

template <int S, bool VIE = false>
__global__ void __launch_bounds__(256, 2) k_ret(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    extern __shared__ double2 smem[];
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, K1 = k + 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int s2 = S * S, JB = RetCfg<S>::JB, E = RetCfg<S>::E;
    using L = VolLayout<S>;
    const double h = g.h;
    double2 *grow = p.gret + tri(n) * s2;  // G(n, 0..n)
    for (long e = tid; e < (long)(n + 1) * s2; e += blockDim.x) {
        int ab = (int)(e % s2);
        if (VIE) grow[e] = e / s2 == n ? p.qret[(tri(n) + n) * s2 + ab] : cmk(0, 0);  // G(n,n) = Q(n,n)
        else grow[e] = (e / s2 == n && (ab / S == ab % S)) ? cmk(0.0, -1.0) : cmk(0, 0);
    }
    __syncthreads();
    if (VIE) ret_start_block_vie<S>(g, p, n, smem);
    else ret_start_block<S>(g, p, n, smem);
    double2 *part = smem + L::part, *qv = smem + L::qv;
    double2 ibd[NESSI_K1MAX + 1];
#pragma unroll
    for (int pp = 0; pp <= NESSI_K1MAX; pp++) ibd[pp] = cmk(0.0, pp <= K1 ? bd_w(k, pp) / h : 0.0);
    __shared__ double2 ibds[NESSI_K1MAX + 1];
    if (tid <= NESSI_K1MAX) ibds[tid] = cmk(0.0, tid <= K1 ? bd_w(k, tid) / h : 0.0);
    const int jtop = n - k - 1;
    auto ACC = [&](int bf) { return smem + L::acc + bf * JB * s2; };
    auto SIG = [&](int bf) { return smem + L::sig + bf * L::TRI * s2; };
    auto WBF = [&](int bf) { return (double *)(smem + L::w + bf * L::WB); };
    auto MNV = [&](int bf) { return smem + L::minv + bf * JB * s2; };
    auto QB = [&](int bf) { return smem + L::gl + bf * JB * s2; };  // VIE2: Q(n, j) of the block
    auto XS = [&](int bf) { return smem + L::xs + bf * L::XS * s2; };
    // prologue: block 0 with all threads
    {
        const int jhi = jtop, jlo = jhi - JB + 1 < 0 ? 0 : jhi - JB + 1, nb = jhi - jlo + 1;
        ret_phaseA<S, false>(g, grow, n, jlo, nb, jhi + 1, part, ACC(0), tid, 256);
        ret_stage<S, VIE>(g, p, n, jlo, nb, SIG(0), WBF(0), MNV(0), QB(0), tid, 256);
        for (int e = tid; e < K1 * s2; e += 256) XS(0)[nb * s2 + e] = grow[(long)(jhi + 1) * s2 + e];
        __syncthreads();
    }
    for (int b = 0;; b++) {
        const int cur = b & 1, nxt = cur ^ 1;
        const int jhi = jtop - b * JB, jlo = jhi - JB + 1 < 0 ? 0 : jhi - JB + 1, nb = jhi - jlo + 1;
        const bool has_next = jlo > 0;
        const int jhi2 = jlo - 1, jlo2 = jhi2 - JB + 1 < 0 ? 0 : jhi2 - JB + 1, nb2 = jhi2 - jlo2 + 1;
        if (warp == 0 && S <= 2) {
            ret_chain<S, VIE>(ACC(cur), SIG(cur), WBF(cur), MNV(cur), QB(cur), XS(cur), grow + (long)jlo * s2, nb, K1,
                              ibds, h, lane);
        } else if (warp == 0) {
            // ---- phase B: solve j = jhi .. jlo
            double2 *acc = ACC(cur), *sig = SIG(cur), *minv = MNV(cur), *xs = XS(cur), *qb = QB(cur);
            const double *wb = WBF(cur);
            for (int r = nb - 1; r >= 0; r--) {
                for (int e = lane; e < s2; e += 32) {
                    double2 q = cscale(acc[r * s2 + e], h);
                    if (VIE) {
                        q = csub(qb[r * s2 + e], q);
                    } else {
#pragma unroll
                        for (int pp = 1; pp <= NESSI_K1MAX; pp++)
                            if (pp <= K1) q = csub(q, cmul(ibd[pp], xs[(r + pp) * s2 + e]));
                    }
                    qv[e] = q;
                }
                __syncwarp();
                for (int e = lane; e < s2; e += 32) {
                    const int a = e / S, d = e % S;
                    double2 x = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) x = cfma(qv[a * S + bb], minv[r * s2 + bb * S + d], x);
                    xs[r * s2 + e] = x;
                    grow[(long)(jlo + r) * s2 + e] = x;
                }
                __syncwarp();
                for (int it = lane; it < r * s2; it += 32) {
                    const int r2 = it / s2, e = it % s2, a = e / S, d = e % S;
                    const int q = pk(r, r2);
                    double2 tt = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) tt = cfma(xs[r * s2 + a * S + bb], sig[q * s2 + bb * S + d], tt);
                    acc[r2 * s2 + e] = cfma(cmk(wb[q], 0.0), tt, acc[r2 * s2 + e]);
                }
                __syncwarp();
            }
        } else if (has_next) {
            // ---- look-ahead: phase A of block b+1 over m > jhi, and its staging
            ret_phaseA<S, true>(g, grow, n, jlo2, nb2, jhi + 1, part, ACC(nxt), tid - 32, 224);
            ret_stage<S, VIE>(g, p, n, jlo2, nb2, SIG(nxt), WBF(nxt), MNV(nxt), QB(nxt), tid - 32, 224);
        }
        __syncthreads();
        if (!has_next) break;
        // ---- phase C: contribution of block b (m = jlo..jhi) to block b+1
        {
            const double2 *xs = XS(cur);
            constexpr int GC = 256 / E > 0 ? 256 / E : 1;
            for (int idx = tid; idx < GC * E; idx += 256) {
                const int gi = idx / E, e = idx % E, r = e / s2, ad = e % s2, a = ad / S, d = ad % S;
                double2 sum = cmk(0, 0);
                if (r < nb2) {
                    const int j = jlo2 + r;
#pragma unroll 4
                    for (int mm = gi; mm < nb; mm += GC) {
                        const int m = jlo + mm;
                        const double2 *sm = g.rret + (tri(m) + j) * s2 + d;
                        double2 tt = cmk(0, 0);
#pragma unroll
                        for (int bb = 0; bb < S; bb++) tt = cfma(xs[mm * s2 + a * S + bb], sm[bb * S], tt);
                        sum = cfma(cmk(greg_w(k, n - j, n - m), 0.0), tt, sum);
                    }
                }
                part[idx] = sum;
            }
            // the x values above block b+1 are the first K1 rows of block b's window
            for (int e = tid; e < K1 * s2; e += 256) XS(nxt)[nb2 * s2 + e] = xs[e];
            __syncthreads();
            double2 *acc = ACC(nxt);
            for (int e = tid; e < E; e += 256) {
                double2 v = acc[e];
                for (int gi = 0; gi < GC; gi++) v = cadd(v, part[gi * E + e]);
                acc[e] = v;
            }
            __syncthreads();
        }
    }
}

// =======================================================================================
// lesser component
// =======================================================================================
// acc[r] = sum_{m<mhi} w(j,m) Sigma^R(j,m) x_m, j = jlo + r; warp per row (warps w0..w0+nw-1)
template <int S>
__device__ void les_phaseA(const GroupDev &g, const double2 *xcol, int jlo, int nb, int mhi, double2 *acc,
                           double2 *redbase, int wi, int nw, int lane, int warp) {
    constexpr int s2 = S * S, LPG = S, NG = 32 / S;
    const int k = g.k;
    for (int r = wi; r < nb; r += nw) {
        const int j = jlo + r;
        const int mg = lane / LPG, dd = lane % LPG;
        double2 a_[S];
#pragma unroll
        for (int a = 0; a < S; a++) a_[a] = cmk(0, 0);
        if (mg < NG) {
            const double2 *srow = g.sret + tri(j) * s2;
            constexpr int U = S == 1 ? 4 : (S == 2 ? 2 : 1);
            int m = mg;
            for (; m + (U - 1) * NG < mhi; m += U * NG) {
                double2 sv[U][s2], xv[U][S];
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const long mu = m + u * NG;
#pragma unroll
                    for (int i = 0; i < s2; i++) sv[u][i] = srow[mu * s2 + i];
#pragma unroll
                    for (int b = 0; b < S; b++) xv[u][b] = xcol[mu * s2 + b * S + dd];
                }
#pragma unroll
                for (int u = 0; u < U; u++) {
                    const double w = greg_w(k, j, m + u * NG);
#pragma unroll
                    for (int a = 0; a < S; a++) {
                        double2 tt = cmk(0, 0);
#pragma unroll
                        for (int b = 0; b < S; b++) tt = cfma(sv[u][a * S + b], xv[u][b], tt);
                        a_[a] = cfma(cmk(w, 0.0), tt, a_[a]);
                    }
                }
            }
            for (; m < mhi; m += NG) {
                const double w = greg_w(k, j, m);
                const double2 *sm = srow + (long)m * s2;
                const double2 *xm = xcol + (long)m * s2;
#pragma unroll
                for (int a = 0; a < S; a++) {
                    double2 tt = cmk(0, 0);
#pragma unroll
                    for (int b = 0; b < S; b++) tt = cfma(sm[a * S + b], xm[b * S + dd], tt);
                    a_[a] = cfma(cmk(w, 0.0), tt, a_[a]);
                }
            }
        }
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
                for (int a = 0; a < S; a++) acc[r * s2 + a * S + dd] = a_[a];
        } else {
            double2 *red = redbase + warp * 32 * S;
            for (int a = 0; a < S; a++) red[lane * S + a] = (mg < NG) ? a_[a] : cmk(0, 0);
            __syncwarp();
            if (lane < S) {
                for (int a = 0; a < S; a++) {
                    double2 v = cmk(0, 0);
                    for (int g2 = 0; g2 < NG; g2++) v = cadd(v, red[(g2 * S + lane) * S + a]);
                    acc[r * s2 + a * S + lane] = v;
                }
            }
            __syncwarp();
        }
    }
}

template <int S, bool VIE>
__device__ void les_stage(const GroupDev &g, const ProbDev &p, int n, const double2 *gl, long ldc, int jlo, int nb,
                          double2 *sig, double *wb, double2 *minv, double2 *glb, int t, int nthr) {
    constexpr int s2 = S * S;
    const int k = g.k;
    for (int e = t; e < RetCfg<S>::TRI * s2; e += nthr) {
        const int q = e / s2, ab = e % s2;
        int r, r2;
        pk_inv(q, r, r2);
        if (r < nb) {
            sig[e] = g.sret[(tri(jlo + r) + jlo + r2) * s2 + ab];
            if (ab == 0) wb[q] = greg_w(k, jlo + r, jlo + r2);
        }
    }
    for (int e = t; e < nb * s2; e += nthr) {
        minv[e] = p.minv_les[(long)jlo * s2 + e];
        const int r = e / s2, ad = e % s2, a = ad / S, d = ad % S;
        glb[e] = gl[((long)(jlo + r) * S + a) * ldc + d];
        if (VIE) glb[e] = cadd(glb[e], p.qles[(tri(n) + jlo + r) * s2 + ad]);  // + Q^<(j,n), j <= n
    }
}

template <int S, bool VIE = false>
__global__ void __launch_bounds__(256, 2) k_les(GroupDev g, const ProbDev *__restrict__ probs, int n) {
    extern __shared__ double2 smem[];
    const ProbDev p = probs[blockIdx.x];
    const int k = g.k, K1 = k + 1, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int s2 = S * S, JB = RetCfg<S>::JB, E = RetCfg<S>::E;
    using L = VolLayout<S>;
    const double h = g.h;
    const long ldc = g.ldc;
    const double2 *gl = g.gles + (long)p.col * S;   // gles(j)[a][d] at gl[(j*S+a)*ldc + d]
    double2 *xcol = p.gles + tri(n) * s2;           // G^<(0..n, n)
    if (VIE) {
        les_start_block_vie<S>(g, p, n, gl, ldc, xcol, smem);
    } else {
        for (int ad = tid; ad < s2; ad += blockDim.x) {
            int a = ad / S, d = ad % S;
            xcol[ad] = cneg(cconj(p.gtv[((long)n * s2 + d * S + a) * (g.ntau + 1) + 0]));
        }
        __syncthreads();
        les_start_block<S>(g, p, n, gl, ldc, xcol, smem);
    }
    if (n <= k) return;
    double2 *part = smem + L::part, *qv = smem + L::qv, *red = smem + L::red;
    double2 ibd[NESSI_K1MAX + 1];
#pragma unroll
    for (int pp = 0; pp <= NESSI_K1MAX; pp++) ibd[pp] = cmk(0.0, pp <= K1 ? bd_w(k, pp) / h : 0.0);
    __shared__ double2 ibds[NESSI_K1MAX + 1];
    if (tid <= NESSI_K1MAX) ibds[tid] = cmk(0.0, tid <= K1 ? bd_w(k, tid) / h : 0.0);
    auto ACC = [&](int bf) { return smem + L::acc + bf * JB * s2; };
    auto SIG = [&](int bf) { return smem + L::sig + bf * L::TRI * s2; };
    auto WBF = [&](int bf) { return (double *)(smem + L::w + bf * L::WB); };
    auto MNV = [&](int bf) { return smem + L::minv + bf * JB * s2; };
    auto GLB = [&](int bf) { return smem + L::gl + bf * JB * s2; };
    auto XS = [&](int bf) { return smem + L::xs + bf * L::XS * s2; };
    const int jstart = K1;
    {
        const int jlo = jstart, jhi = jlo + JB - 1 > n ? n : jlo + JB - 1, nb = jhi - jlo + 1;
        les_phaseA<S>(g, xcol, jlo, nb, jlo, ACC(0), red, warp, 8, lane, warp);
        les_stage<S, VIE>(g, p, n, gl, ldc, jlo, nb, SIG(0), WBF(0), MNV(0), GLB(0), tid, 256);
        for (int e = tid; e < K1 * s2; e += 256) XS(0)[e] = xcol[(long)(jlo - K1) * s2 + e];
        __syncthreads();
    }
    for (int b = 0;; b++) {
        const int cur = b & 1, nxt = cur ^ 1;
        const int jlo = jstart + b * JB, jhi = jlo + JB - 1 > n ? n : jlo + JB - 1, nb = jhi - jlo + 1;
        const bool has_next = jhi < n;
        const int jlo2 = jhi + 1, jhi2 = jlo2 + JB - 1 > n ? n : jlo2 + JB - 1, nb2 = jhi2 - jlo2 + 1;
        if (warp == 0 && S <= 2) {
            les_chain<S, VIE>(ACC(cur), SIG(cur), WBF(cur), MNV(cur), GLB(cur), XS(cur), xcol + (long)jlo * s2, nb, K1,
                              ibds, h, lane);
        } else if (warp == 0) {
            double2 *acc = ACC(cur), *sig = SIG(cur), *minv = MNV(cur), *glb = GLB(cur), *xs = XS(cur);
            const double *wb = WBF(cur);
            for (int r = 0; r < nb; r++) {
                for (int e = lane; e < s2; e += 32) {
                    double2 q = cfma(cmk(VIE ? -h : h, 0.0), acc[r * s2 + e], glb[r * s2 + e]);
                    if (!VIE) {
#pragma unroll
                        for (int pp = 1; pp <= NESSI_K1MAX; pp++)
                            if (pp <= K1) q = csub(q, cmul(ibd[pp], xs[(r + K1 - pp) * s2 + e]));
                    }
                    qv[e] = q;
                }
                __syncwarp();
                for (int e = lane; e < s2; e += 32) {
                    const int a = e / S, d = e % S;
                    double2 x = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) x = cfma(minv[r * s2 + a * S + bb], qv[bb * S + d], x);
                    xs[(r + K1) * s2 + e] = x;
                    xcol[(long)(jlo + r) * s2 + e] = x;
                }
                __syncwarp();
                for (int it = lane; it < (nb - 1 - r) * s2; it += 32) {
                    const int r2 = r + 1 + it / s2, e = it % s2, a = e / S, d = e % S;
                    const int q = pk(r2, r);
                    double2 tt = cmk(0, 0);
#pragma unroll
                    for (int bb = 0; bb < S; bb++) tt = cfma(sig[q * s2 + a * S + bb], xs[(r + K1) * s2 + bb * S + d], tt);
                    acc[r2 * s2 + e] = cfma(cmk(wb[q], 0.0), tt, acc[r2 * s2 + e]);
                }
                __syncwarp();
            }
        } else if (has_next) {
            les_phaseA<S>(g, xcol, jlo2, nb2, jlo, ACC(nxt), red, warp - 1, 7, lane, warp);
            les_stage<S, VIE>(g, p, n, gl, ldc, jlo2, nb2, SIG(nxt), WBF(nxt), MNV(nxt), GLB(nxt), tid - 32, 224);
        }
        __syncthreads();
        if (!has_next) break;
        // ---- phase C: contribution of block b (m = jlo..jhi) to block b+1
        {
            const double2 *xs = XS(cur);
            constexpr int GC = 256 / E > 0 ? 256 / E : 1;
            for (int idx = tid; idx < GC * E; idx += 256) {
                const int gi = idx / E, e = idx % E, r = e / s2, ad = e % s2, a = ad / S, d = ad % S;
                double2 sum = cmk(0, 0);
                if (r < nb2) {
                    const int j = jlo2 + r;
                    const double2 *srow = g.sret + tri(j) * s2;
#pragma unroll 4
                    for (int mm = gi; mm < nb; mm += GC) {
                        const int m = jlo + mm;
                        double2 tt = cmk(0, 0);
#pragma unroll
                        for (int bb = 0; bb < S; bb++)
                            tt = cfma(srow[(long)m * s2 + a * S + bb], xs[(mm + K1) * s2 + bb * S + d], tt);
                        sum = cfma(cmk(greg_w(k, j, m), 0.0), tt, sum);
                    }
                }
                part[idx] = sum;
            }
            // x values below block b+1: the last K1 rows of block b's window
            for (int e = tid; e < K1 * s2; e += 256) XS(nxt)[e] = xs[nb * s2 + e];
            __syncthreads();
            double2 *acc = ACC(nxt);
            for (int e = tid; e < E; e += 256) {
                double2 v = acc[e];
                for (int gi = 0; gi < GC; gi++) v = cadd(v, part[gi * E + e]);
                acc[e] = v;
            }
            __syncthreads();
        }
    }
}
