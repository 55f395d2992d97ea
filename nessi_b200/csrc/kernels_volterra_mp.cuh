// Volterra recursions of one Dyson / VIE2 time step for size1 <= 2, several problems per CTA.
//
// The retarded row G^R(n, j), j = n-k-1 .. 0 (dyson_impl :158-213, vie2_impl :60-140) and the
// lesser column G^<(j, n), j = k+1 .. n (dyson_impl :983-1011, vie2_impl :847-990) are solved in
// blocks of 32 rows.  For a block, the sum over every row solved before it ("phase A") is
//   ret:  acc(j) = sum_{m > jhi} w(n-j, n-m) G(n,m) Sigma^R(m,j)
//   les:  acc(j) = sum_{m < jlo} w(j,m) Sigma^R(j,m) G^<(m,n)
// Sigma (F / Fcc for VIE2) is shared by all problems of a group, so a CTA takes PP <= 8 problems
// and computes phase A for all of them at once as a complex GEMM on the FP64 tensor cores
// (mma.sync m8n8k4 .f64), its operands staged through shared memory with cp.async: each Sigma
// tile is read once per CTA instead of once per problem.  Away from the diagonal (|m - j| > k) the
// Gregory weight depends on m alone (c_m: omega at the n / 0 end, else 1), so it is a column
// scale of the GEMM; the <= k terms next to the block are corrected to the exact weight
// afterwards.  Warp q then solves the block's rows of problem q with each lane owning one row in
// registers (as in the one-problem kernels), and the next block starts.  PP is chosen by the
// autotuner on the host.
#pragma once

#define MP_JB 32  // rows per block (lane = row)

template <int S> struct MpCfg {
    static constexpr int s2 = S * S;
    static constexpr int TRI = MP_JB * (MP_JB - 1) / 2;    // packed strictly-lower block triangle
    static constexpr int WSW = 2 * NESSI_K1MAX * NESSI_K1MAX * s2 + 2 * NESSI_K1MAX * s2 + 2;  // start work/warp
    static constexpr int KC = 32;                           // k per staged chunk (8 MMA k-steps)
    static constexpr int LDA = KC + 4;                      // padded row of a staged A chunk
    static constexpr int RMAX = MP_JB * S, NMAX = MP_JB * S;
    static constexpr int LDB = NMAX + 2;                    // padded row of a staged B chunk
    static constexpr int ASZ = RMAX * LDA, BSZ = KC * LDB;
    static constexpr int stage = 0;                         // 2 x (A chunk, B chunk)
    static constexpr int acc = stage + 2 * (ASZ + BSZ);     // 8 problems x 32 rows x s2: phase-A sums
    static constexpr int red = acc + 8 * MP_JB * s2;        // 8 warps x 32 lanes x 2 tiles x 2 double2
    static constexpr int sig = red + 8 * 32 * 4;            // TRI x s2
    static constexpr int wb = sig + TRI * s2;               // TRI doubles
    static constexpr int total = wb + TRI / 2 + 1;
    static_assert(acc >= 8 * WSW, "start workspaces must fit in the staging buffers");
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_but_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// D += A B on the FP64 tensor cores, one 8x8x4 tile: lane holds A[lane/4][lane%4],
// B[lane%4][lane/4] and D[lane/4][2(lane%4) + {0,1}] (mma.m8n8k4 .f64 fragment layout).
__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Phase A as a complex GEMM C (R x N) = A (R x K) B (K x N), R, N <= 32 S, with the operands
// staged in shared memory: chunks of KC k-values of A and B are copied with cp.async (double
// buffered, every thread issuing copies, so many loads are in flight), and the warps take their
// MMA fragments from the padded chunks (A rows padded to LDA = KC + 4, B rows to LDB = N + 2,
// which keeps the fragment reads free of bank conflicts).  srcA(r, kk) / srcB(kk, c) give the
// address of an operand element or nullptr for a zero; wA(kk) / wB(kk) scale column kk of A /
// row kk of B.  The 8 warps share the 8x8 tiles, or the k-steps of a chunk when there are fewer
// than 8 tiles (then summed in warp order).  put(r, c, value) stores an element of C.
template <int S, class SA, class SB, class WA, class WB, class PUT>
__device__ void zgemm_staged(const SA &srcA, const SB &srcB, const WA &wA, const WB &wB, const PUT &put, int R,
                             int N, int K, double2 *stage, double2 *red, int tid) {
    using C = MpCfg<S>;
    const int warp = tid >> 5, lane = tid & 31;
    const int MT = (R + 7) / 8, NT = (N + 7) / 8, tiles = MT * NT;
    const int ksplit = tiles >= 8 ? 1 : 8 / tiles;
    const int nmy = tiles >= 8 ? (tiles - warp + 7) / 8 : (warp / tiles < ksplit ? 1 : 0);  // tiles of this warp
    double c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    const int nch = (K + C::KC - 1) / C::KC;
    auto load = [&](int ch, int buf) {
        double2 *As = stage + buf * (C::ASZ + C::BSZ), *Bs = As + C::ASZ;
        const int k0 = ch * C::KC;
        for (int e = tid; e < R * C::KC; e += 256) {
            const int r = e / C::KC, kk = e % C::KC;
            const double2 *src = k0 + kk < K ? srcA(r, k0 + kk) : nullptr;
            if (src) cp_async16(As + r * C::LDA + kk, src);
            else As[r * C::LDA + kk] = cmk(0, 0);
        }
        for (int e = tid; e < C::KC * N; e += 256) {
            const int kk = e / N, cc = e % N;
            const double2 *src = k0 + kk < K ? srcB(k0 + kk, cc) : nullptr;
            if (src) cp_async16(Bs + kk * C::LDB + cc, src);
            else Bs[kk * C::LDB + cc] = cmk(0, 0);
        }
        cp_async_commit();
    };
    if (nch > 0) load(0, 0);
    for (int ch = 0; ch < nch; ch++) {
        if (ch + 1 < nch) { load(ch + 1, (ch + 1) & 1); cp_async_wait_all_but_one(); }
        else cp_async_wait_all();
        __syncthreads();
        const double2 *As = stage + (ch & 1) * (C::ASZ + C::BSZ), *Bs = As + C::ASZ;
        const int k0 = ch * C::KC;
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (i >= nmy) break;
            const int t = tiles >= 8 ? warp + 8 * i : warp % tiles;
            const int ksl = tiles >= 8 ? 0 : warp / tiles;
            const int ar = (t / NT) * 8 + (lane >> 2), bc = (t % NT) * 8 + (lane >> 2), kq = lane & 3;
#pragma unroll
            for (int ks = 0; ks < C::KC / 4; ks++) {
                if (ks % ksplit != ksl) continue;
                const int kk = ks * 4 + kq;
                const double2 a = cscale(As[ar * C::LDA + kk], wA(k0 + kk));
                const double2 b = cscale(Bs[kk * C::LDB + bc], wB(k0 + kk));
                dmma884(c[i][0], c[i][1], a.x, b.x);
                dmma884(c[i][0], c[i][1], -a.y, b.y);
                dmma884(c[i][2], c[i][3], a.x, b.y);
                dmma884(c[i][2], c[i][3], a.y, b.x);
            }
        }
        __syncthreads();
    }
    const int r0 = lane >> 2, c0 = 2 * (lane & 3);
    if (tiles >= 8) {
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (i >= nmy) break;
            const int t = warp + 8 * i;
            const int r = (t / NT) * 8 + r0, cc = (t % NT) * 8 + c0;
            put(r, cc, cmk(c[i][0], c[i][2]));
            put(r, cc + 1, cmk(c[i][1], c[i][3]));
        }
        __syncthreads();
        return;
    }
    red[(warp * 32 + lane) * 2] = cmk(c[0][0], c[0][2]);
    red[(warp * 32 + lane) * 2 + 1] = cmk(c[0][1], c[0][3]);
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
template <int S, bool VIE>
__device__ void mp_ret_chain(double2 *a_, const double2 *sig, const double *wb, const ProbDev &p, const double2 *grow,
                             int n, int jlo, int nb, int K1, const double2 *ibd, double h, int lane) {
    constexpr int s2 = S * S;
    const int r = lane;
    const bool own = r < nb;
    double2 bd[s2], mi[s2];
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
template <int S, bool VIE>
__device__ void mp_les_chain(double2 *a_, const double2 *sig, const double *wb, const ProbDev &p, const double2 *gl,
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
        gv[e] = own ? gl[((long)(jlo + r) * S + a) * ldc + d] : cmk(0, 0);
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

// ======================================================================================
// retarded component
// ======================================================================================
// Phase A of block [jlo, jhi] for the CTA's problems q as C[(q,a)][(jj,d)] =
//   sum_{(m,b)} c_m G_q(n,m)[a][b] Sigma^R(m, jlo+jj)[b][d],  m = jhi+1 .. n.
template <int S, bool VIE>
__global__ void __launch_bounds__(256) k_ret_mp(GroupDev g, const ProbDev *__restrict__ probs, int n, int nact,
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
        double2 *ws = smem + C::stage + warp * C::WSW;
        if (VIE) ret_start_block_vie<S, WarpExec>(g, p, n, ws, WarpExec{lane});
        else ret_start_block<S, WarpExec>(g, p, n, ws, WarpExec{lane});
    }
    __syncthreads();
    double2 *acc_s = smem + C::acc, *red = smem + C::red, *sig = smem + C::sig;
    double *wb = (double *)(smem + C::wb);
    const int jtop = n - k - 1;
    for (int jhi = jtop; jhi >= 0; jhi -= MP_JB) {
        const int jlo = jhi - MP_JB + 1 < 0 ? 0 : jhi - MP_JB + 1, nb = jhi - jlo + 1;
        for (int e = tid; e < C::TRI * s2; e += 256) {
            const int q = e / s2, ab = e % s2;
            int r, r2;
            pk_inv(q, r, r2);
            if (r < nb) {
                sig[e] = g.rret[(tri(jlo + r) + jlo + r2) * s2 + ab];
                if (ab == 0) wb[q] = greg_w(k, n - (jlo + r2), n - (jlo + r));
            }
        }
        const int mb = jhi + 1;
        auto srcA = [&](int r, int kk) -> const double2 * {
            const int q = r / S, a = r % S, m = mb + kk / S, b = kk % S;
            return (q < np && m <= n) ? rows[q] + (long)m * s2 + a * S + b : nullptr;
        };
        auto srcB = [&](int kk, int cc) -> const double2 * {
            const int m = mb + kk / S, b = kk % S, jj = cc / S, d = cc % S;
            return (m <= n && jj < nb) ? g.rret + (tri(m) + jlo + jj) * s2 + b * S + d : nullptr;
        };
        auto wA = [&](int kk) -> double {
            const int m = mb + kk / S;
            return m <= n ? ret_cw(k, n, m) : 0.0;
        };
        auto wB = [](int) -> double { return 1.0; };
        auto put = [&](int r, int cc, double2 v) {
            const int q = r / S, a = r % S, jj = cc / S, d = cc % S;
            if (q < np && jj < MP_JB) acc_s[(q * MP_JB + jj) * s2 + a * S + d] = v;
        };
        zgemm_staged<S>(srcA, srcB, wA, wB, put, np * S, MP_JB * S, (n - jhi) * S, smem + C::stage, red, tid);
        if (owner) {
            const double2 *grow = rows[warp];
            const int j = jlo + lane;
            double2 acc[s2];
#pragma unroll
            for (int e = 0; e < s2; e++) acc[e] = lane < nb ? acc_s[(warp * MP_JB + lane) * s2 + e] : cmk(0, 0);
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
                            acc[aa * S + d] = cfma(cmk(dw, 0.0), t, acc[aa * S + d]);
                        }
                }
            }
            mp_ret_chain<S, VIE>(acc, sig, wb, p, grow, n, jlo, nb, K1, ibd, h, lane);
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
__global__ void __launch_bounds__(256) k_les_mp(GroupDev g, const ProbDev *__restrict__ probs, int n, int nact,
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
        double2 *ws = smem + C::stage + warp * C::WSW;
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
    double2 *acc_s = smem + C::acc, *red = smem + C::red, *sig = smem + C::sig;
    double *wb = (double *)(smem + C::wb);
    for (int jlo = K1; jlo <= n; jlo += MP_JB) {
        const int jhi = jlo + MP_JB - 1 > n ? n : jlo + MP_JB - 1, nb = jhi - jlo + 1;
        for (int e = tid; e < C::TRI * s2; e += 256) {
            const int q = e / s2, ab = e % s2;
            int r, r2;
            pk_inv(q, r, r2);
            if (r < nb) {
                sig[e] = g.sret[(tri(jlo + r) + jlo + r2) * s2 + ab];
                if (ab == 0) wb[q] = greg_w(k, jlo + r, jlo + r2);
            }
        }
        auto srcA = [&](int r, int kk) -> const double2 * {
            const int jj = r / S, a = r % S, m = kk / S, b = kk % S;
            return (jj < nb && m < jlo) ? g.sret + (tri(jlo + jj) + m) * s2 + a * S + b : nullptr;
        };
        auto srcB = [&](int kk, int cc) -> const double2 * {
            const int m = kk / S, b = kk % S, q = cc / S, d = cc % S;
            return (q < np && m < jlo) ? cols[q] + (long)m * s2 + b * S + d : nullptr;
        };
        auto wA = [](int) -> double { return 1.0; };
        auto wB = [&](int kk) -> double {
            const int m = kk / S;
            return m < jlo ? les_cw(k, m) : 0.0;
        };
        auto put = [&](int r, int cc, double2 v) {
            const int jj = r / S, a = r % S, q = cc / S, d = cc % S;
            if (q < np && jj < MP_JB) acc_s[(q * MP_JB + jj) * s2 + a * S + d] = v;
        };
        zgemm_staged<S>(srcA, srcB, wA, wB, put, MP_JB * S, np * S, jlo * S, smem + C::stage, red, tid);
        if (owner) {
            double2 *xcol = cols[warp];
            const int j = jlo + lane;
            double2 acc[s2];
#pragma unroll
            for (int e = 0; e < s2; e++) acc[e] = lane < nb ? acc_s[(warp * MP_JB + lane) * s2 + e] : cmk(0, 0);
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
                            acc[aa * S + d] = cfma(cmk(dw, 0.0), t, acc[aa * S + d]);
                        }
                }
            }
            mp_les_chain<S, VIE>(acc, sig, wb, p, gl, ldc, xcol, n, jlo, nb, K1, ibd, h, lane);
        }
        __syncthreads();
    }
}
