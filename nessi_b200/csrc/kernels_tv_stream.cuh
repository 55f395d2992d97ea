// k_tv_stream: the G^tv row of a Dyson / VIE2 time step (dyson_impl :651-741, vie2_impl :645-725)
// for every problem of a group, with the history read into shared memory by the bulk-copy engine
// (cp.async.bulk global -> shared, completion counted in bytes on an mbarrier):
//   Q(tau) = sum_{j<n} a_j G^tv(j, tau) + Cmat(tau) [+ Q^tv(n, tau) for VIE2]
//   G^tv(n, tau) = Minv_les[n] Q(tau)
// a_j = tvcoef (k_prep_group), Cmat = K_n Gmat_all (the Matsubara integral as one group GEMM).
//
// The history stream is the HBM-bound part of a time step.  The register-load form (k_tv: a
// thread per (tau, column), 4 rows in flight per thread) needs 64 warps per SM to keep enough bytes
// in flight.  Here one persistent CTA per SM keeps up to five stages of ~32 KB in flight through
// the bulk-copy engine, and 8 consumer warps reduce them.
//
// Work items are (problem, tau chunk of width tw); CTA b takes items b, b + G, b + 2G, ... and the
// stages of all its items form one sequence through a ring of STAGES buffers.  A stage holds the
// coefficients a_j of rows r0 .. r0+nr-1 and those rows of the item's history, each row as s^2
// segments (one per element plane e = b s + d of the plane layout (t s^2 + e)(ntau+1) + tau) of tw
// complex: FP32 rows first (mixed precision, j < n-k-1), then FP64 rows.  Lane 0 of warp 8 issues
// the copies.  An FP64 segment starts on a
// 16-byte boundary; an FP32 segment may start 8 bytes past one, and then its copy starts 8 bytes
// early and ends on the next boundary (the consumers index one element on).  The <= 8 bytes read
// before and after a segment lie in the same problem's G^tv buffer: in the previous plane or row,
// or in row n, which exists since n <= nt.  Warps 0-7 own (tau, d) pairs q = t + 256 i and
// accumulate sum_b a_j[a][b] G^tv(j)[b][d](tau) in registers over the rows in order; the solve
// with Minv_les[n] needs only the pair's own column, so there is no reduction.
//
// Every mbarrier wait is bounded (TvsPlan::wait_ns of %globaltimer).  A wait that gives up sets
// *err = NESSI_ERR_TIMEOUT and a shared abort flag; every warp then leaves its loop, the CTA waits
// (bounded again) for the copies it has in flight, and returns without writing G^tv(n).
#pragma once
#include <stdint.h>
#include "kernels_dyson.cuh"

namespace tvs {
constexpr int NCW = 8;                // consumer warps
constexpr int NCT = NCW * 32;         // consumer threads
constexpr int NTH = NCT + 32;         // + the producer warp
constexpr int STAGES = 6;             // ring buffers
constexpr int SEG_TARGET = 32768;     // bytes of a stage's history segments (at least one row)
constexpr int TIMEOUT_CODE = 5;       // NESSI_ERR_TIMEOUT
}  // namespace tvs

// (tau, d) pairs per consumer thread; the widest tau chunk is SLOTS * 256 / S
template <int S> struct TvsCfg {
    static constexpr int SLOTS = S == 1 ? 4 : (S <= 3 ? 2 : 1);
    static constexpr int TWMAX = SLOTS * tvs::NCT / S;
};

// Decomposition of one launch, chosen on the host (tv_stream_plan).
struct TvsPlan {
    int tw;              // tau chunk width (complex)
    int nch;             // chunks per problem: ceil((ntau+1) / tw)
    int items;           // nact * nch
    int r64, r32;        // history rows per stage, FP64 / FP32
    int slot64, slot32;  // bytes of one segment's slot in a stage (multiples of 16)
    int coef;            // bytes of a stage's coefficient area (max(r64, r32) s^2 complex)
    int stb;             // bytes of one stage: coef + segments (multiple of 16)
    long long wait_ns;   // bound of every mbarrier wait
    int *err;            // set to NESSI_ERR_TIMEOUT when a wait gave up
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t a, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t a, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t a) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t a, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the completion of phase `parity`; false when limit_ns passed first, or (abort != null)
// when another thread of the CTA gave up.  A bound <= 0 gives up at once (exercises the timeout path).
__device__ __forceinline__ bool mbar_wait(uint32_t a, uint32_t parity, long long limit_ns, const volatile int *abort) {
    if (limit_ns <= 0) return false;
    if (mbar_try(a, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try(a, parity)) return true;
        if (abort && *abort) return false;
        if ((long long)(global_ns() - t0) > limit_ns) return false;
    }
}
// global -> shared bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) that
// counts its bytes on the mbarrier at `bar`; no multicast
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Offset (0 or 1 elements) of an FP32 segment's first element past the 16-byte boundary below it.
__device__ __forceinline__ int f32_off(const float2 *p) { return (int)(((uintptr_t)p >> 3) & 1); }

template <int S, bool MIXED, bool VIE>
__global__ void __maxnreg__(64) k_tv_stream(GroupDev g, const ProbDev *__restrict__ probs, int n, TvsPlan pl) {
    using namespace tvs;
    constexpr int s2 = S * S, SL = TvsCfg<S>::SLOTS;
    extern __shared__ __align__(128) unsigned char tsm[];
    __shared__ __align__(8) unsigned long long bar_full[STAGES], bar_empty[STAGES];
    __shared__ int s_abort;
    __shared__ long long s_issued;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int M = g.ntau + 1;
    const long rowe = (long)s2 * M;  // complex of one history row
    const int j64 = MIXED ? max(n - g.k - 1, 0) : 0;  // first FP64 row
    const int ns32 = MIXED ? (j64 + pl.r32 - 1) / pl.r32 : 0;
    const int nsi = ns32 + (n - j64 + pl.r64 - 1) / pl.r64;  // stages of one item
    const int nmine = (int)blockIdx.x < pl.items ? (pl.items - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const long nstage = (long)nmine * nsi;
    const uint32_t sbase = smem_u32(tsm);
    if (threadIdx.x == 0) {
        for (int i = 0; i < STAGES; i++) {
            mbar_init(smem_u32(&bar_full[i]), 1);
            mbar_init(smem_u32(&bar_empty[i]), NCW);
        }
        s_abort = 0;
        s_issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    volatile int *abort = &s_abort;

    if (warp == NCW) {
        // ---- producer: lane 0 issues every stage of this CTA's items ----
        if (lane == 0) {
            long i = 0;
            for (; i < nstage; i++) {
                const int buf = (int)(i % STAGES);
                if (i >= STAGES &&
                    !mbar_wait(smem_u32(&bar_empty[buf]), (uint32_t)((i / STAGES - 1) & 1), pl.wait_ns, abort)) {
                    atomicExch(pl.err, TIMEOUT_CODE);
                    *abort = 1;
                    break;
                }
                if (*abort) break;
                const int item = (int)blockIdx.x + (int)(i / nsi) * (int)gridDim.x, si = (int)(i % nsi);
                const ProbDev *p = probs + item / pl.nch;
                const int tau0 = (item % pl.nch) * pl.tw, tw = min(pl.tw, M - tau0);
                const bool f32 = si < ns32;
                const int r0 = f32 ? si * pl.r32 : j64 + (si - ns32) * pl.r64;
                const int nr = f32 ? min(pl.r32, j64 - r0) : min(pl.r64, n - r0);
                const uint32_t fb = smem_u32(&bar_full[buf]), st0 = sbase + (uint32_t)buf * (uint32_t)pl.stb;
                const uint32_t cbytes = (uint32_t)(nr * s2 * 16), dst0 = st0 + (uint32_t)pl.coef;
                if (f32) {
                    const float2 *g32 = p->gtv32;
                    uint32_t bytes = cbytes;
                    for (int r = 0; r < nr; r++)
                        for (int e = 0; e < s2; e++) {
                            const float2 *src = g32 + ((long)(r0 + r) * s2 + e) * M + tau0;
                            bytes += (uint32_t)(((tw + f32_off(src)) * 8 + 15) & ~15);
                        }
                    mbar_arrive_expect_tx(fb, bytes);
                    bulk_g2s(st0, g.tvcoef + (long)r0 * s2, cbytes, fb);
                    for (int r = 0; r < nr; r++)
                        for (int e = 0; e < s2; e++) {
                            const float2 *src = g32 + ((long)(r0 + r) * s2 + e) * M + tau0;
                            const int off = f32_off(src);
                            bulk_g2s(dst0 + (uint32_t)((r * s2 + e) * pl.slot32), src - off,
                                     (uint32_t)(((tw + off) * 8 + 15) & ~15), fb);
                        }
                } else {
                    const double2 *g64 = p->gtv;
                    mbar_arrive_expect_tx(fb, cbytes + (uint32_t)(nr * s2 * tw * 16));
                    bulk_g2s(st0, g.tvcoef + (long)r0 * s2, cbytes, fb);
                    for (int r = 0; r < nr; r++)
                        for (int e = 0; e < s2; e++)
                            bulk_g2s(dst0 + (uint32_t)((r * s2 + e) * pl.slot64),
                                     g64 + ((long)(r0 + r) * s2 + e) * M + tau0, (uint32_t)(tw * 16), fb);
                }
            }
            s_issued = i;
        }
    } else {
        // ---- consumers: warps 0..7 ----
        const int t = threadIdx.x;
        long i = 0;
        for (int ii = 0; ii < nmine; ii++) {
            const int item = (int)blockIdx.x + ii * (int)gridDim.x;
            const ProbDev *p = probs + item / pl.nch;
            const int tau0 = (item % pl.nch) * pl.tw, tw = min(pl.tw, M - tau0), npair = tw * S;
            // the thread's pairs: plane offset d and tau offset tl, hoisted out of the row loops
            int sd[SL], stl[SL];
            bool sv[SL];
#pragma unroll
            for (int sl = 0; sl < SL; sl++) {
                const int q = t + sl * NCT;
                sv[sl] = q < npair;
                sd[sl] = S == 1 ? 0 : q / tw;
                stl[sl] = q - sd[sl] * tw;
            }
            // FP32 segments: parity of the first element's 8-byte offset at row 0, per (slot, b);
            // row j adds j s^2 M (the planes of one row are M apart)
            int par0[SL][S];
            if (MIXED) {
                const long base = (long)(((uintptr_t)p->gtv32 >> 3) & 1);
#pragma unroll
                for (int sl = 0; sl < SL; sl++)
#pragma unroll
                    for (int b = 0; b < S; b++) par0[sl][b] = (int)((base + (long)(b * S + sd[sl]) * M + tau0) & 1);
            }
            const int rowpar = (int)(rowe & 1);
            double2 acc[SL][S];
#pragma unroll
            for (int sl = 0; sl < SL; sl++)
#pragma unroll
                for (int a = 0; a < S; a++) acc[sl][a] = cmk(0, 0);
            bool ok = true;
            for (int si = 0; si < nsi; si++, i++) {
                const int buf = (int)(i % STAGES);
                int got = 1;
                if (lane == 0) got = mbar_wait(smem_u32(&bar_full[buf]), (uint32_t)((i / STAGES) & 1), pl.wait_ns, abort);
                got = __shfl_sync(0xffffffffu, got, 0);
                if (!got) {
                    if (lane == 0) {
                        atomicExch(pl.err, TIMEOUT_CODE);
                        *abort = 1;
                    }
                    ok = false;
                    break;
                }
                const bool f32 = si < ns32;
                const int r0 = f32 ? si * pl.r32 : j64 + (si - ns32) * pl.r64;
                const int nr = f32 ? min(pl.r32, j64 - r0) : min(pl.r64, n - r0);
                const unsigned char *stg = tsm + (long)buf * pl.stb;
                const double2 *cst = (const double2 *)stg;
                const unsigned char *seg0 = stg + pl.coef;
                for (int r = 0; r < nr; r++) {
                    const double2 *cj = cst + r * s2;  // a_j, broadcast from shared memory
                    const int pj = MIXED ? (((r0 + r) & rowpar)) : 0;
#pragma unroll
                    for (int sl = 0; sl < SL; sl++) {
                        if (sv[sl]) {
                            double2 x[S];
#pragma unroll
                            for (int b = 0; b < S; b++) {
                                const int seg = r * s2 + b * S + sd[sl];
                                if (MIXED && f32) {
                                    const int off = par0[sl][b] ^ pj;
                                    const float2 f = *(const float2 *)(seg0 + seg * pl.slot32 + (off + stl[sl]) * 8);
                                    x[b] = cmk((double)f.x, (double)f.y);
                                } else {
                                    x[b] = *(const double2 *)(seg0 + seg * pl.slot64 + stl[sl] * 16);
                                }
                            }
#pragma unroll
                            for (int a = 0; a < S; a++)
#pragma unroll
                                for (int b = 0; b < S; b++) acc[sl][a] = cfma(cj[a * S + b], x[b], acc[sl][a]);
                        }
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(smem_u32(&bar_empty[buf]));
            }
            if (__any_sync(0xffffffffu, !ok || *abort)) break;
            // Matsubara part, VIE2 source, solve with Minv_les[n]; store row n (and its FP32 copy)
            const double2 *mi = p->minv_les + (long)n * s2;
            double2 *gout = p->gtv + (long)n * rowe;
            float2 *gout32 = MIXED ? p->gtv32 + (long)n * rowe : nullptr;
            const double2 *qt = VIE ? p->qtv + (long)n * rowe : nullptr;
            const int col = p->col;
#pragma unroll
            for (int sl = 0; sl < SL; sl++) {
                if (sv[sl]) {
                    const int d = sd[sl], tau = tau0 + stl[sl];
                    double2 v[S];
#pragma unroll
                    for (int a = 0; a < S; a++) {
                        v[a] = cadd(acc[sl][a], g.Cmat[((long)tau * S + a) * g.ldc + (long)col * S + d]);
                        if (VIE) v[a] = cadd(v[a], qt[(long)(a * S + d) * M + tau]);
                    }
#pragma unroll
                    for (int a = 0; a < S; a++) {
                        double2 x = cmk(0, 0);
#pragma unroll
                        for (int b = 0; b < S; b++) x = cfma(mi[a * S + b], v[b], x);
                        gout[(long)(a * S + d) * M + tau] = x;
                        if (MIXED) gout32[(long)(a * S + d) * M + tau] = make_float2((float)x.x, (float)x.y);
                    }
                }
            }
        }
    }
    __syncthreads();
    // after an abort: wait (bounded) for the copies still in flight before the CTA's shared memory goes
    if (*abort && threadIdx.x == NCT) {
        const long hi = s_issued, lo = hi > STAGES ? hi - STAGES : 0;
        for (long i = lo; i < hi; i++)
            mbar_wait(smem_u32(&bar_full[i % STAGES]), (uint32_t)((i / STAGES) & 1), 2000000000LL, nullptr);
    }
}
