// Complex FP64 GEMM tiles on the FP64 tensor cores (mma.sync m16n8k8 .f64), the contraction
// engine of every Sigma-shared product of a time step:
//   Matsubara part of the tv row      Cmat = K_n . Gmat_all          (conv_impl :410-540)
//   les*adv                           gles = Sigma^<_dense . badv     (conv_impl :1244-1394)
//   tv*vt                             gles += Sigma^tv . btv          (conv_impl :1075-1242)
//   Volterra trailing updates         acc += Sigma^R . X_panel        (dyson_impl :179-213, :983-1011)
// In all of them the rows are time indices (t, a) and the columns are the problems of a group
// (p, d), so one product serves every k-point that shares Sigma.
//
// A tile group of 4 warps (128 threads) computes a BM x BN tile of C = A B (complex, row-major
// C[r][c]); each warp owns a (16 MT) x (8 NT) sub-tile as MT x NT m16n8 fragments (32 x 32 or
// 32 x 16), real and imaginary parts accumulated separately (four real MMAs per complex fragment
// product).  The smaller warp tile doubles the tiles of a product, for shapes that give too few
// 64 x 64 tiles to fill the 148 SMs.  Operands are read through loader objects, so that a GEMM
// can read a triangle, a scaled panel or a dense matrix in place: get(mn, k) returns A(m, k) (or B(k, n)) and zero outside the operand; KC tells
// whether consecutive k are adjacent in memory (then consecutive threads load consecutive k,
// otherwise consecutive m / n).  The k loop stages BK complex columns of A and rows of B per
// step through double-buffered shared memory, loading the next step into registers while the
// current one is multiplied; one barrier of the tile group per step.
#pragma once
#include "device_common.cuh"

namespace zg {
constexpr int BK = 8;        // complex k per stage (one m16n8k8 k-step)
constexpr int LDS = BK + 4;  // shared row stride in complex: 12 = 4 (mod 8) -> conflict-free fragment loads
constexpr int NTH = 128;     // threads of a tile group
// shared memory (complex elements) of one tile group
template <int BM, int BN> struct Smem {
    static constexpr int stage = (BM + BN) * LDS;
    static constexpr int total = 2 * stage;
};
}  // namespace zg

// D (16x8, fp64) += A (16x8) B (8x8); fragment layout of mma.m16n8k8 .f64: with g = lane/4,
// q = lane%4: a[v0 + 2 v1] = A[g + 8 v0][q + 4 v1], b[v] = B[q + 4 v][g],
// d[v0 + 2 v1] = D[g + 8 v1][2 q + v0].
__device__ __forceinline__ void dmma1688(double *d, const double *a, const double *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// barrier of the 128 threads of tile group `grp` (named barriers 1 + grp; 0 is __syncthreads)
__device__ __forceinline__ void zg_sync(int grp) { asm volatile("bar.sync %0, 128;" ::"r"(grp + 1) : "memory"); }

// C tile (m0.., n0..) of C = A B over k = 0..K-1, by the 128 threads t = 0..127 of tile group grp.
// Every element of the tile goes through the store object `put` (the loaders return zero outside
// A and B, so rows / columns beyond the matrices carry zeros; put filters them).
template <int BM, int BN, class LA, class LB, class PUT, int NT = 4>
__device__ __forceinline__ void zgemm_tile(const LA &la, const LB &lb, const PUT &put, int m0, int n0, int K,
                                           double2 *sm, int t, int grp) {
    using namespace zg;
    constexpr int MT = 2, WTN = 8 * NT;  // warp tile 32 x WTN
    constexpr int WN = BN / WTN, WM = BM / 32;
    static_assert(WM * WN == 4, "tile group = 4 warps");
    constexpr int AE = BM * BK / NTH, BE = BN * BK / NTH;
    double2 *As0 = sm, *Bs0 = sm + BM * LDS;
    const int warp = t >> 5, lane = t & 31, wm = warp / WN, wn = warp % WN;
    const int g = lane >> 2, q = lane & 3;
    double acc[MT][NT][2][4];
#pragma unroll
    for (int i = 0; i < MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int c = 0; c < 2; c++)
#pragma unroll
                for (int e = 0; e < 4; e++) acc[i][j][c][e] = 0.0;
    double2 ra[AE], rb[BE];
    auto gload = [&](int k0) {
#pragma unroll
        for (int i = 0; i < AE; i++) {
            const int idx = t + NTH * i;
            const int m = LA::KC ? idx / BK : idx % BM, k = LA::KC ? idx % BK : idx / BM;
            ra[i] = la.get(m0 + m, k0 + k);
        }
#pragma unroll
        for (int i = 0; i < BE; i++) {
            const int idx = t + NTH * i;
            const int n = LB::KC ? idx / BK : idx % BN, k = LB::KC ? idx % BK : idx / BN;
            rb[i] = lb.get(n0 + n, k0 + k);
        }
    };
    auto sstore = [&](int buf) {
        double2 *As = As0 + buf * Smem<BM, BN>::stage, *Bs = Bs0 + buf * Smem<BM, BN>::stage;
#pragma unroll
        for (int i = 0; i < AE; i++) {
            const int idx = t + NTH * i;
            const int m = LA::KC ? idx / BK : idx % BM, k = LA::KC ? idx % BK : idx / BM;
            As[m * LDS + k] = ra[i];
        }
#pragma unroll
        for (int i = 0; i < BE; i++) {
            const int idx = t + NTH * i;
            const int n = LB::KC ? idx / BK : idx % BN, k = LB::KC ? idx % BK : idx / BN;
            Bs[n * LDS + k] = rb[i];
        }
    };
    const int nk = (K + BK - 1) / BK;
    if (nk > 0) {
        gload(0);
        sstore(0);
        zg_sync(grp);
    }
    for (int kt = 0; kt < nk; kt++) {
        const int cur = kt & 1;
        if (kt + 1 < nk) gload((kt + 1) * BK);
        const double2 *As = As0 + cur * Smem<BM, BN>::stage + (wm * 32) * LDS;
        const double2 *Bs = Bs0 + cur * Smem<BM, BN>::stage + (wn * WTN) * LDS;
        double ar[MT][4], ai[MT][4], an[MT][4], br[NT][2], bi[NT][2];
#pragma unroll
        for (int i = 0; i < MT; i++)
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const double2 x = As[(i * 16 + g + 8 * (v & 1)) * LDS + q + 4 * (v >> 1)];
                ar[i][v] = x.x;
                ai[i][v] = x.y;
                an[i][v] = -x.y;
            }
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int v = 0; v < 2; v++) {
                const double2 x = Bs[(j * 8 + g) * LDS + q + 4 * v];
                br[j][v] = x.x;
                bi[j][v] = x.y;
            }
#pragma unroll
        for (int i = 0; i < MT; i++)
#pragma unroll
            for (int j = 0; j < NT; j++) {
                dmma1688(acc[i][j][0], ar[i], br[j]);
                dmma1688(acc[i][j][0], an[i], bi[j]);
                dmma1688(acc[i][j][1], ar[i], bi[j]);
                dmma1688(acc[i][j][1], ai[i], br[j]);
            }
        if (kt + 1 < nk) sstore(cur ^ 1);
        zg_sync(grp);
    }
    // epilogue: an accumulating store first reads every old value of the thread's fragments (the
    // loads are independent and overlap), then writes all sums
    double2 old[MT][NT][4];
    if (put.accumulates()) {
#pragma unroll
        for (int i = 0; i < MT; i++)
#pragma unroll
            for (int j = 0; j < NT; j++)
#pragma unroll
                for (int e = 0; e < 4; e++)
                    old[i][j][e] = put.load(m0 + wm * 32 + i * 16 + g + 8 * (e >> 1), n0 + wn * WTN + j * 8 + 2 * q + (e & 1));
    }
#pragma unroll
    for (int i = 0; i < MT; i++)
#pragma unroll
        for (int j = 0; j < NT; j++)
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int r = m0 + wm * 32 + i * 16 + g + 8 * (e >> 1);
                const int c = n0 + wn * WTN + j * 8 + 2 * q + (e & 1);
                const double2 v = cmk(acc[i][j][0][e], acc[i][j][1][e]);
                put.store(r, c, put.accumulates() ? put.combine(old[i][j][e], v) : put.combine(cmk(0, 0), v));
            }
}

// ---- loaders and stores of the standalone products -----------------------------------------
// A(m, k) = p[m * ld + k] (row-major, k contiguous)
struct LdRowK {
    static constexpr bool KC = true;
    const double2 *p;
    long ld;
    int rows, cols;
    __device__ __forceinline__ double2 get(int m, int k) const {
        return (m < rows && k < cols) ? __ldg(p + (long)m * ld + k) : cmk(0, 0);
    }
};
// B(k, n) = p[k * ld + n] (row-major, n contiguous), read as get(n, k)
struct LdRowN {
    static constexpr bool KC = false;
    const double2 *p;
    long ld;
    int rows, cols;  // rows = K extent, cols = N extent
    __device__ __forceinline__ double2 get(int n, int k) const {
        return (n < cols && k < rows) ? __ldg(p + (long)k * ld + n) : cmk(0, 0);
    }
};
// Stores of a GEMM tile: accumulates() tells whether C's old value takes part, load(r, c) reads
// it (zero outside C), combine(old, v) forms the new value and store(r, c, x) writes it inside C.
// C[r][c] = alpha v (+ C[r][c] when accumulate), r < rows, c < cols
struct StRow {
    double2 *p;
    long ld;
    int rows, cols;
    double alpha;
    int accumulate;
    __device__ __forceinline__ bool accumulates() const { return accumulate != 0; }
    __device__ __forceinline__ double2 load(int r, int c) const {
        return (r < rows && c < cols) ? p[(long)r * ld + c] : cmk(0, 0);
    }
    __device__ __forceinline__ double2 combine(double2 old, double2 v) const { return cadd(old, cscale(v, alpha)); }
    __device__ __forceinline__ void store(int r, int c, double2 x) const {
        if (r < rows && c < cols) p[(long)r * ld + c] = x;
    }
};

// Standalone product: grid (ceil(N / BN), ceil(M / BM)), 128 threads, zg::Smem<BM,BN>::total
// complex of dynamic shared memory.
template <int BM, int BN, int NT, class LA, class LB, class PUT>
__global__ void __launch_bounds__(128) k_zgemm(LA la, LB lb, PUT put, int K) {
    extern __shared__ double2 zsm[];
    zgemm_tile<BM, BN, LA, LB, PUT, NT>(la, lb, put, blockIdx.y * BM, blockIdx.x * BN, K, zsm, threadIdx.x, 0);
}
