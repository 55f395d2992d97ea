// libnessi_gpu.so: batches of Kadanoff-Baym problems advanced on one B200.
// Host side of the C ABI declared in include/nessi_gpu.h.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/nessi_gpu.h"
#include "kernels_dyson.cuh"
#include "kernels_tv_stream.cuh"
#include "kernels_start.cuh"
#include "kernels_mat.cuh"
#include "kernels_conv.cuh"
#include "kernels_omp.cuh"
#include "kernels_lattice.cuh"



namespace {

thread_local std::string g_err;
// NVTX range for the time a call spends on the host (launches included); no-op unless a
// profiler is attached
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

int g_device = 0;
std::atomic<int> g_live_batches{0};  // created and not yet destroyed
std::vector<int> g_tables_ready;  // devices whose c_tab was filled
std::mutex g_setup_mutex;         // guards the per-device set-up state (tables, scratch address)

void set_err(const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            set_err("CUDA error %s (%s) at %s:%d", cudaGetErrorName(e_), cudaGetErrorString(e_), \
                    __FILE__, __LINE__);                                                        \
            return e_ == cudaErrorMemoryAllocation ? NESSI_ERR_OOM : NESSI_ERR_CUDA;            \
        }                                                                                       \
    } while (0)

#define CKR(x)                      \
    do {                            \
        int r_ = (x);               \
        if (r_ != NESSI_OK) return r_; \
    } while (0)

inline long tri_h(long t) { return t * (t + 1) / 2; }

// Integration tables into c_tab of device `dev` (current), once per device.  The upload is waited
// for, so that a kernel on any stream of the caller sees the tables.
int ensure_tables(int dev) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (std::find(g_tables_ready.begin(), g_tables_ready.end(), dev) != g_tables_ready.end()) return NESSI_OK;
    IntegTables t;
    std::memcpy(t.greg, cntr_tab_gregory, sizeof t.greg);
    std::memcpy(t.omega, cntr_tab_omega, sizeof t.omega);
    std::memcpy(t.poly_int, cntr_tab_poly_int, sizeof t.poly_int);
    std::memcpy(t.poly_diff, cntr_tab_poly_diff, sizeof t.poly_diff);
    std::memcpy(t.poly_interp, cntr_tab_poly_interp, sizeof t.poly_interp);
    std::memcpy(t.bd, cntr_tab_bd, sizeof t.bd);
    std::memcpy(t.rcorr, cntr_tab_rcorr, sizeof t.rcorr);
    CK(cudaMemcpyToSymbol(c_tab, &t, sizeof t));
    CK(cudaDeviceSynchronize());
    g_tables_ready.push_back(dev);
    return NESSI_OK;
}

// The Matsubara solvers keep 2 ntau twiddle factors in dynamic shared memory next to the
// kernel's static shared memory; check that against the device's opt-in limit per block.
int check_twiddle_smem(const void *kernel, int ntau, const char *name) {
    int dev = 0, optin = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, kernel));
    const size_t need = 2 * (size_t)ntau * 16 + fa.sharedSizeBytes;
    if (need > (size_t)optin) {
        set_err("%s: ntau = %d needs %zu bytes of shared memory per block (2 ntau twiddles), above the device "
                "limit of %d", name, ntau, need, optin);
        return NESSI_ERR_ARG;
    }
    return NESSI_OK;
}

struct Prob {
    nessi_problem_desc d;
    int group = -1;
    double2 *gret = nullptr, *gles = nullptr, *gtv = nullptr, *gmat = nullptr;
    double2 *H = nullptr, *minv_ret = nullptr, *minv_les = nullptr;
    float2 *gtv32 = nullptr;
    double2 *qret = nullptr, *qles = nullptr, *qtv = nullptr, *qmat = nullptr;  // VIE2 source term
};

struct Group {
    int user_id = 0;
    int s = 1, ntau = 0, sig = -1, k = 5, ntmax = 0;
    double h = 0, beta = 0;
    double2 *sret = nullptr, *sles = nullptr, *stv = nullptr, *smat = nullptr;
    double2 *Ldense = nullptr, *Tdense = nullptr, *tvcoef = nullptr;
    double2 *badv = nullptr, *btv = nullptr, *gles = nullptr;
    double2 *Kmat = nullptr, *Gmat_all = nullptr, *Cmat = nullptr;
    int ldc = 0;
    int dense_valid = -1, ret_valid = -1, les_valid = -1;
    bool gmat_valid = false;
    MatScratch *d_mat = nullptr;  // per-member scratch of dyson_mat (allocated on first use)
    std::vector<MatScratch> h_mat;   // host copy of the same pointers
    LocDev loc{nullptr, nullptr, nullptr, nullptr};  // G_loc of the group (allocated on first use)
    double2 *gloc_part = nullptr;    // partial sums of G_loc over chunks of problems
    long gloc_ld = 0;
    bool vie = false;                // VIE2 group: s* hold F, fcc* hold Fcc (nessi_gpu_set_F)
    int pp_ret = 0, pp_les = 0;      // Volterra kernel chosen by the autotuner (0: not yet)
    double2 *fccret = nullptr, *fccles = nullptr;
    double2 *fccmat = nullptr;       // Fcc^mat of a VIE2 group (nessi_gpu_set_Fcc_mat; steepest descent)
    double2 *U = nullptr;            // diagonal interaction U(t), (ntmax+2) x s, t = -1 first
    double2 *accr = nullptr, *accl = nullptr, *panel = nullptr;  // cluster Volterra path
    std::vector<int> members;        // problem indices, nt descending
    std::vector<ProbDev> h_probs;    // same order; col = position
    ProbDev *d_probs = nullptr;
};

}  // namespace

// Per-kernel timing with CUDA events on the batch stream (enabled by nessi_gpu_set_profiling).
struct KProf {
    std::vector<cudaEvent_t> ev;
    int used = 0;
    long launches = 0;
    double bytes = 0;  // algorithmic bytes of the recorded launches
};

struct nessi_batch {
    int device = 0;
    bool prof = false;
    KProf kp[NESSI_KERNEL_COUNT];
    int precision = NESSI_PREC_FP64;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;       // runs the retarded component concurrently with tv
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool own_stream = true;
    cudaGraphExec_t graph = nullptr;                     // recorded time steps (nessi_gpu_graph_record)
    std::vector<Prob> probs;
    std::vector<Group> groups;
    std::vector<void *> allocs;
    long long bytes = 0;
    // Volterra kernels for size1 <= 2: 0 (default) = chosen per group by the autotuner in
    // volterra_step; -1 = the one-problem-per-CTA kernels k_ret / k_les, which overlap the next
    // block's sums with the current block's solve; 1, 2, 4, 8 = problems per CTA of the tensor-core
    // kernels k_ret_mp / k_les_mp, which read each shared Sigma tile once for all of them.
    int volterra_pp = 0;
    double2 *scratch = nullptr;  // G^tv in libcntr layout during layout conversion (size1 > 1)
    long scratch_n = 0;
    // kernel of the tv row: 1 (default) = k_tv (register loads, every size1), 0 = k_tv_stream
    // (history through shared memory by bulk copies, size1 <= 4; NESSI_TV_KERNEL=stream)
    int tv_kernel = 1;
    int nsm = 0;                        // SMs of the device
    int *d_err = nullptr;               // set by a device wait that gave up (NESSI_ERR_TIMEOUT)
    unsigned *d_gbar = nullptr;         // grid barrier of k_volterra_grid: count, generation, abort
    long long wait_ns = 2000000000LL;   // bound of every mbarrier wait in the batch's kernels

    void prof_mark(int id, cudaStream_t st = nullptr) {
        if (!prof) return;
        KProf &k = kp[id];
        if (k.used == (int)k.ev.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            k.ev.push_back(e);
        }
        cudaEventRecord(k.ev[k.used++], st ? st : stream);
    }
    void prof_end(int id, double bytes, cudaStream_t st = nullptr) {
        if (!prof) return;
        prof_mark(id, st);
        kp[id].launches++;
        kp[id].bytes += bytes;
    }

    int alloc(double2 **p, long long n_cplx) {
        if (n_cplx <= 0) { *p = nullptr; return NESSI_OK; }
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, (size_t)n_cplx * sizeof(double2));
        if (e != cudaSuccess) {
            set_err("cudaMalloc of %lld bytes failed: %s", n_cplx * 16LL, cudaGetErrorString(e));
            return NESSI_ERR_OOM;
        }
        e = cudaMemsetAsync(q, 0, (size_t)n_cplx * sizeof(double2), stream);
        if (e != cudaSuccess) { set_err("cudaMemset failed"); return NESSI_ERR_CUDA; }
        allocs.push_back(q);
        bytes += n_cplx * 16LL;
        *p = (double2 *)q;
        return NESSI_OK;
    }
};

namespace {

GroupDev group_dev(const Group &g) {
    GroupDev d;
    d.sret = g.sret; d.sles = g.sles; d.stv = g.stv; d.smat = g.smat;
    d.rret = g.vie ? g.fccret : g.sret;
    d.lcc = g.vie ? g.fccles : g.sles;
    d.Ldense = g.Ldense; d.Tdense = g.Tdense; d.tvcoef = g.tvcoef;
    d.badv = g.badv; d.btv = g.btv; d.gles = g.gles;
    d.Kmat = g.Kmat; d.Gmat_all = g.Gmat_all; d.Cmat = g.Cmat;
    d.fccmat = g.fccmat;
    d.ntmax = g.ntmax; d.ntau = g.ntau; d.s = g.s; d.sig = g.sig; d.k = g.k;
    d.ldc = g.ldc; d.h = g.h; d.beta = g.beta;
    return d;
}

int check_batch(nessi_batch *b) {
    if (!b) { set_err("null batch"); return NESSI_ERR_ARG; }
    CK(cudaSetDevice(b->device));
    return NESSI_OK;
}

int check_prob(nessi_batch *b, int p) {
    CKR(check_batch(b));
    if (p < 0 || p >= (int)b->probs.size()) { set_err("problem index %d out of range", p); return NESSI_ERR_ARG; }
    return NESSI_OK;
}

int find_group(nessi_batch *b, int user_id) {
    for (size_t i = 0; i < b->groups.size(); i++)
        if (b->groups[i].user_id == user_id) return (int)i;
    return -1;
}

// ---- per-size kernel launch table ----------------------------------------------------
template <int S> size_t ret_smem(int k) {
    size_t start = (size_t)(k * k * S * S + k * S * S + (k * S) * (k * S) + k * S * S) * 16 + 16;
    size_t phase = (size_t)VolLayout<S>::total * 16;
    return std::max(start, phase);
}
template <int S> size_t les_smem(int k) {
    const int K1 = k + 1;  // the VIE2 start block has k+1 unknowns
    size_t start = (size_t)((K1 * S) * (K1 * S) + K1 * S * S) * 16 + 16;
    size_t phase = (size_t)VolLayout<S>::total * 16;
    return std::max(start, phase);
}

// C (M x N) = A (M x K) B (K x N) on the repo's DMMA GEMM (kernels_gemm.cuh): 64 x 64 tiles when
// they fill the GPU twice over, else 64 x 32 tiles (warp tiles of 32 x 16); 128 x 32 tiles when
// the problem columns are few.
template <int BM, int BN, int NT, class LA, class LB, class ST>
int zgemm_launch_tiles(const LA &la, const LB &lb, const ST &st, int M, int N, int K, cudaStream_t s) {
    const dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)((M + BM - 1) / BM));
    const size_t sm = (size_t)zg::Smem<BM, BN>::total * sizeof(double2);
    CK(cudaFuncSetAttribute(k_zgemm<BM, BN, NT, LA, LB, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_zgemm<BM, BN, NT><<<grid, 128, sm, s>>>(la, lb, st, K);
    CK(cudaGetLastError());
    return NESSI_OK;
}
template <class LA, class LB, class ST>
int zgemm_launch(const LA &la, const LB &lb, const ST &st, int M, int N, int K, cudaStream_t s) {
    if (M <= 0 || N <= 0) return NESSI_OK;
    if (N <= 32) return zgemm_launch_tiles<128, 32, 4>(la, lb, st, M, N, K, s);
    const long tiles64 = (long)((M + 63) / 64) * ((N + 63) / 64);
    if (tiles64 >= 2 * 148) return zgemm_launch_tiles<64, 64, 4>(la, lb, st, M, N, K, s);
    return zgemm_launch_tiles<64, 32, 2>(la, lb, st, M, N, K, s);
}

// Volterra choice code of the group-wide cluster path (k_ret_start / k_les_start + k_volterra_cl)
#define NESSI_VOLTERRA_CLUSTER 100
#define NESSI_VOLTERRA_GRID 101  // the blocked recursion by one cooperative launch over all SMs
#define NESSI_CL 8  // CTAs per cluster (portable cluster size)

template <int S> size_t ret_start_smem(int k) {
    return (size_t)(k * k * S * S + k * S * S + (k * S) * (k * S) + k * S * S) * 16 + 16;
}
template <int S> size_t les_start_smem(int k) {
    const int K1 = k + 1;
    return (size_t)((K1 * S) * (K1 * S) + K1 * S * S) * 16 + 16;
}

// Clusters of k_volterra_cl that can be resident at once (8 CTAs of one SM each must fit in a
// GPC), asked once per instantiation; the recursion uses at most that many, so that no cluster
// waits for another to finish.
template <int S, bool VIE, bool RET, int BN> int max_active_clusters() {
    static int cached = -1;
    if (cached > 0) return cached;
    const size_t sm = (size_t)std::max(ClSmem<S>::diag, ClGemm<BN>::smem) * sizeof(double2);
    auto kern = k_volterra_cl<S, VIE, RET, BN>;
    int num = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) == cudaSuccess) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(NESSI_CL * 32));
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = sm;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = NESSI_CL;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        if (cudaOccupancyMaxActiveClusters(&num, kern, &cfg) != cudaSuccess) {
            cudaGetLastError();  // a failed query leaves no error behind; the launch reports its own
            num = 0;
        }
    } else {
        cudaGetLastError();
    }
    cached = num > 0 ? num : 16;
    return cached;
}

template <int S, bool VIE, bool RET, int BN>
int cluster_kernel_launch(const GroupDev &gd, const Group &g, int n, int nact, int PT, int ncl, double2 *acc,
                          double2 *panel, cudaStream_t st) {
    const size_t sm = (size_t)std::max(ClSmem<S>::diag, ClGemm<BN>::smem) * sizeof(double2);
    auto kern = k_volterra_cl<S, VIE, RET, BN>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(NESSI_CL * ncl));
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = NESSI_CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kern, gd, (const ProbDev *)g.d_probs, n, nact, PT, acc, panel));
    return NESSI_OK;
}

// Group-wide recursion: the start block of every problem (one CTA each), then the blocked
// recursion by clusters of NESSI_CL CTAs, each owning PT problems (at most NESSI_CL x
// ClCfg::DWMAX problems, one chain warp each).
template <int S, bool VIE>
int cluster_launch(const GroupDev &gd, const Group &g, int n, int nact, bool ret, cudaStream_t st) {
    if (ret) {
        const size_t sm = ret_start_smem<S>(gd.k);
        CK(cudaFuncSetAttribute(k_ret_start<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_ret_start<S, VIE><<<nact, 256, sm, st>>>(gd, g.d_probs, n);
    } else {
        const size_t sm = les_start_smem<S>(gd.k);
        CK(cudaFuncSetAttribute(k_les_start<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_les_start<S, VIE><<<nact, 256, sm, st>>>(gd, g.d_probs, n);
    }
    CK(cudaGetLastError());
    if (n - gd.k <= 0) return NESSI_OK;  // no unknowns below / above the start block
    // as many clusters as fit at once (about 16 on 148 SMs), each with PT problems
    int nfit = ret ? max_active_clusters<S, VIE, true, 32>() : max_active_clusters<S, VIE, false, 32>();
    if constexpr (S <= 2)
        nfit = std::min(nfit, ret ? max_active_clusters<S, VIE, true, 64>() : max_active_clusters<S, VIE, false, 64>());
    int PT = (nact + nfit - 1) / nfit;
    PT = std::max(1, std::min(PT, NESSI_CL * ClCfg<S>::DWMAX));
    const int ncl = (nact + PT - 1) / PT;
    double2 *acc = ret ? g.accr : g.accl;
    if constexpr (S <= 2) {
        if (PT * S > 32) {
            if (ret) return cluster_kernel_launch<S, VIE, true, 64>(gd, g, n, nact, PT, ncl, acc, g.panel, st);
            return cluster_kernel_launch<S, VIE, false, 64>(gd, g, n, nact, PT, ncl, acc, g.panel, st);
        }
    }
    if (ret) return cluster_kernel_launch<S, VIE, true, 32>(gd, g, n, nact, PT, ncl, acc, g.panel, st);
    return cluster_kernel_launch<S, VIE, false, 32>(gd, g, n, nact, PT, ncl, acc, g.panel, st);
}

template <int S, bool VIE, bool RET, int BN>
int grid_kernel_launch(nessi_batch *b, const GroupDev &gd, const Group &g, int n, int p0, int np, double2 *acc,
                       cudaStream_t st) {
    const size_t sm = (size_t)std::max(ClSmem<S>::diag, ClGemm<BN>::smem) * sizeof(double2);
    auto kern = k_volterra_grid<S, VIE, RET, BN>;
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, sm));
    if (per < 1) { set_err("k_volterra_grid: no CTA fits on an SM"); return NESSI_ERR_CUDA; }
    // barrier words: arrival counter, generation, abort flag (cleared before every launch)
    CK(cudaMemsetAsync(b->d_gbar, 0, 4 * sizeof(unsigned), st));
    GridSync gs{b->d_gbar, b->d_gbar + 1, (int *)(b->d_gbar + 2), b->d_err, b->wait_ns};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)b->nsm);  // one CTA per SM, all resident (cooperative launch)
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = sm;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, kern, gd, (const ProbDev *)g.d_probs, n, p0, np, acc, g.panel, gs));
    return NESSI_OK;
}

// Group-wide recursion by the whole GPU: the start block of every problem (one CTA each), then
// the blocked recursion with every block's trailing GEMM over all SMs, in chunks of at most
// nsm x ClCfg::DWMAX problems (one chain warp each).
template <int S, bool VIE>
int grid_launch(nessi_batch *b, const GroupDev &gd, const Group &g, int n, int nact, bool ret, cudaStream_t st) {
    if (ret) {
        const size_t sm = ret_start_smem<S>(gd.k);
        CK(cudaFuncSetAttribute(k_ret_start<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_ret_start<S, VIE><<<nact, 256, sm, st>>>(gd, g.d_probs, n);
    } else {
        const size_t sm = les_start_smem<S>(gd.k);
        CK(cudaFuncSetAttribute(k_les_start<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_les_start<S, VIE><<<nact, 256, sm, st>>>(gd, g.d_probs, n);
    }
    CK(cudaGetLastError());
    if (n - gd.k <= 0) return NESSI_OK;
    double2 *acc = ret ? g.accr : g.accl;
    const int chunk = b->nsm * ClCfg<S>::DWMAX;
    for (int p0 = 0; p0 < nact; p0 += chunk) {
        const int np = std::min(chunk, nact - p0);
        if (np * S > 32) {
            if (ret) CKR((grid_kernel_launch<S, VIE, true, 64>(b, gd, g, n, p0, np, acc, st)));
            else CKR((grid_kernel_launch<S, VIE, false, 64>(b, gd, g, n, p0, np, acc, st)));
        } else {
            if (ret) CKR((grid_kernel_launch<S, VIE, true, 32>(b, gd, g, n, p0, np, acc, st)));
            else CKR((grid_kernel_launch<S, VIE, false, 32>(b, gd, g, n, p0, np, acc, st)));
        }
    }
    return NESSI_OK;
}

// One Volterra recursion (ret or les) of a step: the one-problem kernels (pp = -1), the
// multi-problem tensor-core kernels with pp problems per CTA (size1 <= 2), or the blocked
// recursion by clusters (pp = NESSI_VOLTERRA_CLUSTER) or by the whole GPU (NESSI_VOLTERRA_GRID).
template <int S, bool VIE> int volterra_launch(nessi_batch *b, const GroupDev &gd, const Group &g, int n, int nact,
                                               bool ret, int pp, cudaStream_t st) {
    if (pp == NESSI_VOLTERRA_CLUSTER) return cluster_launch<S, VIE>(gd, g, n, nact, ret, st);
    if (pp == NESSI_VOLTERRA_GRID) return grid_launch<S, VIE>(b, gd, g, n, nact, ret, st);
    if constexpr (S <= 2) {
        if (pp > 0) {
            const size_t sm = (size_t)MpCfg<S>::total * sizeof(double2);
            const unsigned grid = (unsigned)((nact + pp - 1) / pp);
            if (ret) {
                CK(cudaFuncSetAttribute(k_ret_mp<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_ret_mp<S, VIE><<<grid, MP_NW * 32, sm, st>>>(gd, g.d_probs, n, nact, pp);
            } else {
                CK(cudaFuncSetAttribute(k_les_mp<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_les_mp<S, VIE><<<grid, MP_NW * 32, sm, st>>>(gd, g.d_probs, n, nact, pp);
            }
            CK(cudaGetLastError());
            return NESSI_OK;
        }
    }
    const size_t sm = ret ? ret_smem<S>(gd.k) : les_smem<S>(gd.k);
    if (ret) {
        CK(cudaFuncSetAttribute(k_ret<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_ret<S, VIE><<<nact, 256, sm, st>>>(gd, g.d_probs, n);
    } else {
        CK(cudaFuncSetAttribute(k_les<S, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_les<S, VIE><<<nact, 256, sm, st>>>(gd, g.d_probs, n);
    }
    CK(cudaGetLastError());
    return NESSI_OK;
}

// Autotuner of the Volterra kernels.  With volterra_pp = 0 (default), the first eager step of a
// group with n >= the tuning step launches every candidate (one-problem kernels, for size1 <= 2
// the multi-problem kernels with 2, 4, 8 problems per CTA, and the group-wide cluster recursion)
// on the step itself -- each launch recomputes the same row / column from the same inputs, so the
// last one leaves the step's result -- times them with CUDA events and keeps the fastest for the
// group.  The tuning step is 3/4 of the group's longest history (at least min(128, ntmax)): the
// cost of a step grows as n^2, so the late steps carry most of a propagation and the kernels'
// ranking there is the one that counts.  Until then, and while a graph is being recorded, the
// one-problem kernels run.
template <int S, bool VIE> int volterra_step(nessi_batch *b, Group &g, const GroupDev &gd, int n, int nact, bool ret,
                                             cudaStream_t st) {
    int &choice = ret ? g.pp_ret : g.pp_les;
    if (b->volterra_pp != 0) return volterra_launch<S, VIE>(b, gd, g, n, nact, ret, b->volterra_pp, st);
    if (choice != 0) return volterra_launch<S, VIE>(b, gd, g, n, nact, ret, choice, st);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(st, &cap));
    const int tune_n = std::max(std::min(128, g.ntmax), (3 * g.ntmax) / 4);
    if (cap != cudaStreamCaptureStatusNone || n < tune_n)
        return volterra_launch<S, VIE>(b, gd, g, n, nact, ret, -1, st);
    // candidates: one problem per CTA, the per-CTA tensor-core kernels (size1 <= 2), the cluster
    // path; for size1 >= 3 also the whole-GPU path
    const int cand_small[5] = {-1, 2, 4, 8, NESSI_VOLTERRA_CLUSTER};
    const int cand_big[3] = {-1, NESSI_VOLTERRA_CLUSTER, NESSI_VOLTERRA_GRID};
    const int *cand = S <= 2 ? cand_small : cand_big;
    const int ncand = S <= 2 ? 5 : 3;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    float best = 1e30f;
    int bestc = -1;
    for (int pass = 0; pass < 2; pass++)  // the first pass warms up every variant
        for (int ic = 0; ic < ncand; ic++) {
            const int c = cand[ic];
            CK(cudaEventRecord(e0, st));
            CKR((volterra_launch<S, VIE>(b, gd, g, n, nact, ret, c, st)));
            CK(cudaEventRecord(e1, st));
            CK(cudaEventSynchronize(e1));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, e0, e1));
            if (pass == 1 && ms < best) { best = ms; bestc = c; }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    choice = bestc;
    return volterra_launch<S, VIE>(b, gd, g, n, nact, ret, choice, st);  // the kept variant writes last
}

// Decomposition of k_tv_stream: tau chunk width tw <= TWMAX chosen to balance the items
// (problem, chunk) over the CTAs (one per SM): the makespan in rounds of items times the chunk's
// cost (tw plus a fixed cost per segment) is minimised.  Stages hold whole history rows.
TvsPlan tv_stream_plan(int S, int M, int nact, int nsm, int twmax) {
    TvsPlan pl{};
    double best = 1e300;
    const int nch0 = (M + twmax - 1) / twmax;
    for (int nch = nch0; nch < nch0 + 16; nch++) {
        const int tw = (M + nch - 1) / nch, nchr = (M + tw - 1) / tw;
        if (nch > 1 && tw < 32) break;  // segments of at least 512 bytes
        const long items = (long)nact * nchr, grid = std::min<long>(items, nsm);
        const double cost = (double)((items + grid - 1) / grid) * (tw + 16);
        if (cost < best - 1e-9) {
            best = cost;
            pl.tw = tw;
            pl.nch = nchr;
            pl.items = (int)items;
        }
    }
    const int s2 = S * S;
    pl.slot64 = pl.tw * 16;
    pl.slot32 = ((pl.tw + 2) * 8 + 15) & ~15;
    pl.r64 = std::min(64, std::max(1, tvs::SEG_TARGET / (s2 * pl.slot64)));
    pl.r32 = std::min(64, std::max(1, tvs::SEG_TARGET / (s2 * pl.slot32)));
    for (;;) {  // the ring within 216 KB of shared memory
        pl.coef = std::max(pl.r64, pl.r32) * s2 * 16;
        pl.stb = pl.coef + std::max(pl.r64 * s2 * pl.slot64, pl.r32 * s2 * pl.slot32);
        if (tvs::STAGES * pl.stb <= 216 * 1024 || (pl.r64 == 1 && pl.r32 == 1)) break;
        if (pl.r32 * pl.slot32 >= pl.r64 * pl.slot64 && pl.r32 > 1) pl.r32--;
        else if (pl.r64 > 1) pl.r64--;
        else pl.r32--;
    }
    return pl;
}

template <int S, bool MIXED, bool VIE>
int tv_stream_launch(nessi_batch *b, const GroupDev &gd, const Group &g, int n, int nact, cudaStream_t st) {
    TvsPlan pl = tv_stream_plan(S, g.ntau + 1, nact, b->nsm, TvsCfg<S>::TWMAX);
    pl.wait_ns = b->wait_ns;
    pl.err = b->d_err;
    const size_t sm = (size_t)tvs::STAGES * pl.stb;
    if (sm > 220 * 1024) { set_err("k_tv_stream: %zu bytes of shared memory", sm); return NESSI_ERR_ARG; }
    CK(cudaFuncSetAttribute(k_tv_stream<S, MIXED, VIE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int grid = std::min(pl.items, b->nsm);
    k_tv_stream<S, MIXED, VIE><<<grid, tvs::NTH, sm, st>>>(gd, g.d_probs, n, pl);
    CK(cudaGetLastError());
    return NESSI_OK;
}

template <int S, bool VIE> int step_group(nessi_batch *b, Group &g, int n, int nact) {
    const GroupDev gd = group_dev(g);
    cudaStream_t st = b->stream;
    const int k = g.k;
    // step-matrix inverses
    int les_lo = std::min(n, std::max(k + 1, g.les_valid + 1));
    int r0 = g.ret_valid + 1, r1 = n - k - 1;
    b->prof_mark(NESSI_KERNEL_PREP);
    k_prep_problem<S, VIE><<<nact, 64, 0, st>>>(gd, g.d_probs, n, les_lo, r0, r1);
    CK(cudaGetLastError());
    g.les_valid = n - 1;
    if (r1 >= r0) g.ret_valid = r1;
    int d_lo = std::min(n, g.dense_valid + 1);
    {
        long work = (long)(n + 1) * S * S * (n - d_lo + 1) + (long)n * S * S;
        int blocks = (int)std::min<long>(std::max<long>(1, (work + 255) / 256), 1184);
        k_prep_group<S, VIE><<<blocks, 256, 0, st>>>(gd, n, d_lo);
        CK(cudaGetLastError());
        b->prof_end(NESSI_KERNEL_PREP, 0.0);
        g.dense_valid = n - 1;
    }
    // VIE2 moves the convolution to the right-hand side: gles = -(tv*vt + les*adv)
    const double alpha = VIE ? -1.0 : 1.0;
    // Matsubara part of the tv row: Cmat = K_n Gmat_all (one GEMM for the group)
    {
        const long M = g.ntau + 1;
        if (!g.gmat_valid) {
            dim3 grid((unsigned)((M * S * S + 255) / 256), (unsigned)g.members.size());
            k_gmat_stack<S><<<grid, 256, 0, st>>>(gd, g.d_probs);
            CK(cudaGetLastError());
            g.gmat_valid = true;
        }
        b->prof_mark(NESSI_KERNEL_MATOP);
        long work = M * M * S * S;
        k_mat_operator<S><<<(unsigned)std::min<long>((work + 255) / 256, 4736), 256, 0, st>>>(gd, n, VIE ? -1.0 : 1.0);
        CK(cudaGetLastError());
        b->prof_end(NESSI_KERNEL_MATOP, 16.0 * (double)work + 16.0 * M * S * S);
        b->prof_mark(NESSI_KERNEL_GEMM);
        const int MS = (int)(M * S);
        CKR(zgemm_launch(LdRowK{g.Kmat, MS, MS, MS}, LdRowN{g.Gmat_all, g.ldc, MS, nact * S},
                         StRow{g.Cmat, g.ldc, MS, nact * S, 1.0, 0}, MS, nact * S, MS, st));
        b->prof_end(NESSI_KERNEL_GEMM, 8.0 * (double)nact * S * (M * S) * (M * S));
    }
    const int m = nact * S, nn = (n + 1) * S;
    const long ldL = (long)(g.ntmax + 1) * S, ldT = (long)(g.ntau + 1) * S;
    // side stream: retarded row, then les*adv = Ldense * badv (needs only G^R(n, .))
    CK(cudaEventRecord(b->ev_fork, st));
    CK(cudaStreamWaitEvent(b->side, b->ev_fork, 0));
    {
        b->prof_mark(NESSI_KERNEL_RET, b->side);
        CKR((volterra_step<S, VIE>(b, g, gd, n, nact, true, b->side)));
        // flops: every pair m > j of the row, an s x s complex product (8 s^3) per problem
        b->prof_end(NESSI_KERNEL_RET, 8.0 * S * S * S * (double)nact * tri_h(n), b->side);
        b->prof_mark(NESSI_KERNEL_LES_OPERANDS, b->side);
        dim3 grid((unsigned)((n + 1 + LoCfg<S>::LOR - 1) / LoCfg<S>::LOR), (unsigned)((nact + LOT - 1) / LOT));
        k_les_operands_t<S><<<grid, 256, 0, b->side>>>(gd, g.d_probs, n, 1, nact);
        CK(cudaGetLastError());
        b->prof_end(NESSI_KERNEL_LES_OPERANDS, 32.0 * S * S * (double)nact * (n + 1), b->side);
        b->prof_mark(NESSI_KERNEL_GEMM, b->side);
        CKR(zgemm_launch(LdRowK{g.Ldense, ldL, nn, nn}, LdRowN{g.badv, g.ldc, nn, m},
                         StRow{g.gles, g.ldc, nn, m, alpha, 0}, nn, m, nn, b->side));
        b->prof_end(NESSI_KERNEL_GEMM, 8.0 * (double)m * nn * ((n + 1) * S), b->side);
    }
    CK(cudaEventRecord(b->ev_join, b->side));
    // main stream: tv row, then the tv*vt operand
    {
        dim3 grid((g.ntau + 1 + 31) / 32, nact);
        b->prof_mark(NESSI_KERNEL_TV);
        const bool mixed = b->precision == NESSI_PREC_MIXED;
        bool streamed = false;
        if constexpr (S <= 4) {
            if (b->tv_kernel == 0) {
                if (mixed) CKR((tv_stream_launch<S, true, VIE>(b, gd, g, n, nact, st)));
                else CKR((tv_stream_launch<S, false, VIE>(b, gd, g, n, nact, st)));
                streamed = true;
            }
        }
        if (!streamed) {
            if (mixed) k_tv<S, true, VIE><<<grid, 256, 0, st>>>(gd, g.d_probs, n);
            else k_tv<S, false, VIE><<<grid, 256, 0, st>>>(gd, g.d_probs, n);
            CK(cudaGetLastError());
        }
        // per problem: G^tv history rows 0..n-1 read (FP32 below the k+1 BDF rows when mixed),
        // row n written, Cmat column read; shared: the n coefficient blocks
        const double M = g.ntau + 1;
        const double n32 = mixed ? std::max(0, n - k - 1) : 0, n64 = n - n32;
        b->prof_end(NESSI_KERNEL_TV, S * S * ((double)nact * (8.0 * n32 * M + 16.0 * n64 * M + 32.0 * M +
                                                                 (mixed ? 8.0 * M : 0.0)) + 16.0 * n));
        b->prof_mark(NESSI_KERNEL_LES_OPERANDS);
        dim3 grid2((unsigned)((g.ntau + 1 + LoCfg<S>::LOR - 1) / LoCfg<S>::LOR), (unsigned)((nact + LOT - 1) / LOT));
        k_les_operands_t<S><<<grid2, 256, 0, st>>>(gd, g.d_probs, n, 2, nact);
        CK(cudaGetLastError());
        b->prof_end(NESSI_KERNEL_LES_OPERANDS, 32.0 * S * S * (double)nact * (g.ntau + 1));
    }
    CK(cudaStreamWaitEvent(st, b->ev_join, 0));
    // tv*vt: gles += Sigma^tv * btv
    {
        b->prof_mark(NESSI_KERNEL_GEMM);
        const double2 *T = S == 1 ? g.stv : g.Tdense;
        const int MS = (g.ntau + 1) * S;
        CKR(zgemm_launch(LdRowK{T, ldT, nn, MS}, LdRowN{g.btv, g.ldc, MS, m}, StRow{g.gles, g.ldc, nn, m, alpha, 1},
                         nn, m, MS, st));
        b->prof_end(NESSI_KERNEL_GEMM, 8.0 * (double)m * nn * ((g.ntau + 1) * S));
    }
    // lesser column
    {
        b->prof_mark(NESSI_KERNEL_LES);
        CKR((volterra_step<S, VIE>(b, g, gd, n, nact, false, st)));
        b->prof_end(NESSI_KERNEL_LES, 8.0 * S * S * S * (double)nact * tri_h(n));
    }
    return NESSI_OK;
}

template <int S> int start_group(nessi_batch *b, Group &g) {
    const GroupDev gd = group_dev(g);
    const size_t sm = NESSI_START_SMEM * sizeof(double2);
    if (g.vie) {
        CK(cudaFuncSetAttribute(k_vie2_start<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_vie2_start<S><<<(unsigned)g.members.size(), 256, sm, b->stream>>>(gd, g.d_probs);
    } else {
        CK(cudaFuncSetAttribute(k_dyson_start<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_dyson_start<S><<<(unsigned)g.members.size(), 256, sm, b->stream>>>(gd, g.d_probs);
    }
    CK(cudaGetLastError());
    return NESSI_OK;
}

static int ensure_mat_scratch(nessi_batch *b, Group &g) {
    if (g.d_mat) return NESSI_OK;
    const long M = g.ntau + 1, s2 = (long)g.s * g.s;
    std::vector<MatScratch> h(g.members.size());
    for (auto &w : h) {
        int r;
        if ((r = b->alloc(&w.G0, M * s2)) || (r = b->alloc(&w.F, M * s2)) || (r = b->alloc(&w.Q, M * s2)) ||
            (r = b->alloc(&w.dG, M * s2)) || (r = b->alloc(&w.fdft, M * s2)) || (r = b->alloc(&w.qdft, M * s2)) ||
            (r = b->alloc(&w.Z, 2 * g.ntau * s2)))
            return r;
    }
    void *q = nullptr;
    CK(cudaMalloc(&q, h.size() * sizeof(MatScratch)));
    b->allocs.push_back(q);
    g.d_mat = (MatScratch *)q;
    g.h_mat = h;
    CK(cudaMemcpyAsync(g.d_mat, h.data(), h.size() * sizeof(MatScratch), cudaMemcpyHostToDevice, b->stream));
    return NESSI_OK;
}

template <int S> int mat_group(nessi_batch *b, Group &g, int method, int force_herm) {
    const GroupDev gd = group_dev(g);
    CKR(check_twiddle_smem((const void *)k_dyson_mat<S>, g.ntau, "dyson_mat"));
    CKR(ensure_mat_scratch(b, g));
    const size_t sm = 2 * (size_t)g.ntau * sizeof(double2);
    CK(cudaFuncSetAttribute(k_dyson_mat<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_dyson_mat<S><<<(unsigned)g.members.size(), 256, sm, b->stream>>>(gd, g.d_probs, g.d_mat, method, force_herm);
    CK(cudaGetLastError());
    g.gmat_valid = false;
    return NESSI_OK;
}

// vie2_mat of a VIE2 group: Q^mat of every member is copied into its scratch slot G0 first
template <int S> int vie2_mat_group(nessi_batch *b, Group &g, int method) {
    const GroupDev gd = group_dev(g);
    CKR(check_twiddle_smem((const void *)k_vie2_mat<S>, g.ntau, "vie2_mat"));
    CKR(ensure_mat_scratch(b, g));
    const long M = g.ntau + 1, s2 = (long)g.s * g.s;
    for (size_t c = 0; c < g.members.size(); c++) {
        const Prob &q = b->probs[g.members[c]];
        if (!q.qmat) { set_err("vie2_mat: Q of problem %d not set", g.members[c]); return NESSI_ERR_ARG; }
        CK(cudaMemcpyAsync(g.h_mat[c].G0, q.qmat, (size_t)M * s2 * sizeof(double2), cudaMemcpyDeviceToDevice,
                           b->stream));
    }
    const size_t sm = 2 * (size_t)g.ntau * sizeof(double2);
    CK(cudaFuncSetAttribute(k_vie2_mat<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_vie2_mat<S><<<(unsigned)g.members.size(), 256, sm, b->stream>>>(gd, g.d_probs, g.d_mat, method);
    CK(cudaGetLastError());
    g.gmat_valid = false;
    return NESSI_OK;
}

// ---- lattice pieces: predictor, k-average, local second-order self-energy ---------------
int active_members(const nessi_batch *b, const Group &g, int tstp) {
    int nact = 0;
    for (int i : g.members) nact += b->probs[i].d.nt >= tstp ? 1 : 0;
    return nact;
}

template <int S> int extrap_group(nessi_batch *b, Group &g, int n) {
    const long work = ((long)g.ntau + 1 + 2L * (n + 2)) * S * S;
    dim3 grid((unsigned)std::min<long>((work + 255) / 256, 64), (unsigned)g.members.size());
    k_extrapolate<S><<<grid, 256, 0, b->stream>>>(group_dev(g), g.d_probs, n);
    CK(cudaGetLastError());
    return NESSI_OK;
}

template <int S> int gloc_group(nessi_batch *b, Group &g, int tstp) {
    const int nact = active_members(b, g, tstp);
    if (nact == 0) { set_err("gloc: no problem of the group reaches time step %d", tstp); return NESSI_ERR_ARG; }
    const long M = g.ntau + 1, s2 = (long)S * S;
    const long total = tstp >= 0 ? (2L * (tstp + 1) + M) * s2 : M * s2;
    const int nchunk = (nact + GLOC_CHUNK - 1) / GLOC_CHUNK;
    k_gloc<S><<<dim3((unsigned)((total + 31) / 32), (unsigned)nchunk), dim3(32, 8), 0, b->stream>>>(
        group_dev(g), g.d_probs, nact, tstp, g.gloc_part, g.gloc_ld);
    CK(cudaGetLastError());
    k_gloc_final<S><<<(unsigned)std::min<long>((total + 255) / 256, 1184), 256, 0, b->stream>>>(
        group_dev(g), nact, tstp, g.gloc_part, g.gloc_ld, nchunk, g.loc);
    CK(cudaGetLastError());
    return NESSI_OK;
}

void sigma_changed(Group &g, int tstp) {
    if (tstp < 0) return;  // Sigma^mat is read only by dyson_mat, which caches nothing
    g.ret_valid = std::min(g.ret_valid, tstp - 1);
    g.les_valid = std::min(g.les_valid, tstp - 1);
    g.dense_valid = std::min(g.dense_valid, tstp - 1);
}

template <int S> int sigma2b_group(nessi_batch *b, Group &g, int tstp) {
    const long M = g.ntau + 1, s2 = (long)S * S;
    const long work = tstp >= 0 ? ((long)tstp + 1 + M) * s2 : M * s2;
    SigOut o{g.sret, g.sles, g.stv, g.smat};
    k_sigma_2b<S><<<(unsigned)std::min<long>((work + 255) / 256, 1184), 256, 0, b->stream>>>(group_dev(g), g.loc,
                                                                                           g.U, tstp, o);
    CK(cudaGetLastError());
    sigma_changed(g, tstp);
    return NESSI_OK;
}

#define NESSI_SIZE_SWITCH(fn, ...)                 \
    switch (g.s) {                                 \
        case 1: return fn<1>(__VA_ARGS__);         \
        case 2: return fn<2>(__VA_ARGS__);         \
        case 3: return fn<3>(__VA_ARGS__);         \
        case 4: return fn<4>(__VA_ARGS__);         \
        case 5: return fn<5>(__VA_ARGS__);         \
        case 6: return fn<6>(__VA_ARGS__);         \
        case 7: return fn<7>(__VA_ARGS__);         \
        case 8: return fn<8>(__VA_ARGS__);         \
    }                                              \
    set_err("size1 = %d not supported (1..8)", g.s); \
    return NESSI_ERR_ARG;

int start_dispatch(nessi_batch *b, Group &g) { NESSI_SIZE_SWITCH(start_group, b, g) }
int extrap_dispatch(nessi_batch *b, Group &g, int n) { NESSI_SIZE_SWITCH(extrap_group, b, g, n) }
int gloc_dispatch(nessi_batch *b, Group &g, int tstp) { NESSI_SIZE_SWITCH(gloc_group, b, g, tstp) }
int sigma2b_dispatch(nessi_batch *b, Group &g, int tstp) { NESSI_SIZE_SWITCH(sigma2b_group, b, g, tstp) }
int mat_dispatch(nessi_batch *b, Group &g, int method, int force_herm) {
    NESSI_SIZE_SWITCH(mat_group, b, g, method, force_herm)
}
int vie2_mat_dispatch(nessi_batch *b, Group &g, int method) { NESSI_SIZE_SWITCH(vie2_mat_group, b, g, method) }

template <int S> int step_group_any(nessi_batch *b, Group &g, int n, int nact) {
    return g.vie ? step_group<S, true>(b, g, n, nact) : step_group<S, false>(b, g, n, nact);
}

int step_dispatch(nessi_batch *b, Group &g, int n, int nact) {
    switch (g.s) {
        case 1: return step_group_any<1>(b, g, n, nact);
        case 2: return step_group_any<2>(b, g, n, nact);
        case 3: return step_group_any<3>(b, g, n, nact);
        case 4: return step_group_any<4>(b, g, n, nact);
        case 5: return step_group_any<5>(b, g, n, nact);
        case 6: return step_group_any<6>(b, g, n, nact);
        case 7: return step_group_any<7>(b, g, n, nact);
        case 8: return step_group_any<8>(b, g, n, nact);
    }
    set_err("size1 = %d not supported (1..8)", g.s);
    return NESSI_ERR_ARG;
}

}  // namespace

// =====================================================================================
// C ABI
// =====================================================================================
extern "C" {

const char *nessi_gpu_last_error(void) { return g_err.c_str(); }

int nessi_gpu_init(int device) {
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) { set_err("device %d not present (%d devices)", device, n); return NESSI_ERR_ARG; }
    g_device = device;
    CK(cudaSetDevice(device));
    return ensure_tables(device);
}

int nessi_gpu_batch_create(nessi_batch **out, const nessi_problem_desc *desc, int count, int precision) {
    if (!out || !desc || count <= 0) { set_err("batch_create: bad arguments"); return NESSI_ERR_ARG; }
    if (precision != NESSI_PREC_FP64 && precision != NESSI_PREC_MIXED) { set_err("bad precision %d", precision); return NESSI_ERR_ARG; }
    *out = nullptr;
    for (int i = 0; i < count; i++) {
        const nessi_problem_desc &d = desc[i];
        if (d.nt < 0 || d.ntau < d.solve_order || d.size1 < 1 || d.size1 > NESSI_MAXS || (d.sig != 1 && d.sig != -1) ||
            d.solve_order < 1 || d.solve_order > CNTR_KMAX || !(d.h > 0) || !(d.beta > 0)) {
            set_err("problem %d: bad descriptor (nt=%d ntau=%d size1=%d sig=%d k=%d)", i, d.nt, d.ntau, d.size1,
                    d.sig, d.solve_order);
            return NESSI_ERR_ARG;
        }
    }
    CK(cudaSetDevice(g_device));
    CKR(ensure_tables(g_device));
    nessi_batch *b = new nessi_batch();
    g_live_batches++;
    b->device = g_device;
    b->precision = precision;
    if (const char *v = getenv("NESSI_VOLTERRA_PP")) {
        const int pp = atoi(v);
        if (pp == -1 || pp == 0 || pp == 1 || pp == 2 || pp == 4 || pp == 8 || pp == NESSI_VOLTERRA_CLUSTER ||
            pp == NESSI_VOLTERRA_GRID)
            b->volterra_pp = pp;
    }
    if (const char *v = getenv("NESSI_TV_KERNEL")) b->tv_kernel = strcmp(v, "stream") == 0 ? 0 : 1;
    auto fail = [&](int r) { nessi_gpu_batch_destroy(b); return r; };
    if (cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess || b->nsm <= 0) {
        set_err("SM count query failed");
        return fail(NESSI_ERR_CUDA);
    }
    {
        void *q = nullptr;
        if (cudaMalloc(&q, sizeof(int)) != cudaSuccess || cudaMemset(q, 0, sizeof(int)) != cudaSuccess) {
            set_err("cudaMalloc of the error word failed");
            return fail(NESSI_ERR_OOM);
        }
        b->allocs.push_back(q);
        b->d_err = (int *)q;
        q = nullptr;
        if (cudaMalloc(&q, 4 * sizeof(unsigned)) != cudaSuccess || cudaMemset(q, 0, 4 * sizeof(unsigned)) != cudaSuccess) {
            set_err("cudaMalloc of the grid barrier failed");
            return fail(NESSI_ERR_OOM);
        }
        b->allocs.push_back(q);
        b->d_gbar = (unsigned *)q;
    }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_err("stream creation failed");
        return fail(NESSI_ERR_CUDA);
    }
    if (cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        set_err("stream/event creation failed");
        return fail(NESSI_ERR_CUDA);
    }
    b->probs.resize(count);
    // groups
    for (int i = 0; i < count; i++) {
        const nessi_problem_desc &d = desc[i];
        b->probs[i].d = d;
        int gi = find_group(b, d.sigma_group);
        if (gi < 0) {
            Group g;
            g.user_id = d.sigma_group; g.s = d.size1; g.ntau = d.ntau; g.sig = d.sig; g.k = d.solve_order;
            g.h = d.h; g.beta = d.beta; g.ntmax = d.nt;
            b->groups.push_back(g);
            gi = (int)b->groups.size() - 1;
        }
        Group &g = b->groups[gi];
        if (g.s != d.size1 || g.ntau != d.ntau || g.sig != d.sig || g.k != d.solve_order || g.h != d.h || g.beta != d.beta) {
            set_err("problem %d does not match the other problems of sigma_group %d", i, d.sigma_group);
            return fail(NESSI_ERR_ARG);
        }
        g.ntmax = std::max(g.ntmax, d.nt);
        g.members.push_back(i);
        b->probs[i].group = gi;
    }
    // device storage
    for (int i = 0; i < count; i++) {
        Prob &p = b->probs[i];
        const long s2 = (long)p.d.size1 * p.d.size1, nt = p.d.nt, M = p.d.ntau + 1;
        int r;
        if ((r = b->alloc(&p.gret, tri_h(nt + 1) * s2)) || (r = b->alloc(&p.gles, tri_h(nt + 1) * s2)) ||
            (r = b->alloc(&p.gtv, (nt + 1) * M * s2)) || (r = b->alloc(&p.gmat, M * s2)) ||
            (r = b->alloc(&p.H, (nt + 2) * s2)) || (r = b->alloc(&p.minv_ret, (nt + 1) * s2)) ||
            (r = b->alloc(&p.minv_les, (nt + 1) * s2)))
            return fail(r);
        if (precision == NESSI_PREC_MIXED) {
            void *q = nullptr;
            size_t nb_ = (size_t)(nt + 1) * M * s2 * sizeof(float2);
            if (cudaMalloc(&q, nb_) != cudaSuccess) { set_err("cudaMalloc of %zu bytes failed", nb_); return fail(NESSI_ERR_OOM); }
            b->allocs.push_back(q);
            b->bytes += nb_;
            p.gtv32 = (float2 *)q;
        }
    }
    {
        long need = 0;
        for (const Prob &p : b->probs)
            if (p.d.size1 > 1) need = std::max(need, (long)(p.d.nt + 1) * (p.d.ntau + 1) * p.d.size1 * p.d.size1);
        int r;
        if (need > 0 && (r = b->alloc(&b->scratch, need))) return fail(r);
        b->scratch_n = need;
    }
    for (Group &g : b->groups) {
        std::stable_sort(g.members.begin(), g.members.end(),
                         [&](int x, int y) { return b->probs[x].d.nt > b->probs[y].d.nt; });
        const long S = g.s, s2 = S * S, N = g.ntmax + 1, M = g.ntau + 1;
        g.ldc = (int)(g.members.size() * S);
        int r;
        if ((r = b->alloc(&g.sret, tri_h(N) * s2)) || (r = b->alloc(&g.sles, tri_h(N) * s2)) ||
            (r = b->alloc(&g.stv, N * M * s2)) || (r = b->alloc(&g.smat, M * s2)) ||
            (r = b->alloc(&g.Ldense, N * S * N * S)) || (S > 1 && (r = b->alloc(&g.Tdense, N * S * M * S))) ||
            (r = b->alloc(&g.tvcoef, N * s2)) || (r = b->alloc(&g.badv, N * S * g.ldc)) ||
            (r = b->alloc(&g.btv, M * S * g.ldc)) || (r = b->alloc(&g.gles, N * S * g.ldc)) ||
            (r = b->alloc(&g.Kmat, M * S * M * S)) || (r = b->alloc(&g.Gmat_all, M * S * g.ldc)) ||
            (r = b->alloc(&g.Cmat, M * S * g.ldc)) || (r = b->alloc(&g.accr, N * S * g.ldc)) ||
            (r = b->alloc(&g.accl, N * S * g.ldc)) || (r = b->alloc(&g.panel, (32 + NESSI_K1MAX) * S * g.ldc)))
            return fail(r);
        for (size_t c = 0; c < g.members.size(); c++) {
            const Prob &p = b->probs[g.members[c]];
            ProbDev pd;
            pd.gret = p.gret; pd.gles = p.gles; pd.gtv = p.gtv; pd.gmat = p.gmat;
            pd.H = p.H; pd.minv_ret = p.minv_ret; pd.minv_les = p.minv_les; pd.gtv32 = p.gtv32;
            pd.qret = p.qret; pd.qles = p.qles; pd.qtv = p.qtv;
            pd.mu = p.d.mu; pd.nt = p.d.nt; pd.col = (int)c; pd.pad = 0;
            g.h_probs.push_back(pd);
        }
        void *q = nullptr;
        if (cudaMalloc(&q, g.h_probs.size() * sizeof(ProbDev)) != cudaSuccess) { set_err("cudaMalloc failed"); return fail(NESSI_ERR_OOM); }
        b->allocs.push_back(q);
        g.d_probs = (ProbDev *)q;
        if (cudaMemcpyAsync(g.d_probs, g.h_probs.data(), g.h_probs.size() * sizeof(ProbDev), cudaMemcpyHostToDevice,
                            b->stream) != cudaSuccess) {
            set_err("descriptor upload failed");
            return fail(NESSI_ERR_CUDA);
        }
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) { set_err("stream sync failed"); return fail(NESSI_ERR_CUDA); }
    *out = b;
    return NESSI_OK;
}

int nessi_gpu_batch_destroy(nessi_batch *b) {
    if (!b) return NESSI_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (void *q : b->allocs) cudaFree(q);
    for (auto &k : b->kp)
        for (cudaEvent_t e : k.ev) cudaEventDestroy(e);
    if (b->side) { cudaStreamSynchronize(b->side); cudaStreamDestroy(b->side); }
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    g_live_batches--;
    return NESSI_OK;
}

int nessi_gpu_finalize(void) {
    if (g_live_batches.load() != 0) {
        set_err("finalize: %d batches are still alive", g_live_batches.load());
        return NESSI_ERR_ARG;
    }
    for (int dev : g_tables_ready) {
        CK(cudaSetDevice(dev));
        CK(cudaDeviceSynchronize());
    }
    g_tables_ready.clear();  // the next init or batch uploads the integration tables again
    return NESSI_OK;
}

int nessi_gpu_batch_bytes(nessi_batch *b, long long *bytes) {
    CKR(check_batch(b));
    *bytes = b->bytes;
    return NESSI_OK;
}

static int copy_cplx(nessi_batch *b, void *dst, const void *src, long n_cplx, cudaMemcpyKind kind) {
    if (!dst || !src || n_cplx <= 0) return NESSI_OK;
    CK(cudaMemcpyAsync(dst, src, (size_t)n_cplx * 16, kind, b->stream));
    return NESSI_OK;
}

static int refresh32(nessi_batch *b, float2 *dst, const double2 *src, long n) {
    if (!dst || n <= 0) return NESSI_OK;
    k_tv_to32<<<(int)std::min<long>((n + 255) / 256, 4096), 256, 0, b->stream>>>(dst, src, n);
    CK(cudaGetLastError());
    return NESSI_OK;
}

// G^tv rows [t0, t0+rows) between a host buffer in libcntr layout and the device planes
static int tv_transfer(nessi_batch *b, double2 *dev_planes, void *host, long t0, long rows, int M, int s,
                       bool to_device) {
    if (!host || rows <= 0) return NESSI_OK;
    const long s2 = (long)s * s, n = rows * M * s2;
    double2 *dev = dev_planes + t0 * M * s2;
    if (s == 1) {
        return to_device ? copy_cplx(b, dev, host, n, cudaMemcpyHostToDevice)
                         : copy_cplx(b, host, dev, n, cudaMemcpyDeviceToHost);
    }
    if (n > b->scratch_n) { set_err("internal: scratch too small"); return NESSI_ERR_ARG; }
    const int blocks = (int)std::min<long>((n + 255) / 256, 4096);
    if (to_device) {
        CKR(copy_cplx(b, b->scratch, host, n, cudaMemcpyHostToDevice));
        k_tv_relayout<<<blocks, 256, 0, b->stream>>>(dev, b->scratch, rows, M, (int)s2, 1);
        CK(cudaGetLastError());
    } else {
        k_tv_relayout<<<blocks, 256, 0, b->stream>>>(b->scratch, dev, rows, M, (int)s2, 0);
        CK(cudaGetLastError());
        CKR(copy_cplx(b, host, b->scratch, n, cudaMemcpyDeviceToHost));
    }
    return NESSI_OK;
}

int nessi_gpu_set_G(nessi_batch *b, int p, const void *ret, const void *les, const void *tv, const void *mat) {
    CKR(check_prob(b, p));
    Prob &q = b->probs[p];
    const long s2 = (long)q.d.size1 * q.d.size1, nt = q.d.nt, M = q.d.ntau + 1;
    CKR(copy_cplx(b, q.gret, ret, tri_h(nt + 1) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, q.gles, les, tri_h(nt + 1) * s2, cudaMemcpyHostToDevice));
    CKR(tv_transfer(b, q.gtv, (void *)tv, 0, nt + 1, (int)M, q.d.size1, true));
    if (tv) CKR(refresh32(b, q.gtv32, q.gtv, (nt + 1) * M * s2));
    CKR(copy_cplx(b, q.gmat, mat, M * s2, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    if (mat) b->groups[q.group].gmat_valid = false;
    return NESSI_OK;
}

int nessi_gpu_get_G(nessi_batch *b, int p, void *ret, void *les, void *tv, void *mat) {
    CKR(check_prob(b, p));
    Prob &q = b->probs[p];
    const long s2 = (long)q.d.size1 * q.d.size1, nt = q.d.nt, M = q.d.ntau + 1;
    CKR(copy_cplx(b, ret, q.gret, tri_h(nt + 1) * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, les, q.gles, tri_h(nt + 1) * s2, cudaMemcpyDeviceToHost));
    CKR(tv_transfer(b, q.gtv, tv, 0, nt + 1, (int)M, q.d.size1, false));
    CKR(copy_cplx(b, mat, q.gmat, M * s2, cudaMemcpyDeviceToHost));
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

static int slice_copy(nessi_batch *b, double2 *ret, double2 *tv, double2 *les, double2 *mat, int nt, int ntau, int s,
                      int tstp, void *slice, bool to_device, bool tv_planes) {
    const long s2 = (long)s * s, M = ntau + 1;
    if (tstp < -1 || tstp > nt) { set_err("time step %d out of range [-1, %d]", tstp, nt); return NESSI_ERR_ARG; }
    if (!slice) { set_err("null slice"); return NESSI_ERR_ARG; }
    double2 *h = (double2 *)slice;
    cudaMemcpyKind kd = to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    auto cp = [&](double2 *dev, double2 *host, long n) {
        return to_device ? copy_cplx(b, dev, host, n, kd) : copy_cplx(b, host, dev, n, kd);
    };
    if (tstp == -1) {
        CKR(cp(mat, h, M * s2));
    } else {
        const long n1 = tstp + 1;
        CKR(cp(ret + tri_h(tstp) * s2, h, n1 * s2));
        if (tv_planes) CKR(tv_transfer(b, tv, h + n1 * s2, tstp, 1, (int)M, s, to_device));
        else CKR(cp(tv + tstp * M * s2, h + n1 * s2, M * s2));
        CKR(cp(les + tri_h(tstp) * s2, h + (n1 + M) * s2, n1 * s2));
    }
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_get_timestep(nessi_batch *b, int p, int tstp, void *slice) {
    CKR(check_prob(b, p));
    Prob &q = b->probs[p];
    return slice_copy(b, q.gret, q.gtv, q.gles, q.gmat, q.d.nt, q.d.ntau, q.d.size1, tstp, slice, false, true);
}

int nessi_gpu_set_timestep(nessi_batch *b, int p, int tstp, const void *slice) {
    CKR(check_prob(b, p));
    Prob &q = b->probs[p];
    if (tstp == -1) b->groups[q.group].gmat_valid = false;
    CKR(slice_copy(b, q.gret, q.gtv, q.gles, q.gmat, q.d.nt, q.d.ntau, q.d.size1, tstp, (void *)slice, true, true));
    if (tstp >= 0) {
        const long row = (long)(q.d.ntau + 1) * q.d.size1 * q.d.size1;
        CKR(refresh32(b, q.gtv32 ? q.gtv32 + tstp * row : nullptr, q.gtv + tstp * row, row));
        CK(cudaStreamSynchronize(b->stream));
    }
    return NESSI_OK;
}

int nessi_gpu_set_H(nessi_batch *b, int p, const void *H) {
    CKR(check_prob(b, p));
    Prob &q = b->probs[p];
    if (!H) { set_err("null H"); return NESSI_ERR_ARG; }
    CKR(copy_cplx(b, q.H, H, (long)(q.d.nt + 2) * q.d.size1 * q.d.size1, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    Group &g = b->groups[q.group];
    g.ret_valid = -1;
    g.les_valid = -1;
    return NESSI_OK;
}

int nessi_gpu_set_sigma(nessi_batch *b, int group, const void *ret, const void *les, const void *tv, const void *mat) {
    CKR(check_batch(b));
    int gi = find_group(b, group);
    if (gi < 0) { set_err("unknown sigma_group %d", group); return NESSI_ERR_ARG; }
    Group &g = b->groups[gi];
    const long s2 = (long)g.s * g.s, N = g.ntmax + 1, M = g.ntau + 1;
    CKR(copy_cplx(b, g.sret, ret, tri_h(N) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g.sles, les, tri_h(N) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g.stv, tv, N * M * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g.smat, mat, M * s2, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    g.ret_valid = g.les_valid = g.dense_valid = -1;
    return NESSI_OK;
}

int nessi_gpu_set_sigma_timestep(nessi_batch *b, int group, int tstp, const void *slice) {
    CKR(check_batch(b));
    int gi = find_group(b, group);
    if (gi < 0) { set_err("unknown sigma_group %d", group); return NESSI_ERR_ARG; }
    Group &g = b->groups[gi];
    CKR(slice_copy(b, g.sret, g.stv, g.sles, g.smat, g.ntmax, g.ntau, g.s, tstp, (void *)slice, true, false));
    if (tstp >= 0) {
        g.ret_valid = std::min(g.ret_valid, tstp - 1);
        g.les_valid = std::min(g.les_valid, tstp - 1);
        g.dense_valid = std::min(g.dense_valid, tstp - 1);
    }
    return NESSI_OK;
}

static int find_group_checked(nessi_batch *b, int group, Group **out) {
    CKR(check_batch(b));
    int gi = find_group(b, group);
    if (gi < 0) { set_err("unknown sigma_group %d", group); return NESSI_ERR_ARG; }
    *out = &b->groups[gi];
    return NESSI_OK;
}

static int timestep_kind(nessi_batch *b, int n, bool vie, const char *name) {
    NvtxRange nvtx_(vie ? "nessi::vie2_timestep" : "nessi::dyson_timestep");
    CKR(check_batch(b));
    bool any = false;
    for (Group &g : b->groups) {
        if (g.vie != vie) continue;
        any = true;
        if (n <= g.k) { set_err("%s: n = %d must exceed the solve order %d", name, n, g.k); return NESSI_ERR_ARG; }
    }
    if (!any) { set_err("%s: the batch has no %s group", name, vie ? "VIE2 (nessi_gpu_set_F)" : "Dyson"); return NESSI_ERR_ARG; }
    for (Group &g : b->groups) {
        if (g.vie != vie) continue;
        int nact = 0;
        for (int i : g.members) nact += b->probs[i].d.nt >= n ? 1 : 0;
        if (nact == 0) continue;
        if (vie)
            for (int i = 0; i < nact; i++)
                if (!b->probs[g.members[i]].qret) { set_err("%s: Q of problem %d not set", name, g.members[i]); return NESSI_ERR_ARG; }
        CKR(step_dispatch(b, g, n, nact));
    }
    return NESSI_OK;
}

int nessi_gpu_dyson_timestep(nessi_batch *b, int n) { return timestep_kind(b, n, false, "dyson_timestep"); }

int nessi_gpu_vie2_timestep(nessi_batch *b, int n) { return timestep_kind(b, n, true, "vie2_timestep"); }

int nessi_gpu_set_stream(nessi_batch *b, void *stream) {
    CKR(check_batch(b));
    CK(cudaStreamSynchronize(b->stream));
    if (b->own_stream) { cudaStreamDestroy(b->stream); b->own_stream = false; }
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        CK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->own_stream = true;
    }
    return NESSI_OK;
}

int nessi_gpu_set_profiling(nessi_batch *b, int on) {
    CKR(check_batch(b));
    CK(cudaStreamSynchronize(b->stream));
    b->prof = on != 0;
    for (auto &k : b->kp) { k.used = 0; k.launches = 0; k.bytes = 0; }
    return NESSI_OK;
}

int nessi_gpu_read_profile(nessi_batch *b, int kernel, double *ms, long long *launches, double *bytes) {
    CKR(check_batch(b));
    if (kernel < 0 || kernel >= NESSI_KERNEL_COUNT) { set_err("bad kernel id %d", kernel); return NESSI_ERR_ARG; }
    CK(cudaStreamSynchronize(b->stream));
    KProf &k = b->kp[kernel];
    double t = 0;
    for (int i = 0; i + 1 < k.used; i += 2) {
        float x = 0;
        CK(cudaEventElapsedTime(&x, k.ev[i], k.ev[i + 1]));
        t += x;
    }
    if (ms) *ms = t;
    if (launches) *launches = k.launches;
    if (bytes) *bytes = k.bytes;
    k.used = 0; k.launches = 0; k.bytes = 0;
    return NESSI_OK;
}

// libcntr's Matsubara methods (cntr_global_settings.hpp): 0 Fourier, 1 steepest descent (CG), 2 fixpoint.
// vie2_mat by steepest descent also needs Fcc^mat (nessi_gpu_set_Fcc_mat; checked per group).
static int check_mat_method(int method, bool vie, const char *name) {
    (void)vie;
    if (method == 0 || method == 1 || method == 2) return NESSI_OK;
    set_err("%s: method %d not available (0 = Fourier, 1 = steepest descent, 2 = fixpoint)", name, method);
    return NESSI_ERR_ARG;
}

int nessi_gpu_dyson_mat_method(nessi_batch *b, int method, int force_hermitian) {
    NvtxRange nvtx_("nessi::dyson_mat");
    CKR(check_batch(b));
    CKR(check_mat_method(method, false, "dyson_mat"));
    for (Group &g : b->groups) {
        if (g.vie) continue;  // VIE2 groups take G^mat from the caller
        if (g.ntau % 2) { set_err("dyson_mat: ntau must be even (matsubara_inverse)"); return NESSI_ERR_ARG; }
        CKR(mat_dispatch(b, g, method, force_hermitian ? 1 : 0));
    }
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_dyson_mat(nessi_batch *b) { return nessi_gpu_dyson_mat_method(b, 2, 1); }

static int start_kind(nessi_batch *b, bool vie, const char *name) {
    NvtxRange nvtx_(vie ? "nessi::vie2_start" : "nessi::dyson_start");
    CKR(check_batch(b));
    bool any = false;
    for (Group &g : b->groups) {
        if (g.vie != vie) continue;
        any = true;
        for (int i : g.members) {
            if (b->probs[i].d.nt < g.k) { set_err("%s: nt must be >= SolveOrder", name); return NESSI_ERR_ARG; }
            if (vie && !b->probs[i].qret) { set_err("%s: Q of problem %d not set", name, i); return NESSI_ERR_ARG; }
        }
    }
    if (!any) { set_err("%s: the batch has no %s group", name, vie ? "VIE2 (nessi_gpu_set_F)" : "Dyson"); return NESSI_ERR_ARG; }
    for (Group &g : b->groups)
        if (g.vie == vie) CKR(start_dispatch(b, g));
    for (Prob &q : b->probs) {
        if (b->groups[q.group].vie != vie) continue;
        const long row = (long)(q.d.ntau + 1) * q.d.size1 * q.d.size1;
        CKR(refresh32(b, q.gtv32, q.gtv, (b->groups[q.group].k + 1) * row));
    }
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_dyson_start(nessi_batch *b) { return start_kind(b, false, "dyson_start"); }

int nessi_gpu_vie2_start(nessi_batch *b) { return start_kind(b, true, "vie2_start"); }

int nessi_gpu_vie2_mat(nessi_batch *b) { return nessi_gpu_vie2_mat_method(b, 2); }

int nessi_gpu_vie2_mat_method(nessi_batch *b, int method) {
    NvtxRange nvtx_("nessi::vie2_mat");
    CKR(check_batch(b));
    CKR(check_mat_method(method, true, "vie2_mat"));
    bool any = false;
    for (Group &g : b->groups) {
        if (!g.vie) continue;
        any = true;
        if (g.ntau % 2) { set_err("vie2_mat: ntau must be even (matsubara_inverse)"); return NESSI_ERR_ARG; }
        if (method == 1 && !g.fccmat) {
            set_err("vie2_mat: steepest descent needs Fcc^mat of the group (nessi_gpu_set_Fcc_mat)");
            return NESSI_ERR_ARG;
        }
        CKR(vie2_mat_dispatch(b, g, method));
    }
    if (!any) { set_err("vie2_mat: the batch has no VIE2 group (nessi_gpu_set_F)"); return NESSI_ERR_ARG; }
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

static int sync_probdev(nessi_batch *b, int p) {
    Prob &q = b->probs[p];
    Group &g = b->groups[q.group];
    for (size_t c = 0; c < g.members.size(); c++) {
        if (g.members[c] != p) continue;
        ProbDev &pd = g.h_probs[c];
        pd.qret = q.qret; pd.qles = q.qles; pd.qtv = q.qtv;
        CK(cudaMemcpyAsync(g.d_probs + c, &pd, sizeof(ProbDev), cudaMemcpyHostToDevice, b->stream));
        CK(cudaStreamSynchronize(b->stream));
    }
    return NESSI_OK;
}

static int ensure_q(nessi_batch *b, int p) {
    Prob &q = b->probs[p];
    if (q.qret) return NESSI_OK;
    const long s2 = (long)q.d.size1 * q.d.size1, nt = q.d.nt, M = q.d.ntau + 1;
    CKR(b->alloc(&q.qret, tri_h(nt + 1) * s2));
    CKR(b->alloc(&q.qles, tri_h(nt + 1) * s2));
    CKR(b->alloc(&q.qtv, (nt + 1) * M * s2));
    CKR(b->alloc(&q.qmat, M * s2));
    return sync_probdev(b, p);
}

int nessi_gpu_set_Q(nessi_batch *b, int p, const void *ret, const void *les, const void *tv, const void *mat) {
    CKR(check_prob(b, p));
    CKR(ensure_q(b, p));
    Prob &q = b->probs[p];
    const long s2 = (long)q.d.size1 * q.d.size1, nt = q.d.nt, M = q.d.ntau + 1;
    CKR(copy_cplx(b, q.qret, ret, tri_h(nt + 1) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, q.qles, les, tri_h(nt + 1) * s2, cudaMemcpyHostToDevice));
    CKR(tv_transfer(b, q.qtv, (void *)tv, 0, nt + 1, (int)M, q.d.size1, true));
    CKR(copy_cplx(b, q.qmat, mat, M * s2, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_set_Q_timestep(nessi_batch *b, int p, int tstp, const void *slice) {
    CKR(check_prob(b, p));
    CKR(ensure_q(b, p));
    Prob &q = b->probs[p];
    return slice_copy(b, q.qret, q.qtv, q.qles, q.qmat, q.d.nt, q.d.ntau, q.d.size1, tstp, (void *)slice, true, true);
}

static int ensure_fcc(nessi_batch *b, Group &g) {
    g.vie = true;
    if (g.fccret) return NESSI_OK;
    const long s2 = (long)g.s * g.s, N = g.ntmax + 1;
    CKR(b->alloc(&g.fccret, tri_h(N) * s2));
    CKR(b->alloc(&g.fccles, tri_h(N) * s2));
    return NESSI_OK;
}

int nessi_gpu_set_F(nessi_batch *b, int group, const void *ret, const void *les, const void *tv, const void *mat,
                    const void *cc_ret, const void *cc_les) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    if (g->U) { set_err("set_F: group %d is a lattice (Dyson) group", group); return NESSI_ERR_ARG; }
    CKR(ensure_fcc(b, *g));
    const long s2 = (long)g->s * g->s, N = g->ntmax + 1, M = g->ntau + 1;
    CKR(copy_cplx(b, g->sret, ret, tri_h(N) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g->sles, les, tri_h(N) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g->stv, tv, N * M * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g->smat, mat, M * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g->fccret, cc_ret, tri_h(N) * s2, cudaMemcpyHostToDevice));
    CKR(copy_cplx(b, g->fccles, cc_les, tri_h(N) * s2, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    g->ret_valid = g->les_valid = g->dense_valid = -1;
    return NESSI_OK;
}

int nessi_gpu_set_Fcc_mat(nessi_batch *b, int group, const void *cc_mat) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    if (g->U) { set_err("set_Fcc_mat: group %d is a lattice (Dyson) group", group); return NESSI_ERR_ARG; }
    if (!cc_mat) { set_err("set_Fcc_mat: null Fcc^mat"); return NESSI_ERR_ARG; }
    CKR(ensure_fcc(b, *g));
    const long M = g->ntau + 1, s2 = (long)g->s * g->s;
    if (!g->fccmat) CKR(b->alloc(&g->fccmat, M * s2));
    CKR(copy_cplx(b, g->fccmat, cc_mat, M * s2, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_set_F_timestep(nessi_batch *b, int group, int tstp, const void *slice, const void *cc_slice) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    if (g->U) { set_err("set_F_timestep: group %d is a lattice (Dyson) group", group); return NESSI_ERR_ARG; }
    CKR(ensure_fcc(b, *g));
    CKR(slice_copy(b, g->sret, g->stv, g->sles, g->smat, g->ntmax, g->ntau, g->s, tstp, (void *)slice, true, false));
    if (tstp >= 0) {
        // the ret and les parts of the Fcc slice; its tv part is not used by the VIE2 step
        if (!cc_slice) { set_err("set_F_timestep: null Fcc slice"); return NESSI_ERR_ARG; }
        const long s2 = (long)g->s * g->s, n1 = tstp + 1, M = g->ntau + 1;
        const double2 *h = (const double2 *)cc_slice;
        CKR(copy_cplx(b, g->fccret + tri_h(tstp) * s2, h, n1 * s2, cudaMemcpyHostToDevice));
        CKR(copy_cplx(b, g->fccles + tri_h(tstp) * s2, h + (n1 + M) * s2, n1 * s2, cudaMemcpyHostToDevice));
        CK(cudaStreamSynchronize(b->stream));
        sigma_changed(*g, tstp);
    }
    return NESSI_OK;
}


static int ensure_loc(nessi_batch *b, Group &g) {
    if (g.loc.ret) return NESSI_OK;
    const long s2 = (long)g.s * g.s, N = g.ntmax + 1, M = g.ntau + 1;
    CKR(b->alloc(&g.loc.ret, tri_h(N) * s2));
    CKR(b->alloc(&g.loc.les, tri_h(N) * s2));
    CKR(b->alloc(&g.loc.tv, N * M * s2));
    CKR(b->alloc(&g.loc.mat, M * s2));
    g.gloc_ld = (2 * N + M) * s2;  // longest slice
    const long nchunk = ((long)g.members.size() + GLOC_CHUNK - 1) / GLOC_CHUNK;
    CKR(b->alloc(&g.gloc_part, nchunk * g.gloc_ld));
    return NESSI_OK;
}

int nessi_gpu_set_U(nessi_batch *b, int group, const void *U) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    if (!U) { set_err("null U"); return NESSI_ERR_ARG; }
    if (g->vie) { set_err("set_U: group %d is a VIE2 group", group); return NESSI_ERR_ARG; }
    CKR(ensure_loc(b, *g));
    if (!g->U) CKR(b->alloc(&g->U, (long)(g->ntmax + 2) * g->s));
    CKR(copy_cplx(b, g->U, U, (long)(g->ntmax + 2) * g->s, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_extrapolate_timestep(nessi_batch *b, int n) {
    NvtxRange nvtx_("nessi::extrapolate_timestep");
    CKR(check_batch(b));
    for (Group &g : b->groups)
        if (n < g.k) { set_err("extrapolate_timestep: n = %d below the solve order %d", n, g.k); return NESSI_ERR_ARG; }
    b->prof_mark(NESSI_KERNEL_LATTICE);
    for (Group &g : b->groups) {
        if (active_members(b, g, n + 1) == 0) continue;
        CKR(extrap_dispatch(b, g, n));
    }
    b->prof_end(NESSI_KERNEL_LATTICE, 0.0);
    return NESSI_OK;
}

int nessi_gpu_gloc_timestep(nessi_batch *b, int group, int tstp) {
    NvtxRange nvtx_("nessi::gloc_timestep");
    Group *g;
    CKR(find_group_checked(b, group, &g));
    if (tstp < -1 || tstp > g->ntmax) { set_err("gloc: time step %d out of range", tstp); return NESSI_ERR_ARG; }
    CKR(ensure_loc(b, *g));
    b->prof_mark(NESSI_KERNEL_LATTICE);
    CKR(gloc_dispatch(b, *g, tstp));
    b->prof_end(NESSI_KERNEL_LATTICE, 0.0);
    return NESSI_OK;
}

int nessi_gpu_sigma_2b_timestep(nessi_batch *b, int group, int tstp) {
    NvtxRange nvtx_("nessi::sigma_2b_timestep");
    Group *g;
    CKR(find_group_checked(b, group, &g));
    if (!g->U) { set_err("sigma_2b: nessi_gpu_set_U was not called for group %d", group); return NESSI_ERR_ARG; }
    if (tstp < -1 || tstp > g->ntmax) { set_err("sigma_2b: time step %d out of range", tstp); return NESSI_ERR_ARG; }
    b->prof_mark(NESSI_KERNEL_LATTICE);
    CKR(sigma2b_dispatch(b, *g, tstp));
    b->prof_end(NESSI_KERNEL_LATTICE, 0.0);
    return NESSI_OK;
}

int nessi_gpu_get_gloc(nessi_batch *b, int group, void *ret, void *les, void *tv, void *mat) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    CKR(ensure_loc(b, *g));
    const long s2 = (long)g->s * g->s, N = g->ntmax + 1, M = g->ntau + 1;
    CKR(copy_cplx(b, ret, g->loc.ret, tri_h(N) * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, les, g->loc.les, tri_h(N) * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, tv, g->loc.tv, N * M * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, mat, g->loc.mat, M * s2, cudaMemcpyDeviceToHost));
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_get_sigma(nessi_batch *b, int group, void *ret, void *les, void *tv, void *mat) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    const long s2 = (long)g->s * g->s, N = g->ntmax + 1, M = g->ntau + 1;
    CKR(copy_cplx(b, ret, g->sret, tri_h(N) * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, les, g->sles, tri_h(N) * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, tv, g->stv, N * M * s2, cudaMemcpyDeviceToHost));
    CKR(copy_cplx(b, mat, g->smat, M * s2, cudaMemcpyDeviceToHost));
    CK(cudaStreamSynchronize(b->stream));
    return NESSI_OK;
}

int nessi_gpu_gloc_device(nessi_batch *b, int group, void **ret, void **les, void **tv, void **mat) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    CKR(ensure_loc(b, *g));
    if (ret) *ret = g->loc.ret;
    if (les) *les = g->loc.les;
    if (tv) *tv = g->loc.tv;
    if (mat) *mat = g->loc.mat;
    return NESSI_OK;
}

// distance_norm2 of time step t between two herm_matrix_timestep-like host buffers (ret row,
// tv row, les column of t; cntr_utilities_impl.hpp:607-650)
static double slice_distance(const double2 *a, const double2 *b, long n_elem, int s2) {
    double err = 0;
    for (long e = 0; e < n_elem; e++) {
        double r = 0;
        for (int i = 0; i < s2; i++) {
            const double dx = a[e * s2 + i].x - b[e * s2 + i].x, dy = a[e * s2 + i].y - b[e * s2 + i].y;
            r += dx * dx + dy * dy;
        }
        err += std::sqrt(r);
    }
    return err;
}

int nessi_gpu_lattice_2b_start(nessi_batch *b, int max_iter, double tol, int *iters, double *err_out) {
    NvtxRange nvtx_("nessi::lattice_2b_start");
    CKR(check_batch(b));
    if (max_iter < 0) { set_err("lattice_2b_start: max_iter < 0"); return NESSI_ERR_ARG; }
    std::vector<Group *> lat;
    for (Group &g : b->groups)
        if (g.U) lat.push_back(&g);
    if (lat.empty()) { set_err("lattice_2b_start: no group has an interaction (nessi_gpu_set_U)"); return NESSI_ERR_ARG; }
    // G_loc slices 0..k of every lattice group, downloaded after each iteration
    auto snapshot = [&](std::vector<std::vector<double2>> &out) -> int {
        out.resize(lat.size());
        for (size_t i = 0; i < lat.size(); i++) {
            Group &g = *lat[i];
            const long s2 = (long)g.s * g.s, M = g.ntau + 1, tk = tri_h(g.k + 1) * s2;
            out[i].resize(2 * tk + (g.k + 1) * M * s2);
            CKR(copy_cplx(b, out[i].data(), g.loc.ret, tk, cudaMemcpyDeviceToHost));
            CKR(copy_cplx(b, out[i].data() + tk, g.loc.les, tk, cudaMemcpyDeviceToHost));
            CKR(copy_cplx(b, out[i].data() + 2 * tk, g.loc.tv, (g.k + 1) * M * s2, cudaMemcpyDeviceToHost));
        }
        CK(cudaStreamSynchronize(b->stream));
        return NESSI_OK;
    };
    auto distance = [&](const std::vector<std::vector<double2>> &x, const std::vector<std::vector<double2>> &y) {
        double e = 0;
        for (size_t i = 0; i < lat.size(); i++) {
            const Group &g = *lat[i];
            const int s2 = g.s * g.s;
            const long M = g.ntau + 1, tk = tri_h(g.k + 1) * s2;
            for (int t = 0; t <= g.k; t++) {
                e += slice_distance(x[i].data() + tri_h(t) * s2, y[i].data() + tri_h(t) * s2, t + 1, s2);
                e += slice_distance(x[i].data() + 2 * tk + t * M * s2, y[i].data() + 2 * tk + t * M * s2, M, s2);
                e += slice_distance(x[i].data() + tk + tri_h(t) * s2, y[i].data() + tk + tri_h(t) * s2, t + 1, s2);
            }
        }
        return e;
    };
    for (Group *g : lat)
        for (int t = 0; t <= g->k; t++) CKR(gloc_dispatch(b, *g, t));
    std::vector<std::vector<double2>> prev, cur;
    CKR(snapshot(prev));
    int iter = 0;
    double err = 0;
    for (iter = 0; iter <= max_iter; iter++) {
        for (Group *g : lat)
            for (int t = 0; t <= g->k; t++) CKR(sigma2b_dispatch(b, *g, t));
        CKR(nessi_gpu_dyson_start(b));
        for (Group *g : lat)
            for (int t = 0; t <= g->k; t++) CKR(gloc_dispatch(b, *g, t));
        CKR(snapshot(cur));
        err = distance(cur, prev);
        if (err < tol && iter > 2) break;
        prev.swap(cur);
    }
    if (iters) *iters = iter > max_iter ? max_iter + 1 : iter + 1;
    if (err_out) *err_out = err;
    return NESSI_OK;
}

int nessi_gpu_lattice_2b_timestep(nessi_batch *b, int n, int corrector_steps) {
    NvtxRange nvtx_("nessi::lattice_2b_timestep");
    CKR(check_batch(b));
    if (corrector_steps < 1) { set_err("lattice_2b_timestep: corrector_steps must be >= 1"); return NESSI_ERR_ARG; }
    bool any = false;
    for (Group &g : b->groups) {
        if (n <= g.k) { set_err("lattice_2b_timestep: n = %d must exceed the solve order %d", n, g.k); return NESSI_ERR_ARG; }
        any = any || g.U != nullptr;
    }
    if (!any) { set_err("lattice_2b_timestep: no group has an interaction (nessi_gpu_set_U)"); return NESSI_ERR_ARG; }
    CKR(nessi_gpu_extrapolate_timestep(b, n - 1));
    for (int it = 0; it < corrector_steps; it++) {
        b->prof_mark(NESSI_KERNEL_LATTICE);
        for (Group &g : b->groups) {
            if (!g.U || active_members(b, g, n) == 0) continue;
            CKR(gloc_dispatch(b, g, n));
            CKR(sigma2b_dispatch(b, g, n));
        }
        b->prof_end(NESSI_KERNEL_LATTICE, 0.0);
        CKR(nessi_gpu_dyson_timestep(b, n));
    }
    b->prof_mark(NESSI_KERNEL_LATTICE);
    for (Group &g : b->groups)
        if (g.U && active_members(b, g, n) > 0) CKR(gloc_dispatch(b, g, n));
    b->prof_end(NESSI_KERNEL_LATTICE, 0.0);
    return NESSI_OK;
}

int nessi_gpu_get_volterra_choice(nessi_batch *b, int group, int *pp_ret, int *pp_les) {
    Group *g;
    CKR(find_group_checked(b, group, &g));
    const int fixed = b->volterra_pp;
    if (pp_ret) *pp_ret = fixed != 0 ? fixed : g->pp_ret;
    if (pp_les) *pp_les = fixed != 0 ? fixed : g->pp_les;
    return NESSI_OK;
}

int nessi_gpu_graph_record(nessi_batch *b, int kind, int n0, int n1, int corrector_steps) {
    NvtxRange nvtx_("nessi::graph_record");
    CKR(check_batch(b));
    if (kind < 0 || kind > 2 || n1 < n0) { set_err("graph_record: bad arguments"); return NESSI_ERR_ARG; }
    CK(cudaStreamSynchronize(b->stream));
    CK(cudaStreamSynchronize(b->side));
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    const bool prof = b->prof;
    b->prof = false;  // no timing events inside the graph
    CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = NESSI_OK;
    for (int n = n0; n <= n1 && rc == NESSI_OK; n++) {
        if (kind == 0) rc = nessi_gpu_dyson_timestep(b, n);
        else if (kind == 1) rc = nessi_gpu_vie2_timestep(b, n);
        else rc = nessi_gpu_lattice_2b_timestep(b, n, corrector_steps);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    b->prof = prof;
    if (rc != NESSI_OK) { if (g) cudaGraphDestroy(g); return rc; }
    if (e != cudaSuccess) {
        set_err("graph_record: capture failed: %s", cudaGetErrorString(e));
        if (g) cudaGraphDestroy(g);
        return NESSI_ERR_CUDA;
    }
    const cudaError_t e2 = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e2 != cudaSuccess) { b->graph = nullptr; set_err("graph_record: instantiate failed: %s", cudaGetErrorString(e2)); return NESSI_ERR_CUDA; }
    return NESSI_OK;
}

int nessi_gpu_graph_launch(nessi_batch *b) {
    NvtxRange nvtx_("nessi::graph_launch");
    CKR(check_batch(b));
    if (!b->graph) { set_err("graph_launch: nothing recorded"); return NESSI_ERR_ARG; }
    CK(cudaGraphLaunch(b->graph, b->stream));
    return NESSI_OK;
}

int nessi_gpu_synchronize(nessi_batch *b) {
    CKR(check_batch(b));
    CK(cudaStreamSynchronize(b->stream));
    int err = 0;
    CK(cudaMemcpy(&err, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        CK(cudaMemset(b->d_err, 0, sizeof(int)));
        set_err("a bounded device wait gave up; the time steps since the last check are invalid");
        return NESSI_ERR_TIMEOUT;
    }
    return NESSI_OK;
}

int nessi_gpu_set_wait_limit(nessi_batch *b, long long ns) {
    CKR(check_batch(b));
    if (ns < 0) { set_err("wait limit %lld < 0", ns); return NESSI_ERR_ARG; }
    b->wait_ns = ns;
    return NESSI_OK;
}

}  // extern "C"

// =====================================================================================
// dyson_mat without allocation
// =====================================================================================
// Some callers cannot let a library call cudaMalloc: a host application whose device memory is
// owned by another allocator (a framework's memory pool, a preallocated arena sized at start-up),
// or one that must not take the device-wide synchronisation a cudaMalloc / cudaFree can bring.
// nessi_gpu_dyson_mat_noalloc serves them: the caller passes every input and output as device
// pointers and the scratch lives in the fixed array below, which every GPU that loads this
// library holds until the process exits.  The first call on a device does the set-up (tables,
// scratch address; guarded by a mutex), so make it before any stream capture.
#define NESSI_NOALLOC_MAX_CPLX (1 << 17)  // 131072 complex<double> = 2 MiB
static __device__ __align__(256) double2 g_noalloc_scratch[NESSI_NOALLOC_MAX_CPLX];

namespace {
// device address of g_noalloc_scratch per device, looked up once with that device current
double2 *g_noalloc_addr[64] = {nullptr};

template <int S>
__global__ void __launch_bounds__(256) k_dyson_mat_single(GroupDev g, ProbDev p, MatScratch w) {
    dyson_mat_body<S>(g, p, w);
}

template <int S>
int noalloc_launch(const GroupDev &gd, const ProbDev &pd, const MatScratch &w, int ntau, cudaStream_t st) {
    CKR(check_twiddle_smem((const void *)k_dyson_mat_single<S>, ntau, "dyson_mat_noalloc"));
    const size_t sm = 2 * (size_t)ntau * sizeof(double2);
    CK(cudaFuncSetAttribute(k_dyson_mat_single<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_dyson_mat_single<S><<<1, 256, sm, st>>>(gd, pd, w);
    CK(cudaGetLastError());
    return NESSI_OK;
}
}  // namespace

extern "C" int nessi_gpu_dyson_mat_noalloc(int ntau, int size1, int sig, int solve_order, double beta, double mu,
                                           const void *H, const void *sigma_mat, void *gmat, void *stream) {
    NvtxRange nvtx_("nessi::dyson_mat_noalloc");
    if (!H || !sigma_mat || !gmat) { set_err("dyson_mat_noalloc: null pointer"); return NESSI_ERR_ARG; }
    if (size1 < 1 || size1 > NESSI_MAXS || (sig != 1 && sig != -1) || solve_order < 1 || solve_order > CNTR_KMAX ||
        ntau < solve_order || ntau % 2 || !(beta > 0)) {
        set_err("dyson_mat_noalloc: bad arguments (ntau=%d size1=%d sig=%d k=%d)", ntau, size1, sig, solve_order);
        return NESSI_ERR_ARG;
    }
    const long s2 = (long)size1 * size1, M = ntau + 1;
    const long need = 6 * M * s2 + 2L * ntau * s2;
    if (need > NESSI_NOALLOC_MAX_CPLX) {
        set_err("dyson_mat_noalloc: 6(ntau+1)s^2 + 2 ntau s^2 = %ld complex exceeds the fixed scratch of %d", need,
                NESSI_NOALLOC_MAX_CPLX);
        return NESSI_ERR_ARG;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { set_err("dyson_mat_noalloc: device index %d unsupported", dev); return NESSI_ERR_ARG; }
    double2 *base = nullptr;
    {
        // set-up on the first call on this device: integration tables and the scratch address
        CKR(ensure_tables(dev));
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_noalloc_addr[dev]) {
            void *ptr = nullptr;
            CK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
            g_noalloc_addr[dev] = (double2 *)ptr;
        }
        base = g_noalloc_addr[dev];
    }
    MatScratch w;
    w.G0 = base; w.F = base + M * s2; w.Q = base + 2 * M * s2; w.dG = base + 3 * M * s2;
    w.fdft = base + 4 * M * s2; w.qdft = base + 5 * M * s2; w.Z = base + 6 * M * s2;
    GroupDev gd;
    std::memset(&gd, 0, sizeof gd);
    gd.smat = (const double2 *)sigma_mat;
    gd.ntau = ntau; gd.s = size1; gd.sig = sig; gd.k = solve_order; gd.beta = beta;
    ProbDev pd;
    std::memset(&pd, 0, sizeof pd);
    pd.H = (const double2 *)H;
    pd.gmat = (double2 *)gmat;
    pd.mu = mu;
    cudaStream_t st = (cudaStream_t)stream;
    switch (size1) {
        case 1: return noalloc_launch<1>(gd, pd, w, ntau, st);
        case 2: return noalloc_launch<2>(gd, pd, w, ntau, st);
        case 3: return noalloc_launch<3>(gd, pd, w, ntau, st);
        case 4: return noalloc_launch<4>(gd, pd, w, ntau, st);
        case 5: return noalloc_launch<5>(gd, pd, w, ntau, st);
        case 6: return noalloc_launch<6>(gd, pd, w, ntau, st);
        case 7: return noalloc_launch<7>(gd, pd, w, ntau, st);
        case 8: return noalloc_launch<8>(gd, pd, w, ntau, st);
    }
    set_err("dyson_mat_noalloc: size1 %d unsupported", size1);
    return NESSI_ERR_ARG;
}

// =====================================================================================
// convolution_timestep on device-resident herm_matrix data
// =====================================================================================
namespace {
template <int S> int conv_launch(const ConvBatch &cb, int n, cudaStream_t st) {
    const long s2 = (long)S * S, M = cb.ntau + 1;
    auto blocks = [](long items) { return (unsigned)std::min<long>(std::max<long>(1, (items + 127) / 128), 1024); };
    if (n < 0) {
        k_conv_mat<S><<<dim3(blocks(M * s2), cb.count), 128, 0, st>>>(cb);
        CK(cudaGetLastError());
        return NESSI_OK;
    }
    k_conv_ret<S><<<dim3(blocks((n + 1) * s2), cb.count), 128, 0, st>>>(cb, n);
    CK(cudaGetLastError());
    k_conv_tv<S><<<dim3(blocks(M * s2), cb.count), 128, 0, st>>>(cb, n);
    CK(cudaGetLastError());
    k_conv_les<S><<<dim3(blocks((n + 1) * s2), cb.count), 128, 0, st>>>(cb, n);
    CK(cudaGetLastError());
    return NESSI_OK;
}
}  // namespace

extern "C" int nessi_gpu_convolution_timestep(int n, int count, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                              const nessi_hm_ptrs *Acc, const nessi_hm_ptrs *B,
                                              const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1, int sig_a,
                                              int sig_b, int solve_order, double beta, double h, void *stream) {
    NvtxRange nvtx_("nessi::convolution_timestep");
    if (count < 0 || !C || !A || !Acc || !B || !Bcc) { set_err("convolution_timestep: bad arguments"); return NESSI_ERR_ARG; }
    if (size1 < 1 || size1 > NESSI_MAXS || solve_order < 1 || solve_order > CNTR_KMAX || nt < solve_order ||
        ntau < solve_order || n < -1 || n > nt || (sig_a != 1 && sig_a != -1) || (sig_b != 1 && sig_b != -1) ||
        !(beta > 0) || !(h > 0)) {
        set_err("convolution_timestep: bad dimensions (n=%d nt=%d ntau=%d size1=%d k=%d)", n, nt, ntau, size1,
                solve_order);
        return NESSI_ERR_ARG;
    }
    for (int i = 0; i < count; i++) {
        const nessi_hm_ptrs *all[5] = {&C[i], &A[i], &Acc[i], &B[i], &Bcc[i]};
        bool ok = B[i].mat != nullptr;  // B^mat enters C^tv and C^mat
        if (n >= 0)
            for (const nessi_hm_ptrs *x : all) ok = ok && x->ret && x->les && x->tv;
        else
            ok = ok && A[i].mat && C[i].mat;
        if (!ok) { set_err("convolution_timestep: problem %d has a null pointer it needs", i); return NESSI_ERR_ARG; }
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { set_err("convolution_timestep: device index %d unsupported", dev); return NESSI_ERR_ARG; }
    CKR(ensure_tables(dev));
    cudaStream_t st = (cudaStream_t)stream;
    auto conv = [](const nessi_hm_ptrs &x) {
        ConvHM y;
        y.ret = (double2 *)x.ret; y.les = (double2 *)x.les; y.tv = (double2 *)x.tv; y.mat = (double2 *)x.mat;
        return y;
    };
    for (int i0 = 0; i0 < count; i0 += NESSI_CONV_MAXP) {
        ConvBatch cb;
        std::memset(&cb, 0, sizeof cb);
        cb.count = std::min(NESSI_CONV_MAXP, count - i0);
        for (int i = 0; i < cb.count; i++) {
            cb.p[i].C = conv(C[i0 + i]); cb.p[i].A = conv(A[i0 + i]); cb.p[i].Acc = conv(Acc[i0 + i]);
            cb.p[i].B = conv(B[i0 + i]); cb.p[i].Bcc = conv(Bcc[i0 + i]);
        }
        cb.ntau = ntau; cb.sig_a = sig_a; cb.sig_b = sig_b; cb.k = solve_order; cb.h = h; cb.beta = beta;
        int r = NESSI_ERR_ARG;
        switch (size1) {
            case 1: r = conv_launch<1>(cb, n, st); break;
            case 2: r = conv_launch<2>(cb, n, st); break;
            case 3: r = conv_launch<3>(cb, n, st); break;
            case 4: r = conv_launch<4>(cb, n, st); break;
            case 5: r = conv_launch<5>(cb, n, st); break;
            case 6: r = conv_launch<6>(cb, n, st); break;
            case 7: r = conv_launch<7>(cb, n, st); break;
            case 8: r = conv_launch<8>(cb, n, st); break;
        }
        if (r != NESSI_OK) return r;
    }
    return NESSI_OK;
}

// Host-data convenience for single calls with libcntr's signature: copies the five herm_matrix
// objects to the device, runs the convolution for time step n and copies C's time step back.
// time steps n0..n1 of C = A * B on host herm_matrix data: upload the operands once, run the
// steps on the device, bring back C's steps n0..n1 (all of C when the range is -1..nt)
static int convolution_host_range(int n0, int n1, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                  const nessi_hm_ptrs *Acc, const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt,
                                  int ntau, int size1, int sig_a, int sig_b, int solve_order, double beta, double h,
                                  const char *name) {
    if (!C || !A || !Acc || !B || !Bcc || nt < 0 || ntau < 0 || size1 < 1 || size1 > NESSI_MAXS) {
        set_err("%s: bad arguments", name);
        return NESSI_ERR_ARG;
    }
    CK(cudaSetDevice(g_device));
    const long s2 = (long)size1 * size1, M = ntau + 1;
    const long len[4] = {tri_h(nt + 1) * s2, tri_h(nt + 1) * s2, (long)(nt + 1) * M * s2, M * s2};
    const nessi_hm_ptrs *hs[5] = {C, A, Acc, B, Bcc};
    nessi_hm_ptrs ds[5];
    std::vector<void *> owned;
    int rc = NESSI_OK;
    for (int i = 0; i < 5 && rc == NESSI_OK; i++) {
        void **dst[4] = {&ds[i].ret, &ds[i].les, &ds[i].tv, &ds[i].mat};
        void *const src[4] = {hs[i]->ret, hs[i]->les, hs[i]->tv, hs[i]->mat};
        for (int c = 0; c < 4; c++) {
            *dst[c] = nullptr;
            if (!src[c]) continue;
            if (cudaMalloc(dst[c], (size_t)len[c] * 16) != cudaSuccess) { set_err("cudaMalloc failed"); rc = NESSI_ERR_OOM; break; }
            owned.push_back(*dst[c]);
            if (cudaMemcpy(*dst[c], src[c], (size_t)len[c] * 16, cudaMemcpyHostToDevice) != cudaSuccess) {
                set_err("upload failed");
                rc = NESSI_ERR_CUDA;
                break;
            }
        }
    }
    for (int n = n0; n <= n1 && rc == NESSI_OK; n++)
        rc = nessi_gpu_convolution_timestep(n, 1, &ds[0], &ds[1], &ds[2], &ds[3], &ds[4], nt, ntau, size1, sig_a, sig_b,
                                            solve_order, beta, h, nullptr);
    if (rc == NESSI_OK && cudaDeviceSynchronize() != cudaSuccess) { set_err("convolution failed"); rc = NESSI_ERR_CUDA; }
    if (rc == NESSI_OK) {
        // C's time steps n0..n1: ret rows, tv rows, les columns (and mat for n0 = -1)
        auto back = [&](void *hp, const void *d, long off, long cnt) {
            if (!hp || !d) return cudaSuccess;
            return cudaMemcpy((char *)hp + off * 16, (const char *)d + off * 16, (size_t)cnt * 16, cudaMemcpyDeviceToHost);
        };
        cudaError_t e = cudaSuccess;
        if (n0 < 0) e = back(C->mat, ds[0].mat, 0, M * s2);
        const int t0 = n0 < 0 ? 0 : n0;
        if (n1 >= t0 && e == cudaSuccess) {
            // rows / columns t0..n1 are contiguous in the packed triangles and in tv
            e = back(C->ret, ds[0].ret, tri_h(t0) * s2, (tri_h(n1 + 1) - tri_h(t0)) * s2);
            if (e == cudaSuccess) e = back(C->tv, ds[0].tv, (long)t0 * M * s2, (long)(n1 - t0 + 1) * M * s2);
            if (e == cudaSuccess) e = back(C->les, ds[0].les, tri_h(t0) * s2, (tri_h(n1 + 1) - tri_h(t0)) * s2);
        }
        if (e != cudaSuccess) { set_err("download failed"); rc = NESSI_ERR_CUDA; }
    }
    for (void *q : owned) cudaFree(q);
    return rc;
}

extern "C" int nessi_gpu_convolution_timestep_host(int n, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                                   const nessi_hm_ptrs *Acc, const nessi_hm_ptrs *B,
                                                   const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1, int sig_a,
                                                   int sig_b, int solve_order, double beta, double h) {
    if (n < -1 || n > nt) { set_err("convolution_timestep_host: time step %d out of range", n); return NESSI_ERR_ARG; }
    return convolution_host_range(n, n, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h,
                                  "convolution_timestep_host");
}

extern "C" int nessi_gpu_convolution_host(const nessi_hm_ptrs *C, const nessi_hm_ptrs *A, const nessi_hm_ptrs *Acc,
                                          const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1,
                                          int sig_a, int sig_b, int solve_order, double beta, double h) {
    return convolution_host_range(-1, nt, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h,
                                  "convolution_host");
}

// =====================================================================================
// distance_norm2 on device-resident herm_matrix data
// =====================================================================================
extern "C" int nessi_gpu_distance_norm2(int tstp, const nessi_hm_ptrs *g1, const nessi_hm_ptrs *g2, int nt, int ntau,
                                        int size1, double *out, void *stream) {
    NvtxRange nvtx_("nessi::distance_norm2");
    if (!g1 || !g2 || !out || nt < -1 || ntau < 0 || size1 < 1 || size1 > NESSI_MAXS || tstp < -1 || tstp > nt) {
        set_err("distance_norm2: bad arguments (tstp=%d nt=%d ntau=%d size1=%d)", tstp, nt, ntau, size1);
        return NESSI_ERR_ARG;
    }
    const bool ok = tstp < 0 ? (g1->mat && g2->mat) : (g1->ret && g1->les && g1->tv && g2->ret && g2->les && g2->tv);
    if (!ok) { set_err("distance_norm2: a component it reads is null"); return NESSI_ERR_ARG; }
    auto conv = [](const nessi_hm_ptrs &x) {
        ConvHM y;
        y.ret = (double2 *)x.ret; y.les = (double2 *)x.les; y.tv = (double2 *)x.tv; y.mat = (double2 *)x.mat;
        return y;
    };
    k_distance_norm2<<<1, 256, 0, (cudaStream_t)stream>>>(tstp, conv(*g1), conv(*g2), ntau, size1 * size1, out);
    CK(cudaGetLastError());
    return NESSI_OK;
}

// =====================================================================================
// GW diagrams on device herm_matrix data
// =====================================================================================
static int gw_launch(int which, int tstp, int nk, const nessi_hm_ptrs *G, const nessi_hm_ptrs *W,
                     const nessi_hm_ptrs *out, const double *w, int nt, int ntau, int size1, int sig_b, void *stream,
                     const char *name) {
    if (!G || !out || !w || (which == 2 && !W) || nk < 1 || nt < -1 || ntau < 0 || size1 < 1 || size1 > NESSI_MAXS ||
        tstp < -1 || tstp > nt || (sig_b != 1 && sig_b != -1)) {
        set_err("%s: bad arguments (tstp=%d nk=%d nt=%d ntau=%d size1=%d)", name, tstp, nk, nt, ntau, size1);
        return NESSI_ERR_ARG;
    }
    const long items = tstp < 0 ? (long)(ntau + 1) * size1 * size1 : (long)(tstp + 1 + ntau + 1) * size1 * size1;
    const dim3 grid((unsigned)std::min<long>((items + 127) / 128, 1024), (unsigned)nk);
    static_assert(sizeof(nessi_hm_ptrs) == sizeof(ConvHM), "pointer tables share one layout");
    k_gw_bubbles<<<grid, 128, 0, (cudaStream_t)stream>>>(which, tstp, nk, (const ConvHM *)G, (const ConvHM *)W,
                                                         (const ConvHM *)out, w, ntau, size1, (double)sig_b);
    CK(cudaGetLastError());
    return NESSI_OK;
}

extern "C" int nessi_gpu_gw_polarization_timestep(int tstp, int nk, const nessi_hm_ptrs *G, const nessi_hm_ptrs *P,
                                                  const double *w, int nt, int ntau, int size1, int sig_g,
                                                  void *stream) {
    NvtxRange nvtx_("nessi::gw_polarization_timestep");
    return gw_launch(1, tstp, nk, G, nullptr, P, w, nt, ntau, size1, sig_g, stream, "gw_polarization_timestep");
}

extern "C" int nessi_gpu_gw_sigma_timestep(int tstp, int nk, const nessi_hm_ptrs *G, const nessi_hm_ptrs *W,
                                           const nessi_hm_ptrs *S, const double *w, int nt, int ntau, int size1,
                                           void *stream) {
    NvtxRange nvtx_("nessi::gw_sigma_timestep");
    return gw_launch(2, tstp, nk, G, W, S, w, nt, ntau, size1, 1, stream, "gw_sigma_timestep");
}

// =====================================================================================
// The element-parallel path: incr_convolution, convolution_timestep_new, dyson_timestep_omp,
// vie2_timestep_omp on device-resident herm_matrix data (kernels_omp.cuh)
// =====================================================================================
namespace {
ConvHM omp_hm(const nessi_hm_ptrs &x) {
    ConvHM y;
    y.ret = (double2 *)x.ret; y.les = (double2 *)x.les; y.tv = (double2 *)x.tv; y.mat = (double2 *)x.mat;
    return y;
}

template <class Fn> int size_dispatch(int size1, Fn &&fn) {
    switch (size1) {
        case 1: return fn(std::integral_constant<int, 1>{});
        case 2: return fn(std::integral_constant<int, 2>{});
        case 3: return fn(std::integral_constant<int, 3>{});
        case 4: return fn(std::integral_constant<int, 4>{});
        case 5: return fn(std::integral_constant<int, 5>{});
        case 6: return fn(std::integral_constant<int, 6>{});
        case 7: return fn(std::integral_constant<int, 7>{});
        case 8: return fn(std::integral_constant<int, 8>{});
    }
    set_err("size1 %d unsupported", size1);
    return NESSI_ERR_ARG;
}

unsigned omp_grid(long items) { return (unsigned)std::min<long>(std::max<long>(1, (items + 127) / 128), 1024); }

// one incr_convolution component (0 mat, 1 ret, 2 tv, 3 les) over output indices [ob.lo, ob.hi)
template <int S> int incr_launch(const OmpBatch &ob, int which, int tstp, cudaStream_t st) {
    const long items = (long)(ob.hi - ob.lo) * S * S;
    if (items <= 0 || ob.count <= 0) return NESSI_OK;
    const dim3 grid(omp_grid(items), ob.count);
    if (which == 0) k_incr_mat<S><<<grid, 128, 0, st>>>(ob);
    else if (which == 1) k_incr_ret<S><<<grid, 128, 0, st>>>(ob, tstp);
    else if (which == 2) k_incr_tv<S><<<grid, 128, 0, st>>>(ob, tstp);
    else k_incr_les<S><<<grid, 128, 0, st>>>(ob, tstp);
    CK(cudaGetLastError());
    return NESSI_OK;
}

int omp_common_checks(const char *name, int tstp, int nt, int ntau, int size1, int solve_order, double beta, double h) {
    if (size1 < 1 || size1 > NESSI_MAXS || solve_order < 1 || solve_order > CNTR_KMAX || nt < solve_order ||
        ntau < solve_order || tstp < -1 || tstp > nt || !(beta > 0) || !(h > 0)) {
        set_err("%s: bad dimensions (tstp=%d nt=%d ntau=%d size1=%d k=%d)", name, tstp, nt, ntau, size1, solve_order);
        return NESSI_ERR_ARG;
    }
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) { set_err("%s: device index %d unsupported", name, dev); return NESSI_ERR_ARG; }
    return ensure_tables(dev);
}

// the arguments of an incr_convolution call, checked before anything is queued
int incr_check(const char *name, int which, int tstp, int count, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
               const nessi_hm_ptrs *Acc, const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau,
               int size1, int sig_a, int sig_b, int solve_order, double beta, double h) {
    if (count < 0 || (count > 0 && (!C || !A || !Acc || !B || !Bcc)) || (sig_a != 1 && sig_a != -1) ||
        (sig_b != 1 && sig_b != -1) || which < -1 || which > 3 || (which == 0 && tstp != -1) ||
        (which > 0 && tstp < 0)) {
        set_err("%s: bad arguments", name);
        return NESSI_ERR_ARG;
    }
    for (int i = 0; i < count; i++) {
        bool ok = B[i].mat && (tstp >= 0 || (A[i].mat && C[i].mat));
        const nessi_hm_ptrs *all[5] = {&C[i], &A[i], &Acc[i], &B[i], &Bcc[i]};
        if (tstp >= 0)
            for (const nessi_hm_ptrs *x : all) ok = ok && x->ret && x->les && x->tv;
        if (!ok) { set_err("%s: problem %d has a null pointer it needs", name, i); return NESSI_ERR_ARG; }
    }
    return omp_common_checks(name, tstp, nt, ntau, size1, solve_order, beta, h);
}

// incr_convolution over components `which` (-1: every component of tstp, mat for tstp = -1)
int incr_run(const char *name, int which, int tstp, const unsigned char *mask, int count, double2 alpha,
             const nessi_hm_ptrs *C, const nessi_hm_ptrs *A, const nessi_hm_ptrs *Acc, const void *const *ft,
             const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1, int sig_a, int sig_b,
             int solve_order, double beta, double h, void *stream) {
    CKR(incr_check(name, which, tstp, count, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h));
    cudaStream_t st = (cudaStream_t)stream;
    for (int i0 = 0; i0 < count; i0 += NESSI_OMP_MAXP) {
        OmpBatch ob;
        std::memset(&ob, 0, sizeof ob);
        ob.count = std::min(NESSI_OMP_MAXP, count - i0);
        for (int i = 0; i < ob.count; i++) {
            OmpProb &P = ob.p[i];
            P.C = P.Cin = omp_hm(C[i0 + i]); P.A = omp_hm(A[i0 + i]); P.Acc = omp_hm(Acc[i0 + i]);
            P.B = omp_hm(B[i0 + i]); P.Bcc = omp_hm(Bcc[i0 + i]);
            P.f = ft ? (const double2 *)ft[i0 + i] : nullptr;
        }
        ob.mask = mask; ob.alpha = alpha; ob.ntau = ntau; ob.sig_a = sig_a; ob.sig_b = sig_b; ob.k = solve_order;
        ob.h = h; ob.beta = beta; ob.out_mode = 0; ob.skip_tstp = 0;
        const int w0 = which >= 0 ? which : (tstp < 0 ? 0 : 1), w1 = which >= 0 ? which : (tstp < 0 ? 0 : 3);
        for (int w = w0; w <= w1; w++) {
            ob.lo = 0;
            ob.hi = (w == 0 || w == 2) ? ntau + 1 : tstp + 1;
            CKR(size_dispatch(size1, [&](auto sz) { return incr_launch<decltype(sz)::value>(ob, w, tstp, st); }));
        }
    }
    return NESSI_OK;
}
}  // namespace

extern "C" int nessi_gpu_incr_convolution_timestep(int tstp, int count, double alpha_re, double alpha_im,
                                                   const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                                   const nessi_hm_ptrs *Acc, const void *const *ft,
                                                   const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau,
                                                   int size1, int sig_a, int sig_b, int solve_order, double beta,
                                                   double h, void *stream) {
    NvtxRange nvtx_("nessi::incr_convolution");
    return incr_run("incr_convolution", -1, tstp, nullptr, count, cmk(alpha_re, alpha_im), C, A, Acc, ft, B, Bcc, nt,
                    ntau, size1, sig_a, sig_b, solve_order, beta, h, stream);
}

extern "C" int nessi_gpu_incr_convolution_component(int which, int tstp, const unsigned char *mask, int count,
                                                    double alpha_re, double alpha_im, const nessi_hm_ptrs *C,
                                                    const nessi_hm_ptrs *A, const nessi_hm_ptrs *Acc,
                                                    const void *const *ft, const nessi_hm_ptrs *B,
                                                    const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1, int sig_a,
                                                    int sig_b, int solve_order, double beta, double h, void *stream) {
    NvtxRange nvtx_("nessi::incr_convolution_component");
    if (which < 0) { set_err("incr_convolution_component: which = %d", which); return NESSI_ERR_ARG; }
    return incr_run("incr_convolution_component", which, tstp, mask, count, cmk(alpha_re, alpha_im), C, A, Acc, ft,
                    B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h, stream);
}

extern "C" int nessi_gpu_convolution_timestep_new(int tstp, int count, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                                  const nessi_hm_ptrs *Acc, const void *const *ft,
                                                  const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau,
                                                  int size1, int sig_a, int sig_b, int solve_order, double beta,
                                                  double h, void *stream) {
    NvtxRange nvtx_("nessi::convolution_timestep_new");
    CKR(incr_check("convolution_timestep_new", -1, tstp, count, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b,
                   solve_order, beta, h));
    // C.set_timestep_zero(tstp): ret row, tv row and les column of tstp are contiguous
    const long s2 = (long)size1 * size1, M = ntau + 1;
    cudaStream_t st = (cudaStream_t)stream;
    for (int i = 0; i < count; i++) {
        if (tstp < 0) {
            if (!C[i].mat) { set_err("convolution_timestep_new: problem %d has no mat", i); return NESSI_ERR_ARG; }
            CK(cudaMemsetAsync(C[i].mat, 0, (size_t)M * s2 * 16, st));
        } else {
            if (!C[i].ret || !C[i].tv || !C[i].les) {
                set_err("convolution_timestep_new: problem %d has a null pointer", i);
                return NESSI_ERR_ARG;
            }
            CK(cudaMemsetAsync((char *)C[i].ret + tri_h(tstp) * s2 * 16, 0, (size_t)(tstp + 1) * s2 * 16, st));
            CK(cudaMemsetAsync((char *)C[i].tv + (long)tstp * M * s2 * 16, 0, (size_t)M * s2 * 16, st));
            CK(cudaMemsetAsync((char *)C[i].les + tri_h(tstp) * s2 * 16, 0, (size_t)(tstp + 1) * s2 * 16, st));
        }
    }
    return incr_run("convolution_timestep_new", -1, tstp, nullptr, count, cmk(1.0, 0.0), C, A, Acc, ft, B, Bcc, nt,
                    ntau, size1, sig_a, sig_b, solve_order, beta, h, stream);
}

namespace {
template <int S> int dyson_omp_launch(int n, const OmpBatch &base, int ntau, int *status, cudaStream_t st) {
    const int k = base.k, M = ntau + 1, KS = k * S, s2 = S * S;
    const dim3 tb(128);
    auto grid = [&](long items) { return dim3(omp_grid(items), base.count); };
    // retarded: start block, the convolution for columns j < n-k (G^R(n, j) read as zero), solves
    {
        OmpBatch ob = base;  // C = B = Bcc = G, A = Acc = Sigma
        const size_t smem = (size_t)(2 * KS * KS + 2 * k * s2) * 16 + 16;
        CK(cudaFuncSetAttribute(k_omp_ret_start<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_omp_ret_start<S><<<base.count, 256, smem, st>>>(ob, n, status);
        CK(cudaGetLastError());
        ob.lo = 0; ob.hi = n - k; ob.out_mode = 2; ob.skip_tstp = 1;
        CKR(incr_launch<S>(ob, 1, n, st));
        k_omp_ret_solve<S><<<grid(n - k), tb, 0, st>>>(ob, n, status);
        CK(cudaGetLastError());
    }
    // left-mixing: the convolution (G^tv(n, .) read as zero), then the BDF solves
    {
        OmpBatch ob = base;
        ob.lo = 0; ob.hi = M; ob.out_mode = 2; ob.skip_tstp = 1;
        CKR(incr_launch<S>(ob, 2, n, st));
        k_omp_tv_solve<S><<<grid(M), tb, 0, st>>>(ob, n, status);
        CK(cudaGetLastError());
    }
    // lesser: rows j < n-k from the conjugate equation (n >= 2k+1), then rows n-k..n in sequence
    const bool full = n < 2 * k + 1;
    if (!full) {
        OmpBatch ob = base;  // [G * Sigma]^<: A = Acc = G, B = Bcc = Sigma
        for (int i = 0; i < ob.count; i++) {
            ob.p[i].A = ob.p[i].Acc = base.p[i].C;
            ob.p[i].B = ob.p[i].Bcc = base.p[i].A;
        }
        ob.lo = 0; ob.hi = n - k; ob.out_mode = 2; ob.skip_tstp = 1;
        CKR(incr_launch<S>(ob, 3, n, st));
        OmpBatch os = base;
        k_omp_les_solve<S><<<grid(n - k), tb, 0, st>>>(os, n, status);
        CK(cudaGetLastError());
    }
    {
        OmpBatch ob = base;  // A = Sigma, B = Bcc = G (the serial step's gles)
        const int nthr = 256, ngrp = nthr / s2;
        const size_t smem = (size_t)(ngrp * s2 + 2 * s2 + KS * KS + KS * S) * 16 + 16;
        k_omp_les_serial<S><<<base.count, nthr, smem, st>>>(ob, n, full ? 1 : 0, status);
        CK(cudaGetLastError());
    }
    return NESSI_OK;
}

template <int S> int vie2_omp_launch(int tstp, const OmpBatch &base, int ntau, int *status, cudaStream_t st) {
    const int M = ntau + 1;
    const dim3 tb(128);
    auto grid = [&](long items) { return dim3(omp_grid(items), base.count); };
    // base: C = G, Cin = Q, A = F, Acc = Fcc, B = Bcc = G, alpha = -1, Q as the base
    {
        OmpBatch ob = base;
        ob.lo = 0; ob.hi = tstp + 1;
        CKR(incr_launch<S>(ob, 1, tstp, st));
        k_omp_vie2_solve<S><<<grid(tstp + 1), tb, 0, st>>>(ob, tstp, 0, status);
        CK(cudaGetLastError());
    }
    {
        OmpBatch ob = base;
        ob.lo = 0; ob.hi = M;
        CKR(incr_launch<S>(ob, 2, tstp, st));
        k_omp_vie2_solve<S><<<grid(M), tb, 0, st>>>(ob, tstp, 1, status);
        CK(cudaGetLastError());
    }
    {
        // lesser: Q - G * Fcc with A = Acc = G, B = Fcc, Bcc = F; rows below tstp, then row tstp
        OmpBatch ob = base;
        for (int i = 0; i < ob.count; i++) {
            ob.p[i].A = ob.p[i].Acc = base.p[i].C;
            ob.p[i].B = base.p[i].Acc;
            ob.p[i].Bcc = base.p[i].A;
        }
        OmpBatch os = base;  // the solves read F^R(tstp, tstp) from A
        for (int part = 0; part < 2; part++) {
            ob.lo = os.lo = part ? tstp : 0;
            ob.hi = os.hi = part ? tstp + 1 : tstp;
            if (ob.hi <= ob.lo) continue;
            CKR(incr_launch<S>(ob, 3, tstp, st));
            k_omp_vie2_solve<S><<<grid(ob.hi - ob.lo), tb, 0, st>>>(os, tstp, 2, status);
            CK(cudaGetLastError());
        }
    }
    return NESSI_OK;
}
}  // namespace

extern "C" int nessi_gpu_dyson_timestep_omp(int n, int count, const nessi_hm_ptrs *G, const nessi_hm_ptrs *Sigma,
                                            const void *const *H, const double *mu, int nt, int ntau, int size1,
                                            int sig, int solve_order, double beta, double h, int *status,
                                            void *stream) {
    NvtxRange nvtx_("nessi::dyson_timestep_omp");
    if (count < 0 || (count > 0 && (!G || !Sigma || !H || !mu)) || (sig != 1 && sig != -1)) {
        set_err("dyson_timestep_omp: bad arguments");
        return NESSI_ERR_ARG;
    }
    if (n < solve_order + 1) {
        set_err("dyson_timestep_omp: n = %d must exceed SolveOrder = %d (dyson_start covers n <= k)", n, solve_order);
        return NESSI_ERR_ARG;
    }
    for (int i = 0; i < count; i++) {
        const nessi_hm_ptrs *all[2] = {&G[i], &Sigma[i]};
        bool ok = H[i] && G[i].mat;
        for (const nessi_hm_ptrs *x : all) ok = ok && x->ret && x->les && x->tv;
        if (!ok) { set_err("dyson_timestep_omp: problem %d has a null pointer it needs", i); return NESSI_ERR_ARG; }
    }
    CKR(omp_common_checks("dyson_timestep_omp", n, nt, ntau, size1, solve_order, beta, h));
    cudaStream_t st = (cudaStream_t)stream;
    for (int i0 = 0; i0 < count; i0 += NESSI_OMP_MAXP) {
        OmpBatch ob;
        std::memset(&ob, 0, sizeof ob);
        ob.count = std::min(NESSI_OMP_MAXP, count - i0);
        for (int i = 0; i < ob.count; i++) {
            OmpProb &P = ob.p[i];
            P.C = P.Cin = P.B = P.Bcc = omp_hm(G[i0 + i]);
            P.A = P.Acc = omp_hm(Sigma[i0 + i]);
            P.H = (const double2 *)H[i0 + i];
            P.mu = mu[i0 + i];
        }
        ob.alpha = cmk(1.0, 0.0); ob.ntau = ntau; ob.sig_a = sig; ob.sig_b = sig; ob.k = solve_order;
        ob.h = h; ob.beta = beta;
        CKR(size_dispatch(size1, [&](auto sz) { return dyson_omp_launch<decltype(sz)::value>(n, ob, ntau, status, st); }));
    }
    return NESSI_OK;
}

extern "C" int nessi_gpu_vie2_timestep_omp(int n, int count, const nessi_hm_ptrs *G, const nessi_hm_ptrs *F,
                                           const nessi_hm_ptrs *Fcc, const nessi_hm_ptrs *Q, int nt, int ntau,
                                           int size1, int sig, int solve_order, double beta, double h, int *status,
                                           void *stream) {
    NvtxRange nvtx_("nessi::vie2_timestep_omp");
    if (count < 0 || (count > 0 && (!G || !F || !Fcc || !Q)) || (sig != 1 && sig != -1)) {
        set_err("vie2_timestep_omp: bad arguments");
        return NESSI_ERR_ARG;
    }
    if (n < solve_order + 1) {
        set_err("vie2_timestep_omp: n = %d must exceed SolveOrder = %d (vie2_start / vie2_mat cover n <= k)", n,
                solve_order);
        return NESSI_ERR_ARG;
    }
    for (int i = 0; i < count; i++) {
        const nessi_hm_ptrs *all[4] = {&G[i], &F[i], &Fcc[i], &Q[i]};
        bool ok = G[i].mat;
        for (const nessi_hm_ptrs *x : all) ok = ok && x->ret && x->les && x->tv;
        if (!ok) { set_err("vie2_timestep_omp: problem %d has a null pointer it needs", i); return NESSI_ERR_ARG; }
    }
    CKR(omp_common_checks("vie2_timestep_omp", n, nt, ntau, size1, solve_order, beta, h));
    cudaStream_t st = (cudaStream_t)stream;
    for (int i0 = 0; i0 < count; i0 += NESSI_OMP_MAXP) {
        OmpBatch ob;
        std::memset(&ob, 0, sizeof ob);
        ob.count = std::min(NESSI_OMP_MAXP, count - i0);
        for (int i = 0; i < ob.count; i++) {
            OmpProb &P = ob.p[i];
            P.C = P.B = P.Bcc = omp_hm(G[i0 + i]);
            P.Cin = omp_hm(Q[i0 + i]);
            P.A = omp_hm(F[i0 + i]);
            P.Acc = omp_hm(Fcc[i0 + i]);
        }
        ob.alpha = cmk(-1.0, 0.0); ob.ntau = ntau; ob.sig_a = sig; ob.sig_b = sig; ob.k = solve_order;
        ob.h = h; ob.beta = beta; ob.out_mode = 1; ob.skip_tstp = 1;
        CKR(size_dispatch(size1, [&](auto sz) { return vie2_omp_launch<decltype(sz)::value>(n, ob, ntau, status, st); }));
    }
    return NESSI_OK;
}

// ---- the same on HOST herm_matrix data (single calls with libcntr's signatures) ------------
namespace {
// Device copies of host herm_matrix data and function arrays for one call; the output's time
// step comes back on success.  Every allocation is freed on every path.
struct HostMirror {
    int nt, ntau;
    long s2, M;
    std::vector<void *> owned;
    std::string err;
    HostMirror(int nt_, int ntau_, int size1) : nt(nt_), ntau(ntau_), s2((long)size1 * size1), M(ntau_ + 1) {}
    ~HostMirror() { for (void *q : owned) cudaFree(q); }
    int upload(const void *src, long count, void **dst) {
        *dst = nullptr;
        if (!src) return NESSI_OK;
        if (cudaMalloc(dst, (size_t)count * 16) != cudaSuccess) { set_err("cudaMalloc failed"); return NESSI_ERR_OOM; }
        owned.push_back(*dst);
        if (cudaMemcpy(*dst, src, (size_t)count * 16, cudaMemcpyHostToDevice) != cudaSuccess) {
            set_err("upload failed");
            return NESSI_ERR_CUDA;
        }
        return NESSI_OK;
    }
    int hm(const nessi_hm_ptrs *h, nessi_hm_ptrs *d) {
        const long tri = tri_h(nt + 1) * s2;
        CKR(upload(h->ret, tri, &d->ret));
        CKR(upload(h->les, tri, &d->les));
        CKR(upload(h->tv, (long)(nt + 1) * M * s2, &d->tv));
        return upload(h->mat, M * s2, &d->mat);
    }
    // time step n of the device herm_matrix d back into the host one (mat for n = -1)
    int download_step(int n, const nessi_hm_ptrs *h, const nessi_hm_ptrs &d) {
        if (cudaDeviceSynchronize() != cudaSuccess) { set_err("device step failed"); return NESSI_ERR_CUDA; }
        auto back = [&](void *hp, const void *dp, long off, long cnt) {
            if (!hp || !dp) return cudaSuccess;
            return cudaMemcpy((char *)hp + off * 16, (const char *)dp + off * 16, (size_t)cnt * 16, cudaMemcpyDeviceToHost);
        };
        cudaError_t e;
        if (n < 0) {
            e = back(h->mat, d.mat, 0, M * s2);
        } else {
            e = back(h->ret, d.ret, tri_h(n) * s2, (long)(n + 1) * s2);
            if (e == cudaSuccess) e = back(h->tv, d.tv, (long)n * M * s2, M * s2);
            if (e == cudaSuccess) e = back(h->les, d.les, tri_h(n) * s2, (long)(n + 1) * s2);
        }
        if (e != cudaSuccess) { set_err("download failed"); return NESSI_ERR_CUDA; }
        return NESSI_OK;
    }
};

int device_status(int *d_status) {
    int hs = 0;
    if (cudaMemcpy(&hs, d_status, sizeof hs, cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_err("status read failed");
        return NESSI_ERR_CUDA;
    }
    if (hs) { set_err("a step matrix is singular"); return NESSI_ERR_SINGULAR; }
    return NESSI_OK;
}
}  // namespace

extern "C" int nessi_gpu_incr_convolution_timestep_host(int tstp, double alpha_re, double alpha_im,
                                                        const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                                        const nessi_hm_ptrs *Acc, const void *ft,
                                                        const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt,
                                                        int ntau, int size1, int sig_a, int sig_b, int solve_order,
                                                        double beta, double h) {
    if (!C || !A || !Acc || !B || !Bcc || nt < 0 || ntau < 0 || size1 < 1 || size1 > NESSI_MAXS || tstp < -1 ||
        tstp > nt) {
        set_err("incr_convolution_timestep_host: bad arguments");
        return NESSI_ERR_ARG;
    }
    CK(cudaSetDevice(g_device));
    HostMirror hm(nt, ntau, size1);
    nessi_hm_ptrs d[5];
    const nessi_hm_ptrs *hs[5] = {C, A, Acc, B, Bcc};
    for (int i = 0; i < 5; i++) CKR(hm.hm(hs[i], &d[i]));
    void *dft = nullptr;
    CKR(hm.upload(ft, (long)(nt + 2) * size1 * size1, &dft));
    const void *fts[1] = {dft};
    CKR(nessi_gpu_incr_convolution_timestep(tstp, 1, alpha_re, alpha_im, &d[0], &d[1], &d[2], ft ? fts : nullptr, &d[3],
                                            &d[4], nt, ntau, size1, sig_a, sig_b, solve_order, beta, h, nullptr));
    return hm.download_step(tstp, C, d[0]);
}

extern "C" int nessi_gpu_dyson_timestep_omp_host(int n, const nessi_hm_ptrs *G, const nessi_hm_ptrs *Sigma,
                                                 const void *H, double mu, int nt, int ntau, int size1, int sig,
                                                 int solve_order, double beta, double h) {
    if (!G || !Sigma || !H || nt < 0 || ntau < 0 || size1 < 1 || size1 > NESSI_MAXS) {
        set_err("dyson_timestep_omp_host: bad arguments");
        return NESSI_ERR_ARG;
    }
    if (n < solve_order + 1 || n > nt) {
        set_err("dyson_timestep_omp_host: n = %d outside SolveOrder+1..nt", n);
        return NESSI_ERR_ARG;
    }
    CK(cudaSetDevice(g_device));
    HostMirror hm(nt, ntau, size1);
    nessi_hm_ptrs dG, dS;
    CKR(hm.hm(G, &dG));
    CKR(hm.hm(Sigma, &dS));
    void *dH = nullptr, *dst = nullptr;
    CKR(hm.upload(H, (long)(nt + 2) * size1 * size1, &dH));
    if (cudaMalloc(&dst, 16) != cudaSuccess) { set_err("cudaMalloc failed"); return NESSI_ERR_OOM; }
    hm.owned.push_back(dst);
    CK(cudaMemset(dst, 0, 16));
    const void *Hs[1] = {dH};
    CKR(nessi_gpu_dyson_timestep_omp(n, 1, &dG, &dS, Hs, &mu, nt, ntau, size1, sig, solve_order, beta, h, (int *)dst,
                                     nullptr));
    CKR(hm.download_step(n, G, dG));
    return device_status((int *)dst);
}

extern "C" int nessi_gpu_vie2_timestep_omp_host(int n, const nessi_hm_ptrs *G, const nessi_hm_ptrs *F,
                                                const nessi_hm_ptrs *Fcc, const nessi_hm_ptrs *Q, int nt, int ntau,
                                                int size1, int sig, int solve_order, double beta, double h) {
    if (!G || !F || !Fcc || !Q || nt < 0 || ntau < 0 || size1 < 1 || size1 > NESSI_MAXS) {
        set_err("vie2_timestep_omp_host: bad arguments");
        return NESSI_ERR_ARG;
    }
    if (n < solve_order + 1 || n > nt) {
        set_err("vie2_timestep_omp_host: n = %d outside SolveOrder+1..nt", n);
        return NESSI_ERR_ARG;
    }
    CK(cudaSetDevice(g_device));
    HostMirror hm(nt, ntau, size1);
    nessi_hm_ptrs d[4];
    const nessi_hm_ptrs *hs[4] = {G, F, Fcc, Q};
    for (int i = 0; i < 4; i++) CKR(hm.hm(hs[i], &d[i]));
    void *dst = nullptr;
    if (cudaMalloc(&dst, 16) != cudaSuccess) { set_err("cudaMalloc failed"); return NESSI_ERR_OOM; }
    hm.owned.push_back(dst);
    CK(cudaMemset(dst, 0, 16));
    CKR(nessi_gpu_vie2_timestep_omp(n, 1, &d[0], &d[1], &d[2], &d[3], nt, ntau, size1, sig, solve_order, beta, h,
                                    (int *)dst, nullptr));
    CKR(hm.download_step(n, G, d[0]));
    return device_status((int *)dst);
}
