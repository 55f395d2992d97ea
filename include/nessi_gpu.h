/* nessi_gpu.h - C ABI of libnessi_gpu.so, the B200 implementation of libcntr's
 * Kadanoff-Baym time-stepping hot path.
 *
 * The reference has no plugin system: its boundary is the C++ template API of namespace
 * cntr (libcntr/cntr/cntr_dyson_decl.hpp, cntr_vie2_decl.hpp, cntr_convolution_decl.hpp),
 * instantiated for double in libcntr.so.  Each entry point below names the reference
 * interface it replaces.  All functions return 0 on success or one of NESSI_ERR_*;
 * nessi_gpu_last_error() gives a one-line description of the last failure.
 *
 * Data are exchanged in libcntr's herm_matrix<double> layout
 * (libcntr/cntr/cntr_herm_matrix_impl.hpp:457-477), so a caller passes
 * G.retptr(0,0), G.lesptr(0,0), G.tvptr(0,0) and G.matptr(0) unchanged:
 *   ret(t,t') [t'<=t] at (t(t+1)/2+t') s^2,  les(t,t') [t<=t'] at (t'(t'+1)/2+t) s^2,
 *   tv(t,tau) at (t(ntau+1)+tau) s^2,        mat(tau) at tau s^2,
 * every element a row-major s x s block of complex<double> (re, im interleaved).
 * cntr::function<double> H is passed as H.ptr(-1): (nt+2) blocks, t = -1 first
 * (libcntr/cntr/cntr_function_decl.hpp:45).
 *
 * A batch holds many problems ("k-points") that are advanced together on one GPU.
 * Problems with the same sigma_group share one self-energy Sigma (a local or
 * k-independent Sigma, as in the reference's lattice drivers, examples/programs/gw.cpp:386-420);
 * all problems of a group have the same size1, ntau, sig, beta, h and solve order.
 * Calls on one batch are stream-ordered on the batch's stream and must come from one host
 * thread at a time.
 */
#ifndef NESSI_GPU_H
#define NESSI_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define NESSI_OK 0
#define NESSI_ERR_ARG 1       /* bad argument or state */
#define NESSI_ERR_OOM 2       /* device allocation failed */
#define NESSI_ERR_CUDA 3      /* CUDA runtime error */
#define NESSI_ERR_SINGULAR 4  /* a step matrix had a zero pivot */
#define NESSI_ERR_TIMEOUT 5   /* a bounded device wait gave up */

#define NESSI_PREC_FP64 0     /* every sum and solve in complex<double> */
#define NESSI_PREC_MIXED 1    /* history sums from an FP32 copy of G^tv, FP64 solves */

typedef struct nessi_batch nessi_batch;

/* One problem: the dimensions of its herm_matrix G and of the Dyson equation
 * [i d/dt + mu - H(t)] G - Sigma * G = delta (cntr_dyson_decl.hpp:92). */
typedef struct {
    int nt, ntau, size1, sig; /* herm_matrix<double>(nt, ntau, size1, sig) */
    int solve_order;          /* SolveOrder k, 1..5 (MAX_SOLVE_ORDER, cntr_global_settings.hpp:37) */
    int sigma_group;          /* problems with equal group share one Sigma */
    double beta, h, mu;
} nessi_problem_desc;

/* Select the CUDA device used by later batches; replaces nothing (libcntr is CPU-only). */
int nessi_gpu_init(int device);
/* End of use: NESSI_ERR_ARG while batches are alive; otherwise waits for the devices used and
 * forgets the per-device state (the next init or batch_create sets it up again).  The CUDA
 * context is left alone, so a host program that also uses the device keeps it. */
int nessi_gpu_finalize(void);
const char *nessi_gpu_last_error(void);

/* Allocate device storage for `count` problems.  precision is NESSI_PREC_*. */
int nessi_gpu_batch_create(nessi_batch **out, const nessi_problem_desc *desc, int count, int precision);
int nessi_gpu_batch_destroy(nessi_batch *b);
/* Bytes of device memory held by the batch. */
int nessi_gpu_batch_bytes(nessi_batch *b, long long *bytes);

/* Copy a whole herm_matrix G of problem p (host, libcntr layout) to / from the device.
 * Any pointer may be NULL to skip that component.  Replaces direct access to
 * herm_matrix<T>::ret_/les_/tv_/mat_ (cntr_herm_matrix_decl.hpp:79-93). */
int nessi_gpu_set_G(nessi_batch *b, int p, const void *ret, const void *les, const void *tv, const void *mat);
int nessi_gpu_get_G(nessi_batch *b, int p, void *ret, void *les, void *tv, void *mat);
/* One time step of G as a herm_matrix_timestep slice [ret(n,0..n) | tv(n,0..ntau) |
 * les(0..n,n)] (cntr_herm_matrix_timestep_decl.hpp:67-75; herm_matrix::get_timestep,
 * cntr_herm_matrix_impl.hpp:2156).  tstp = -1 gives mat. */
int nessi_gpu_get_timestep(nessi_batch *b, int p, int tstp, void *slice);
int nessi_gpu_set_timestep(nessi_batch *b, int p, int tstp, const void *slice);
/* H(t) of problem p as cntr::function<double> data, (nt+2) s^2 complex. */
int nessi_gpu_set_H(nessi_batch *b, int p, const void *H);

/* The shared Sigma of a group: full herm_matrix, or one time step slice
 * (herm_matrix::set_timestep, cntr_herm_matrix_impl.hpp:2098). */
int nessi_gpu_set_sigma(nessi_batch *b, int group, const void *ret, const void *les, const void *tv,
                        const void *mat);
int nessi_gpu_set_sigma_timestep(nessi_batch *b, int group, int tstp, const void *slice);

/* cntr::dyson_mat(G, mu, H, Sigma, beta, SolveOrder) with the default CNTR_MAT_FIXPOINT
 * method and force_hermitian (cntr_dyson_decl.hpp:78, cntr_dyson_impl.hpp:1393-1450): G^mat of
 * every problem from H(-1) and the group's Sigma^mat.  ntau must be even. */
int nessi_gpu_dyson_mat(nessi_batch *b);
/* The same with libcntr's method argument (cntr_dyson_impl.hpp:1393-1450, dispatch :1209-1230):
 * 0 = CNTR_MAT_FOURIER (dyson_mat_fourier_dispatch, :356-446: 21 oversampling copies of the
 * Matsubara frequencies, first-order tail), 1 = CNTR_MAT_CG (dyson_mat_steep_dispatch, :519-540:
 * conjugate gradients from a Fourier start, 40 iterations, tol 1e-12), 2 = CNTR_MAT_FIXPOINT;
 * force_hermitian as libcntr's.  Other methods: NESSI_ERR_ARG. */
int nessi_gpu_dyson_mat_method(nessi_batch *b, int method, int force_hermitian);
/* cntr::dyson_start(G, mu, H, Sigma, beta, h, SolveOrder) (cntr_dyson_decl.hpp:88,
 * cntr_dyson_impl.hpp:1502-1535): time steps 0..k of every problem from G^mat. */
int nessi_gpu_dyson_start(nessi_batch *b);

/* cntr::dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder) for every problem of the
 * batch with nt >= n (cntr_dyson_decl.hpp:92, cntr_dyson_impl.hpp:1618-1648).  n > k.
 * G must hold time steps 0..n-1 and mat; Sigma and H must hold 0..n. */
int nessi_gpu_dyson_timestep(nessi_batch *b, int n);

/* ---- VIE2: [1 + F] G = Q (cntr_vie2_decl.hpp:63-90) ---------------------------------------
 * A group becomes a VIE2 group when its kernel F is set: F (and its hermitian-conjugate partner
 * Fcc, which the retarded and lesser parts need where F is not hermitian) are shared by the
 * group, Q is per problem.  dyson_* calls act on Dyson groups only and vie2_* calls on VIE2
 * groups only, so one batch may hold both kinds.  G^mat of a VIE2 problem comes from
 * nessi_gpu_vie2_mat or from the caller (set_G / set_timestep(-1)). */
/* F and Fcc of a group (herm_matrix layout; Fcc's ret and les only). */
int nessi_gpu_set_F(nessi_batch *b, int group, const void *ret, const void *les, const void *tv, const void *mat,
                    const void *cc_ret, const void *cc_les);
/* One time step of F and Fcc (herm_matrix_timestep slices; tstp = -1: F^mat, cc_slice unused). */
int nessi_gpu_set_F_timestep(nessi_batch *b, int group, int tstp, const void *slice, const void *cc_slice);
/* The source term Q of problem p, whole or one time step. */
int nessi_gpu_set_Q(nessi_batch *b, int p, const void *ret, const void *les, const void *tv, const void *mat);
int nessi_gpu_set_Q_timestep(nessi_batch *b, int p, int tstp, const void *slice);
/* cntr::vie2_mat(G, F, Fcc, Q, beta, SolveOrder) with the default fixpoint method
 * (cntr_vie2_decl.hpp:63, cntr_vie2_impl.hpp:460-484, 1091-1160): G^mat of every VIE2 problem
 * from the group's F^mat and the problem's Q^mat.  ntau must be even. */
int nessi_gpu_vie2_mat(nessi_batch *b);
/* The same with libcntr's method argument (cntr_vie2_impl.hpp:1229-1250): 0 = CNTR_MAT_FOURIER
 * (vie2_mat_fourier with 20 oversampling copies, no corrections), 1 = CNTR_MAT_CG (vie2_mat_steep,
 * :486-600: a Fourier start, then at most 40 conjugate-gradient iterations to 1e-12; needs the
 * group's Fcc^mat from nessi_gpu_set_Fcc_mat, NESSI_ERR_ARG without it), 2 = CNTR_MAT_FIXPOINT. */
int nessi_gpu_vie2_mat_method(nessi_batch *b, int method);
/* Fcc^mat of a VIE2 group (the Matsubara part of the Fcc argument of cntr::vie2_mat,
 * cntr_vie2_decl.hpp:63), host pointer, (ntau+1) s^2; read by the steepest-descent vie2_mat only. */
int nessi_gpu_set_Fcc_mat(nessi_batch *b, int group, const void *cc_mat);
/* cntr::vie2_start(G, F, Fcc, Q, SolveOrder, beta, h) (cntr_vie2_decl.hpp:67,
 * cntr_vie2_impl.hpp:1338-1420): time steps 0..k of every VIE2 problem from G^mat. */
int nessi_gpu_vie2_start(nessi_batch *b);
/* cntr::vie2_timestep(n, G, F, Fcc, Q, SolveOrder, beta, h) (cntr_vie2_decl.hpp:72,
 * cntr_vie2_impl.hpp:1505-1560) for every VIE2 problem with nt >= n; n > k. */
int nessi_gpu_vie2_timestep(nessi_batch *b, int n);

/* Run the batch's work on the caller's cudaStream_t (NULL: a private stream again).
 * libcntr has no streams; this lets a caller order the batch with its own work. */
int nessi_gpu_set_stream(nessi_batch *b, void *stream);

/* Kernel timing with CUDA events on the batch stream.  Kernel ids: */
#define NESSI_KERNEL_PREP 0          /* step-matrix inverses, tv coefficients, dense Sigma copies */
#define NESSI_KERNEL_RET 1           /* G^R(n, .) Volterra recursion */
#define NESSI_KERNEL_TV 2            /* G^tv(n, .) history stream + solve */
#define NESSI_KERNEL_LES_OPERANDS 3  /* operands of the Sigma-shared products */
#define NESSI_KERNEL_GEMM 4          /* K_n G^mat, tv*vt and les*adv products (k_zgemm, FP64 tensor cores) */
#define NESSI_KERNEL_LES 5           /* G^<(., n) Volterra recursion */
#define NESSI_KERNEL_MATOP 6         /* Matsubara operator K_n of the tv row */
#define NESSI_KERNEL_LATTICE 7       /* predictor, G_loc and Sigma_2B of the lattice driver */
#define NESSI_KERNEL_COUNT 8
/* Turn timing on/off (resets counters).  No reference counterpart. */
int nessi_gpu_set_profiling(nessi_batch *b, int on);
/* Total device time (ms), launches and algorithmic bytes recorded for one kernel id since the
 * last read (flops for GEMM, RET and LES: 8 per complex multiply-add); resets that counter.
 * No reference counterpart. */
int nessi_gpu_read_profile(nessi_batch *b, int kernel, double *ms, long long *launches, double *bytes);

/* dyson_mat (fixpoint method) for ONE problem, allocating nothing.  No counterpart in the
 * reference.  It is meant for callers that cannot let a library call cudaMalloc: applications
 * whose device memory is owned by another allocator (a framework's memory pool, an arena sized
 * at start-up), or that must not take the device-wide synchronisation a cudaMalloc / cudaFree can
 * bring.  Every input and output is a device pointer owned by the caller:
 *   H          cntr::function data starting at H(-1) (at least one size1 x size1 block)
 *   sigma_mat  Sigma^mat, (ntau+1) blocks;   gmat  G^mat, (ntau+1) blocks, written
 * The work is queued on `stream` (a cudaStream_t, NULL = legacy default stream) and the call
 * returns without waiting.  Scratch is a fixed device array of 131072 complex<double>
 * (2 MiB) that every GPU loading the library holds until exit; sizes with
 * 6(ntau+1)size1^2 + 2 ntau size1^2 above that limit are rejected with NESSI_ERR_ARG, and so is an
 * ntau whose 2 ntau twiddle factors (32 ntau bytes of shared memory per block) exceed the
 * device's per-block shared-memory limit (about ntau > 7000 on a B200).  The first call on a
 * device looks up the array's device address and uploads the integration tables (under a lock,
 * waiting for the upload), so make that first call before any stream capture.  All calls share
 * the one array: calls whose work overlaps on the GPU race.  Every scratch element is written
 * before it is read, so nothing left by an earlier call leaks into a result.  ntau must be even. */
int nessi_gpu_dyson_mat_noalloc(int ntau, int size1, int sig, int solve_order, double beta, double mu, const void *H,
                                const void *sigma_mat, void *gmat, void *stream);

/* ---- self-consistent lattice (local self-energy recomputed from the k-average) --------
 * The lattice drivers of the reference (examples/programs/hubbard_chain_2b.cpp:245-324,
 * gw.cpp:386-420) gather every k-point's time step, form the local G_loc = (1/Nk) sum_k G_k,
 * recompute the local self-energy from it and solve the Dyson equation of every k-point again,
 * a few times per step.  Here a sigma_group is the set of k-points, its shared Sigma is the
 * local self-energy, and all of it stays on the device. */

/* Diagonal local interaction U(t) of a group, (nt+2) x size1 complex values, t = -1 first
 * (the diagonal of the cntr::function U of hubbard_chain_2b.cpp:170; U(-1) is the value on the
 * Matsubara branch).  Enables the Sigma_2B functions for the group. */
int nessi_gpu_set_U(nessi_batch *b, int group, const void *U);
/* cntr::extrapolate_timestep(n, G, SolveOrder) (cntr_utilities_decl.hpp:23,
 * cntr_utilities_impl.hpp:22-130) for every problem with nt > n: polynomial extrapolation of
 * time step n+1 from steps n-k..n.  n >= k. */
int nessi_gpu_extrapolate_timestep(nessi_batch *b, int n);
/* G_loc(tstp) = (1/P) sum_p G_p(tstp) over the P problems of the group that reach tstp
 * (the k-sum of gw_kpoints_impl.cpp:139-180); tstp = -1 averages G^mat. */
int nessi_gpu_gloc_timestep(nessi_batch *b, int group, int tstp);
/* Sigma(tstp) = Sigma_2B[G_loc, U](tstp) of the group (hubbard_chain_selfen_impl.cpp:63-75:
 * Polarization -> U(t) Pol U(t') -> Bubble2, cntr_bubble_impl.hpp:33-150), written into the
 * group's Sigma; tstp = -1 gives Sigma^mat. */
int nessi_gpu_sigma_2b_timestep(nessi_batch *b, int group, int tstp);
/* Download G_loc / Sigma of a group (libcntr layout; NULL skips a component). */
int nessi_gpu_get_gloc(nessi_batch *b, int group, void *ret, void *les, void *tv, void *mat);
int nessi_gpu_get_sigma(nessi_batch *b, int group, void *ret, void *les, void *tv, void *mat);
/* Device addresses of the group's G_loc (libcntr layout: ret and les packed triangles,
 * tv ((t (ntau+1) + tau) s^2 + e), mat), valid until the batch is destroyed.  For k-points
 * sharded over processes: each process averages its own problems with nessi_gpu_gloc_timestep,
 * and the processes sum the weighted time-step slices in place (an all-reduce over NCCL), which
 * replaces the MPI_Allgatherv of the k-slices in gw_selfene_impl.cpp:18-28 /
 * cntr_distributed_array_impl.hpp:370-399.  Launches nothing; NULL skips a component. */
int nessi_gpu_gloc_device(nessi_batch *b, int group, void **ret, void **les, void **tv, void **mat);
/* Bootstrap (hubbard_chain_2b.cpp:245-290 with G -> G_loc): iterate
 *   Sigma(0..k) = Sigma_2B[G_loc];  dyson_start of every problem;  G_loc(0..k)
 * until sum_t distance_norm2(t) between successive G_loc is below tol after more than 3
 * iterations, or max_iter+1 iterations.  G must hold mat and an initial guess of steps 0..k. */
int nessi_gpu_lattice_2b_start(nessi_batch *b, int max_iter, double tol, int *iters, double *err);
/* One time step n > k (hubbard_chain_2b.cpp:306-324 with G -> G_loc): predictor
 * extrapolate_timestep(n-1), then corrector_steps x [G_loc(n), Sigma_2B(n), dyson_timestep(n)],
 * then G_loc(n) of the final G. */
int nessi_gpu_lattice_2b_timestep(nessi_batch *b, int n, int corrector_steps);

/* ---- convolution on device-resident herm_matrix data ----------------------------------------
 * cntr::convolution_timestep(n, C, A, Acc, B, Bcc, beta, h, SolveOrder)
 * (cntr_convolution_decl.hpp:61, cntr_convolution_impl.hpp:1582-1803): time step n of C = A * B,
 * for `count` independent problems at once; n = -1 gives cntr::convolution_matsubara
 * (C^mat = A^mat * B^mat, :560-605).  Every pointer is a caller-owned DEVICE pointer to a
 * herm_matrix component in libcntr's layout (tv as (t(ntau+1)+tau) s^2, not the batch's planes);
 * all problems have the same nt, ntau, size1.  Acc and Bcc are the hermitian-conjugate partners
 * (pass A and B again for hermitian functions).  Writes C's time step n only; queued on `stream`
 * (NULL = legacy default stream), the call returns without waiting and allocates nothing. */
typedef struct {
    void *ret, *les, *tv, *mat;
} nessi_hm_ptrs;
int nessi_gpu_convolution_timestep(int n, int count, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                   const nessi_hm_ptrs *Acc, const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc,
                                   int nt, int ntau, int size1, int sig_a, int sig_b, int solve_order, double beta,
                                   double h, void *stream);

/* The same on HOST herm_matrix data (libcntr layout): copies A, Acc, B, Bcc and C to the device,
 * computes time step n and writes C's time step n back; allocates and frees device memory and
 * waits for completion.  For single calls with libcntr's signature (cntr_gpu.hpp). */
int nessi_gpu_convolution_timestep_host(int n, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                        const nessi_hm_ptrs *Acc, const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc,
                                        int nt, int ntau, int size1, int sig_a, int sig_b, int solve_order,
                                        double beta, double h);

/* cntr::convolution(C, A, Acc, B, Bcc, beta, h, SolveOrder) (cntr_convolution_decl.hpp:66-68,
 * cntr_convolution_impl.hpp:1805-1812, 3170-3177 without ft): C = A * B at every time step,
 * convolution_matsubara then n = 0..nt, on HOST herm_matrix data.  The operands are copied to the
 * device once, all steps run there, and all of C comes back. */
int nessi_gpu_convolution_host(const nessi_hm_ptrs *C, const nessi_hm_ptrs *A, const nessi_hm_ptrs *Acc,
                               const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1,
                               int sig_a, int sig_b, int solve_order, double beta, double h);

/* ---- the element-parallel path (the routines of libcntr's OpenMP solvers) ---------------------
 * Same data conventions as nessi_gpu_convolution_timestep: caller-owned DEVICE pointers in
 * libcntr's layout, `count` independent problems of equal shape, queued on `stream`, nothing
 * allocated.  `ft` is NULL or a host array of `count` device pointers to cntr::function data
 * (F(-1) first, (nt+2) blocks of s^2; a NULL entry means no function).
 *
 * incr_convolution(tstp, alpha, C, A, Acc, f0, ft, B, Bcc, I, beta, h)
 * (cntr_convolution_impl.hpp:4786-4807; components :4164-4760): C(tstp) += alpha [A * F * B](tstp),
 * every component of time step tstp (mat for tstp = -1), with the reference's per-element
 * quadrature (the tau integral of the lesser part always end-corrected). */
int nessi_gpu_incr_convolution_timestep(int tstp, int count, double alpha_re, double alpha_im, const nessi_hm_ptrs *C,
                                        const nessi_hm_ptrs *A, const nessi_hm_ptrs *Acc, const void *const *ft,
                                        const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1,
                                        int sig_a, int sig_b, int solve_order, double beta, double h, void *stream);

/* One component of incr_convolution: which = 0 incr_convolution_mat (:4164, tstp = -1), 1 _ret
 * (:4243), 2 _tv (:4396), 3 _les (:4539), for the output indices whose byte in the DEVICE array
 * `mask` is nonzero (ntau+1 entries for mat and tv, tstp+1 for ret and les; NULL = all), as the
 * reference's masks select them. */
int nessi_gpu_incr_convolution_component(int which, int tstp, const unsigned char *mask, int count, double alpha_re,
                                         double alpha_im, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                         const nessi_hm_ptrs *Acc, const void *const *ft, const nessi_hm_ptrs *B,
                                         const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1, int sig_a, int sig_b,
                                         int solve_order, double beta, double h, void *stream);

/* convolution_timestep_new(tstp, C, A, Acc, [ft,] B, Bcc, I, beta, h) (cntr_convolution_impl.hpp:4811-4976)
 * and convolution_timestep_omp (:5596-5812), which computes the same elements over threads:
 * C's time step tstp zeroed, then incr_convolution with alpha = 1. */
int nessi_gpu_convolution_timestep_new(int tstp, int count, const nessi_hm_ptrs *C, const nessi_hm_ptrs *A,
                                       const nessi_hm_ptrs *Acc, const void *const *ft, const nessi_hm_ptrs *B,
                                       const nessi_hm_ptrs *Bcc, int nt, int ntau, int size1, int sig_a, int sig_b,
                                       int solve_order, double beta, double h, void *stream);

/* cntr::dyson_timestep_omp(omp_num_threads, n, G, mu, H, Sigma, beta, h, SolveOrder)
 * (cntr_dyson_omp_impl.hpp:37-605): the OpenMP solver's discretization, every element of the
 * step a GPU thread: G^R(n, j) and, for n >= 2k+1, G^<(j, n) for j < n-k from the equation in
 * the other time argument (BD(k+1) derivatives), the k x k start block and the last k+1 lesser
 * rows as the serial step; G^tv as the serial step.  Not the serial dyson_timestep's
 * discretization: when G's mat and steps 0..k solve the same equation (dyson_mat, dyson_start)
 * the two agree to the discretization error; from a start that does not, they can differ by far
 * more, since the two time arguments' equations agree only for a solution.  H[i] is a device
 * pointer to problem i's
 * cntr::function H (H(-1) first), mu[i] its chemical potential (host array); requires
 * SolveOrder + 1 <= n.  If `status` (a DEVICE int) is not NULL it is set to 1 when a step matrix
 * is singular.  No counterpart of the thread count: the device decides. */
int nessi_gpu_dyson_timestep_omp(int n, int count, const nessi_hm_ptrs *G, const nessi_hm_ptrs *Sigma,
                                 const void *const *H, const double *mu, int nt, int ntau, int size1, int sig,
                                 int solve_order, double beta, double h, int *status, void *stream);

/* cntr::vie2_timestep_omp(omp_num_threads, tstp, G, F, Fcc, Q, beta, h, SolveOrder)
 * (cntr_vie2_impl.hpp:1851-2190) for tstp > SolveOrder: [1 + F] G = Q with every element of the
 * time step independent (the reference's vie2_timestep_omp_dispatch); Q is not modified.  The
 * reference dispatches tstp = -1 to vie2_mat and tstp <= SolveOrder to vie2_start of order tstp:
 * use nessi_gpu_vie2_mat / nessi_gpu_vie2_start (the C++ front end does).  `status` as above. */
int nessi_gpu_vie2_timestep_omp(int n, int count, const nessi_hm_ptrs *G, const nessi_hm_ptrs *F,
                                const nessi_hm_ptrs *Fcc, const nessi_hm_ptrs *Q, int nt, int ntau, int size1, int sig,
                                int solve_order, double beta, double h, int *status, void *stream);

/* The three above on HOST herm_matrix data (libcntr layout), for single calls with libcntr's
 * signatures (cntr_gpu.hpp): the operands (whole herm_matrix objects; ft and H as cntr::function
 * data, F(-1) first) are copied to the device, the step is computed there and the output's time
 * step (C's for incr_convolution, G's for the solvers; mat for tstp = -1) is copied back.
 * Allocates and frees device memory and waits; NESSI_ERR_SINGULAR for a singular step matrix. */
int nessi_gpu_incr_convolution_timestep_host(int tstp, double alpha_re, double alpha_im, const nessi_hm_ptrs *C,
                                             const nessi_hm_ptrs *A, const nessi_hm_ptrs *Acc, const void *ft,
                                             const nessi_hm_ptrs *B, const nessi_hm_ptrs *Bcc, int nt, int ntau,
                                             int size1, int sig_a, int sig_b, int solve_order, double beta, double h);
int nessi_gpu_dyson_timestep_omp_host(int n, const nessi_hm_ptrs *G, const nessi_hm_ptrs *Sigma, const void *H,
                                      double mu, int nt, int ntau, int size1, int sig, int solve_order, double beta,
                                      double h);
int nessi_gpu_vie2_timestep_omp_host(int n, const nessi_hm_ptrs *G, const nessi_hm_ptrs *F, const nessi_hm_ptrs *Fcc,
                                     const nessi_hm_ptrs *Q, int nt, int ntau, int size1, int sig, int solve_order,
                                     double beta, double h);

/* cntr::distance_norm2(tstp, g1, g2) (cntr_utilities_decl.hpp, cntr_utilities_impl.hpp:607-650) between two
 * herm_matrix held on the device (libcntr layout, caller-owned device pointers, tv as
 * (t(ntau+1)+tau) s^2): the sum over the elements of time step tstp (ret row, tv row, les column;
 * mat for tstp = -1) of the Frobenius norm of g1 - g2, written to the device double *out.  The
 * reference's convergence measure of self-consistent loops, computed where the data are; queued
 * on `stream` (NULL = legacy default stream), allocates nothing. */
int nessi_gpu_distance_norm2(int tstp, const nessi_hm_ptrs *g1, const nessi_hm_ptrs *g2, int nt, int ntau, int size1,
                             double *out, void *stream);

/* The GW self-energy diagrams of the momentum-resolved example
 * (examples/programs/gw_selfene_impl.cpp:114-153) at time step tstp, for all nk momenta of a 1-d
 * grid k_i = (i - nk/2) 2 pi / nk (gw_latt_impl.cpp:46-51) in one launch, element by element:
 *   polarisation  P_q = -sum_k w_k Bubble1(G_{k-q}, G_k)   (get_Polarization_Bubble)
 *   self-energy   Sigma_k = sum_q w_q Bubble2(G_{k-q}, W_q)  (sigma_GW)
 * with libcntr's bubbles (cntr_bubble_impl.hpp:17-330).  G, W, P, S and w are DEVICE arrays of nk
 * entries (herm_matrix pointers in libcntr's layout, tv as (t(ntau+1)+tau) s^2; weights); sig_g
 * is G's statistics.  tstp = -1 gives the Matsubara branch.  Queued on `stream`, allocates
 * nothing. */
int nessi_gpu_gw_polarization_timestep(int tstp, int nk, const nessi_hm_ptrs *G, const nessi_hm_ptrs *P, const double *w,
                                       int nt, int ntau, int size1, int sig_g, void *stream);
int nessi_gpu_gw_sigma_timestep(int tstp, int nk, const nessi_hm_ptrs *G, const nessi_hm_ptrs *W, const nessi_hm_ptrs *S,
                                const double *w, int nt, int ntau, int size1, void *stream);

/* Volterra kernels in use for a group: -1 = one problem per CTA, 2/4/8 = problems per CTA of the
 * tensor-core kernels, 100 = the group-wide blocked recursion by thread-block clusters (trailing
 * updates on the FP64 tensor cores), 0 = not chosen yet (the autotuner decides at the first eager
 * step with n >= max(min(128, nt), 3 nt / 4); the environment variable NESSI_VOLTERRA_PP read at
 * batch creation fixes the choice).  No reference counterpart. */
int nessi_gpu_get_volterra_choice(nessi_batch *b, int group, int *pp_ret, int *pp_les);

/* ---- CUDA graphs of the per-step launch sequence ---------------------------------------------
 * Record the launches of time steps n0..n1 (kind 0: dyson_timestep, 1: vie2_timestep,
 * 2: lattice_2b_timestep with corrector_steps) into a CUDA graph held by the batch, without
 * executing them; nessi_gpu_graph_launch replays the recording on the batch stream.  A replay
 * repeats exactly the recorded launches, so it reproduces the steps as long as the inputs they
 * read (H, a fixed Sigma, the bootstrap steps) are unchanged; record after the batch has run
 * the same steps once (as a warm-up), so that nothing is set up during the recording.  A new
 * recording replaces the previous one.  No reference counterpart (libcntr has no streams). */
int nessi_gpu_graph_record(nessi_batch *b, int kind, int n0, int n1, int corrector_steps);
int nessi_gpu_graph_launch(nessi_batch *b);

/* Wait for all work queued on the batch.  Returns NESSI_ERR_TIMEOUT (and clears the condition)
 * when a bounded wait inside one of the batch's kernels gave up since the last call: the kernel
 * then returned without writing its results, so the time steps queued since the last check are
 * invalid.  No reference counterpart (libcntr's host loops have no device waits). */
int nessi_gpu_synchronize(nessi_batch *b);

/* Bound, in nanoseconds of the device clock, of every wait of the batch's kernels on an mbarrier
 * (the tv history stream waits for its bulk copies and for its consumers).  Default 2e9; a launch
 * reads the value when it is queued (a recorded graph keeps the value of its recording).  A
 * bound of 0 makes every wait give up at once, so that the next synchronize reports
 * NESSI_ERR_TIMEOUT: a way to exercise the timeout path.  No reference counterpart. */
int nessi_gpu_set_wait_limit(nessi_batch *b, long long ns);

#ifdef __cplusplus
}
#endif
#endif /* NESSI_GPU_H */
