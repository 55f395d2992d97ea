// Oracle: CPU restatement of libcntr's serial Kadanoff-Baym path, for testing.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in nessi_b200/ links, imports or calls this
// code; only tests/, __graft_entry__.smoke() and the cpu_baseline / reference
// arm of bench.py use it, and there only as the checker or the timed CPU
// baseline.
//
// libcntr itself cannot be compiled on this machine: it requires Eigen3
// (libcntr/CMakeLists.txt:46-48), which is absent.  This file restates, in
// complex<double>, the routines of the hot path with the reference's loop order
// and weight selection.  Each function names the reference lines it follows.
//
// Pinned against: the reference's integration tables (bit for bit), the closed-form
// known answers of its test suite (embedding, convolution identities, bubbles, Matsubara
// fixpoint, free propagators), and libcntr's own output: the golden densities of
// libcntr/test/fkm_bethe_quench.h5, reproduced to 4.8e-13 (tests/test_oracle_fkm.py).
//
// Storage follows libcntr's herm_matrix exactly (cntr_herm_matrix_impl.hpp:457-477):
//   ret(t,t'), t' <= t   at ((t(t+1))/2 + t') * s^2
//   les(t,t'), t <= t'   at ((t'(t'+1))/2 + t) * s^2
//   tv(t,tau)            at (t(ntau+1) + tau) * s^2
//   mat(tau)             at tau * s^2
// with every element a row-major s x s block of complex<double>.
#pragma once
#include <complex>

typedef std::complex<double> ocplx;

extern "C" {

// A herm_matrix view over caller-owned arrays (libcntr herm_matrix<double>).
typedef struct {
    int nt, ntau, size, sig;
    ocplx *ret, *les, *tv, *mat;
} orc_hm;

// Integrator tables (integration.hpp:128-504); used by tests to pin the tables.
double orc_gregory_weights(int k, int m, int j);
double orc_gregory_omega(int k, int j);
double orc_poly_integration(int k, int i, int j, int l);
double orc_poly_differentiation(int k, int i, int l);
double orc_poly_interpolation(int k, int a, int l);
double orc_bd_weights(int k, int l);
double orc_rcorr(int k, int m, int j, int l);

// Small dense complex solve X from M X = Q (FullPivLU semantics), n x n, nrhs columns.
int orc_cplx_solve(int n, int nrhs, const ocplx *M, const ocplx *Q, ocplx *X);

// Equilibrium / inputs (cntr_equilibrium_impl.hpp:873-955).  H0 is s x s.
void orc_green_from_H_const(orc_hm *G, double mu, const ocplx *H0, double beta, double h);

// Convolution (cntr_convolution_impl.hpp:1582-1727, 594-605).
void orc_convolution_timestep(int n, orc_hm *C, orc_hm *A, orc_hm *Acc, orc_hm *B, orc_hm *Bcc,
                              int k, double beta, double h);
void orc_convolution_matsubara(orc_hm *C, orc_hm *A, orc_hm *B, int k, double beta);

// Dyson (cntr_dyson_impl.hpp:1393-1648).  H holds (nt+2) s x s blocks, H(-1) first.
void orc_dyson_mat(orc_hm *G, orc_hm *Sigma, double mu, const ocplx *H, int k, double beta,
                   int method, int force_hermitian);
void orc_dyson_start(orc_hm *G, double mu, const ocplx *H, orc_hm *Sigma, int k, double beta,
                     double h);
void orc_dyson_timestep(int n, orc_hm *G, double mu, const ocplx *H, orc_hm *Sigma, int k,
                        double beta, double h);

// VIE2 (cntr_vie2_impl.hpp:1310-1685).
void orc_vie2_mat(orc_hm *G, orc_hm *F, orc_hm *Fcc, orc_hm *Q, double beta, int k, int method);
void orc_vie2_start(orc_hm *G, orc_hm *F, orc_hm *Fcc, orc_hm *Q, int k, double beta, double h);
void orc_vie2_timestep(int n, orc_hm *G, orc_hm *F, orc_hm *Fcc, orc_hm *Q, int k, double beta,
                       double h, int method);
// vie2_timestep_sin (cntr_vie2_impl.hpp:1779-1838): Fsin, Qsin, Gsin are (nt+2) s x s blocks.
void orc_vie2_timestep_sin(int n, orc_hm *G, ocplx *Gsin, orc_hm *F, orc_hm *Fcc, const ocplx *Fsin, orc_hm *Q,
                           const ocplx *Qsin, int k, double beta, double h);

// incr_convolution (cntr_convolution_impl.hpp:4164-4807): C += alpha A * F * B at time step tstp.
// which = 0 mat, 1 ret, 2 tv, 3 les; mask (ntau+1 or tstp+1 entries) null = all; ftdata =
// function data with F(-1) first, or null.
void orc_incr_convolution_part(int which, int tstp, const char *mask, double are, double aim, orc_hm *C,
                               orc_hm *A, orc_hm *Acc, const ocplx *ftdata, orc_hm *B, orc_hm *Bcc, int k,
                               double beta, double h);
void orc_incr_convolution(int tstp, double are, double aim, orc_hm *C, orc_hm *A, orc_hm *Acc, const ocplx *ftdata,
                          orc_hm *B, orc_hm *Bcc, int k, double beta, double h);
// The OpenMP solvers' discretization (cntr_dyson_omp_impl.hpp:37-605, cntr_vie2_impl.hpp:1851-2190),
// run in one thread's order.
void orc_dyson_timestep_omp(int n, orc_hm *G, double mu, const ocplx *H, orc_hm *Sigma, int k, double beta,
                            double h);
void orc_vie2_timestep_omp(int tstp, orc_hm *G, orc_hm *F, orc_hm *Fcc, orc_hm *Q, int k, double beta, double h,
                           int method);

// Utilities (cntr_utilities_impl.hpp:22-170, 607-650, 2077-2110).
void orc_extrapolate_timestep(int n, orc_hm *G, int k);
double orc_distance_norm2(int tstp, orc_hm *g1, orc_hm *g2);
void orc_force_matsubara_hermitian(orc_hm *G);

// Bubbles at one time step (cntr_bubble_impl.hpp:138-330): C(t,t') = i A_a1a2(t,t') B_b2b1(t',t)
// and C = i A(t,t') B(t,t') for scalar (1x1) functions.
void orc_bubble1_scalar(int tstp, orc_hm *C, orc_hm *A, orc_hm *Acc, orc_hm *B, orc_hm *Bcc);
void orc_bubble2_scalar(int tstp, orc_hm *C, orc_hm *A, orc_hm *Acc, orc_hm *B, orc_hm *Bcc);
// element-index forms (cntr_bubble_impl.hpp:17-330): C_{c1c2} from A_{a1a2} and B_{b2b1} / B_{b1b2}
void orc_bubble1(int tstp, orc_hm *C, int c1, int c2, orc_hm *A, orc_hm *Acc, int a1, int a2, orc_hm *B,
                 orc_hm *Bcc, int b1, int b2);
void orc_bubble2(int tstp, orc_hm *C, int c1, int c2, orc_hm *A, orc_hm *Acc, int a1, int a2, orc_hm *B,
                 orc_hm *Bcc, int b1, int b2);

// Self-consistent lattice with a local second-order self-energy (examples/programs/
// hubbard_chain_selfen_impl.cpp:63-75, hubbard_chain_2b.cpp:245-324, with G -> G_loc, the
// k-average of the problems' G).  U holds (nt+2) s x s blocks, U(-1) first.
void orc_sigma_2b_timestep(int tstp, orc_hm *Sigma, orc_hm *G, const ocplx *U);
void orc_gloc_timestep(int tstp, int nprob, orc_hm *G, orc_hm *Gloc);
int orc_lattice2b_start(int nprob, orc_hm *G, orc_hm *Gloc, orc_hm *Sigma, const ocplx *U, double mu,
                        const ocplx *H, long h_stride, int k, double beta, double h, int max_iter, double tol,
                        double *err_out, int nthreads);
void orc_lattice2b_timestep(int n, int nprob, orc_hm *G, orc_hm *Gloc, orc_hm *Sigma, const ocplx *U, double mu,
                            const ocplx *H, long h_stride, int k, double beta, double h, int ncorr, int nthreads);

// Batched driver used as the CPU baseline: Dyson time steps n0..n1 (inclusive) for
// nprob problems that share one Sigma, distributed over nthreads OpenMP threads
// (the "OpenMP over k" harness of the reference's lattice driver, gw.cpp:386-420).
void orc_dyson_timestep_batch(int n0, int n1, int nprob, orc_hm *G, double mu, const ocplx *H,
                              long h_stride, orc_hm *Sigma, int k, double beta, double h,
                              int nthreads);
}
