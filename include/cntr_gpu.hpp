// cntr_gpu.hpp - header-only C++ front end of libnessi_gpu.so with libcntr's call signatures.
//
// A libcntr program replaces
//     cntr::dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder);
// by
//     cntr_gpu::dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder);
// with G, Sigma of type cntr::herm_matrix<double> and H of type cntr::function<double>
// (libcntr/cntr/cntr_dyson_decl.hpp:78-92).  The templates only need the public accessors of
// those classes (nt, ntau, size1, sig, retptr, lesptr, tvptr, matptr; function::ptr), so this
// header does not include libcntr.
//
// The single-problem functions copy the whole G and Sigma to the device on every call, which is
// what a drop-in for one call can do.  Lattice codes advance all k-points of a time step
// together through cntr_gpu::Batch (the replacement of the per-k loop of
// examples/programs/gw.cpp:386-420), which keeps every G and the shared Sigma in device memory
// and moves only time-step slices.
#pragma once

#include <complex>
#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "nessi_gpu.h"
#include "nessi_io.h"

namespace cntr_gpu {

inline void check(int rc) {
    if (rc != NESSI_OK) throw std::runtime_error(std::string("libnessi_gpu: ") + nessi_gpu_last_error());
}

inline void check_io(int rc) {
    if (rc != 0) throw std::runtime_error(std::string("libnessi_io: ") + nessi_io_last_error());
}

// G.print_to_file(file, precision) and G.read_from_file(nt1, file) of libcntr
// (cntr_herm_matrix_impl.hpp:1308-1560) through libnessi_io.so (link -lnessi_io); the files are
// libcntr's text format.  Precision 17 makes the round trip exact.
template <class HM> void print_to_file(HM &G, const char *file, int precision = 16) {
    check_io(nessi_hm_print_to_file(file, G.nt(), G.ntau(), G.size1(), G.sig(), G.nt() >= 0 ? G.retptr(0, 0) : nullptr,
                                    G.nt() >= 0 ? G.lesptr(0, 0) : nullptr, G.nt() >= 0 ? G.tvptr(0, 0) : nullptr,
                                    G.matptr(0), precision));
}
template <class HM> void read_from_file(HM &G, int nt1, const char *file) {
    check_io(nessi_hm_read_from_file_nt1(file, nt1, G.nt(), G.ntau(), G.size1(),
                                         G.nt() >= 0 ? G.retptr(0, 0) : nullptr, G.nt() >= 0 ? G.lesptr(0, 0) : nullptr,
                                         G.nt() >= 0 ? G.tvptr(0, 0) : nullptr, G.matptr(0)));
}

// number of complex<double> in one herm_matrix_timestep slice [ret | tv | les] (n >= 0)
template <class HM> inline long slice_len(const HM &G, int n) {
    return (2L * (n + 1) + G.ntau() + 1) * G.size1() * G.size1();
}

// Problems advanced together; problems added with the same sigma_group share one Sigma.
template <class HM, class FN> class Batch {
  public:
    explicit Batch(int precision = NESSI_PREC_FP64) : precision_(precision) {}
    ~Batch() { if (b_) nessi_gpu_batch_destroy(b_); }
    Batch(const Batch &) = delete;
    Batch &operator=(const Batch &) = delete;

    // register problem p (returns its index); call before build()
    int add(HM &G, FN &H, double mu, double beta, double h, int SolveOrder = 5, int sigma_group = 0) {
        nessi_problem_desc d;
        d.nt = G.nt(); d.ntau = G.ntau(); d.size1 = G.size1(); d.sig = G.sig();
        d.solve_order = SolveOrder; d.sigma_group = sigma_group; d.beta = beta; d.h = h; d.mu = mu;
        descs_.push_back(d);
        G_.push_back(&G);
        H_.push_back(&H);
        return (int)descs_.size() - 1;
    }
    // allocate device storage and upload G (all components), H and the group's Sigma
    void build(HM &Sigma, int sigma_group = 0) {
        check(nessi_gpu_batch_create(&b_, descs_.data(), (int)descs_.size(), precision_));
        for (size_t p = 0; p < G_.size(); p++) {
            HM &G = *G_[p];
            check(nessi_gpu_set_G(b_, (int)p, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0)));
            check(nessi_gpu_set_H(b_, (int)p, H_[p]->ptr(-1)));
        }
        set_sigma(Sigma, sigma_group);
    }
    void set_sigma(HM &Sigma, int sigma_group = 0) {
        check(nessi_gpu_set_sigma(b_, sigma_group, Sigma.retptr(0, 0), Sigma.lesptr(0, 0), Sigma.tvptr(0, 0),
                                  Sigma.matptr(0)));
    }
    // one time step of Sigma, in herm_matrix_timestep order (e.g. from a self-energy diagram)
    void set_sigma_timestep(int n, const std::complex<double> *slice, int sigma_group = 0) {
        check(nessi_gpu_set_sigma_timestep(b_, sigma_group, n, slice));
    }
    // VIE2 groups: kernel F (with partner Fcc) shared by the group, source Q per problem
    void set_F(HM &F, HM &Fcc, int group = 0) {
        check(nessi_gpu_set_F(b_, group, F.retptr(0, 0), F.lesptr(0, 0), F.tvptr(0, 0), F.matptr(0),
                              Fcc.retptr(0, 0), Fcc.lesptr(0, 0)));
        check(nessi_gpu_set_Fcc_mat(b_, group, Fcc.matptr(0)));  // read by the steepest-descent vie2_mat
    }
    void set_Q(int p, HM &Q) {
        check(nessi_gpu_set_Q(b_, p, Q.retptr(0, 0), Q.lesptr(0, 0), Q.tvptr(0, 0), Q.matptr(0)));
    }
    void vie2_mat(int method = 2) { check(nessi_gpu_vie2_mat_method(b_, method)); }
    void vie2_start() { check(nessi_gpu_vie2_start(b_)); }
    void vie2_timestep(int n) { check(nessi_gpu_vie2_timestep(b_, n)); }
    // self-consistent lattice with the local second-order self-energy of G_loc
    void set_U(const std::complex<double> *udiag, int group = 0) { check(nessi_gpu_set_U(b_, group, udiag)); }
    void extrapolate_timestep(int n) { check(nessi_gpu_extrapolate_timestep(b_, n)); }
    int lattice_2b_start(int max_iter, double tol, double *err = nullptr) {
        int it = 0;
        check(nessi_gpu_lattice_2b_start(b_, max_iter, tol, &it, err));
        return it;
    }
    void lattice_2b_timestep(int n, int corrector_steps) { check(nessi_gpu_lattice_2b_timestep(b_, n, corrector_steps)); }
    void dyson_mat(int method = 2, bool force_hermitian = true) {
        check(nessi_gpu_dyson_mat_method(b_, method, force_hermitian ? 1 : 0));
    }
    void dyson_start() { check(nessi_gpu_dyson_start(b_)); }
    void dyson_timestep(int n) { check(nessi_gpu_dyson_timestep(b_, n)); }
    // copy time step n of problem p back into its herm_matrix
    void download_timestep(int p, int n) {
        HM &G = *G_[p];
        std::vector<std::complex<double>> s(n < 0 ? (long)(G.ntau() + 1) * G.size1() * G.size1() : slice_len(G, n));
        check(nessi_gpu_get_timestep(b_, p, n, s.data()));
        const long es = (long)G.size1() * G.size1();
        if (n < 0) {
            std::copy(s.begin(), s.end(), G.matptr(0));
            return;
        }
        const long n1 = n + 1, M = G.ntau() + 1;
        std::copy(s.begin(), s.begin() + n1 * es, G.retptr(n, 0));
        std::copy(s.begin() + n1 * es, s.begin() + (n1 + M) * es, G.tvptr(n, 0));
        std::copy(s.begin() + (n1 + M) * es, s.end(), G.lesptr(0, n));
    }
    void download_all() {
        for (size_t p = 0; p < G_.size(); p++) download(p);
    }
    // all components of problem p: device -> its herm_matrix, and back
    void download(size_t p) {
        HM &G = *G_[p];
        check(nessi_gpu_get_G(b_, (int)p, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0)));
    }
    void upload(size_t p) {
        HM &G = *G_[p];
        check(nessi_gpu_set_G(b_, (int)p, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0)));
    }
    // checkpoint problem p in libcntr's text format; restart it from time steps 0..nt1 of such a
    // file (the propagation continues with nt1 + 1)
    void checkpoint(size_t p, const char *file, int precision = 17) {
        download(p);
        print_to_file(*G_[p], file, precision);
    }
    void restart(size_t p, int nt1, const char *file) {
        read_from_file(*G_[p], nt1, file);
        upload(p);
    }
    nessi_batch *handle() { return b_; }

  private:
    int precision_;
    nessi_batch *b_ = nullptr;
    std::vector<nessi_problem_desc> descs_;
    std::vector<HM *> G_;
    std::vector<FN *> H_;
};

// Matsubara methods of libcntr (cntr_global_settings.hpp); dyson_mat solves by all three on the
// device, vie2_mat by the Fourier and the fixpoint methods (steepest descent needs Fcc^mat)
constexpr int MAT_FOURIER = 0;
constexpr int MAT_CG = 1;
constexpr int MAT_FIXPOINT = 2;
inline void require_device_method(int method, bool vie = false) {
    if (method != MAT_FOURIER && method != MAT_FIXPOINT && method != MAT_CG)
        throw std::invalid_argument("cntr_gpu: Matsubara method " + std::to_string(method) +
                                    " is not available on the device for " + (vie ? "vie2_mat" : "dyson_mat"));
}

// ---- single-problem drop-ins (cntr_dyson_decl.hpp:78-92) -------------------------------
namespace detail {
// The device copy of the last problem stepped by cntr_gpu::dyson_timestep, kept between calls
// (one per host thread), and the bytes the single-call functions moved across PCIe.
struct StepCache {
    nessi_batch *b = nullptr;
    const void *G = nullptr, *Sigma = nullptr, *H = nullptr;
    int nt = 0, ntau = 0, s = 0, sig = 0, k = 0, last_n = -2;
    double mu = 0, beta = 0, h = 0;
    void release() {
        if (b) nessi_gpu_batch_destroy(b);
        b = nullptr;
        last_n = -2;
    }
    ~StepCache() { release(); }
};
inline StepCache &step_cache() {
    thread_local StepCache c;
    return c;
}
inline long long &transfer_bytes_counter() {
    thread_local long long n = 0;
    return n;
}
}  // namespace detail

// Bytes copied between host and device by cntr_gpu::dyson_timestep on this thread so far.
inline long long transfer_bytes() { return detail::transfer_bytes_counter(); }
// Forget the device copy kept by cntr_gpu::dyson_timestep; the next call uploads everything.
inline void dyson_timestep_reset() { detail::step_cache().release(); }

// cntr::dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder).  The first call on a problem
// uploads G, H and Sigma whole and keeps them on the device; a following call on the same objects
// (same addresses and parameters) for the same n (a corrector iteration) or for n + 1 (the next
// step) uploads only Sigma's time step n and H, and every call downloads only G's time step n.
// So between such calls the caller may change Sigma's time step n and H -- as libcntr's
// predictor-corrector drivers do -- but not G's or Sigma's earlier time steps; after changing
// those, call dyson_timestep_reset() (any other n, or other objects, start over by themselves).
template <class HM, class FN>
void dyson_timestep(int n, HM &G, double mu, FN &H, HM &Sigma, double beta, double h, int SolveOrder = 5) {
    detail::StepCache &c = detail::step_cache();
    const long es = (long)G.size1() * G.size1();
    const bool same = c.b && c.G == (const void *)&G && c.Sigma == (const void *)&Sigma && c.H == (const void *)&H &&
                      c.nt == G.nt() && c.ntau == G.ntau() && c.s == G.size1() && c.sig == G.sig() &&
                      c.k == SolveOrder && c.mu == mu && c.beta == beta && c.h == h &&
                      (n == c.last_n || n == c.last_n + 1);
    const long tri = (long)(G.nt() + 1) * (G.nt() + 2) / 2 * es, tvn = (long)(G.nt() + 1) * (G.ntau() + 1) * es;
    const long fn = (long)(G.nt() + 2) * es, matn = (long)(G.ntau() + 1) * es;
    if (!same) {
        c.release();
        nessi_problem_desc d;
        d.nt = G.nt(); d.ntau = G.ntau(); d.size1 = G.size1(); d.sig = G.sig();
        d.solve_order = SolveOrder; d.sigma_group = 0; d.beta = beta; d.h = h; d.mu = mu;
        check(nessi_gpu_batch_create(&c.b, &d, 1, NESSI_PREC_FP64));
        check(nessi_gpu_set_G(c.b, 0, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0)));
        check(nessi_gpu_set_H(c.b, 0, H.ptr(-1)));
        check(nessi_gpu_set_sigma(c.b, 0, Sigma.retptr(0, 0), Sigma.lesptr(0, 0), Sigma.tvptr(0, 0), Sigma.matptr(0)));
        c.G = &G; c.Sigma = &Sigma; c.H = &H;
        c.nt = G.nt(); c.ntau = G.ntau(); c.s = G.size1(); c.sig = G.sig(); c.k = SolveOrder;
        c.mu = mu; c.beta = beta; c.h = h;
        detail::transfer_bytes_counter() += 16 * (4 * tri + 2 * tvn + 2 * matn + fn);
    } else {
        std::vector<std::complex<double>> sl(slice_len(Sigma, n));
        const long n1 = n + 1, M = G.ntau() + 1;
        std::copy(Sigma.retptr(n, 0), Sigma.retptr(n, 0) + n1 * es, sl.begin());
        std::copy(Sigma.tvptr(n, 0), Sigma.tvptr(n, 0) + M * es, sl.begin() + n1 * es);
        for (long j = 0; j <= n; j++) std::copy(Sigma.lesptr(j, n), Sigma.lesptr(j, n) + es, sl.begin() + (n1 + M + j) * es);
        check(nessi_gpu_set_sigma_timestep(c.b, 0, n, sl.data()));
        check(nessi_gpu_set_H(c.b, 0, H.ptr(-1)));
        detail::transfer_bytes_counter() += 16 * ((long)sl.size() + fn);
    }
    c.last_n = -2;  // a failure below leaves no reusable state
    check(nessi_gpu_dyson_timestep(c.b, n));
    std::vector<std::complex<double>> out(slice_len(G, n));
    check(nessi_gpu_get_timestep(c.b, 0, n, out.data()));
    const long n1 = n + 1, M = G.ntau() + 1;
    std::copy(out.begin(), out.begin() + n1 * es, G.retptr(n, 0));
    std::copy(out.begin() + n1 * es, out.begin() + (n1 + M) * es, G.tvptr(n, 0));
    for (long j = 0; j <= n; j++) std::copy(out.begin() + (n1 + M + j) * es, out.begin() + (n1 + M + j + 1) * es, G.lesptr(j, n));
    detail::transfer_bytes_counter() += 16 * (long)out.size();
    c.last_n = n;
}

template <class HM, class FN>
void dyson_start(HM &G, double mu, FN &H, HM &Sigma, double beta, double h, int SolveOrder = 5) {
    Batch<HM, FN> b;
    b.add(G, H, mu, beta, h, SolveOrder);
    b.build(Sigma);
    b.dyson_start();
    for (int n = 0; n <= SolveOrder; n++) b.download_timestep(0, n);
}

// cntr::dyson_mat(G, mu, H, Sigma, beta, SolveOrder, method, force_hermitian)
// (cntr_dyson_decl.hpp:77-79): only H(-1) and Sigma^mat take part, so G may hold the Matsubara
// branch alone (nt = -1); the device problem carries k time steps that stay unused
template <class HM, class FN>
void dyson_mat(HM &G, double mu, FN &H, HM &Sigma, double beta, int SolveOrder = 5, int method = MAT_FIXPOINT,
               bool force_hermitian = true) {
    require_device_method(method);
    nessi_problem_desc d;
    d.nt = SolveOrder; d.ntau = G.ntau(); d.size1 = G.size1(); d.sig = G.sig();
    d.solve_order = SolveOrder; d.sigma_group = 0; d.beta = beta; d.h = 1.0; d.mu = mu;
    const long es = (long)G.size1() * G.size1();
    std::vector<std::complex<double>> h0((long)(SolveOrder + 2) * es);
    for (int t = 0; t < SolveOrder + 2; t++) std::copy(H.ptr(-1), H.ptr(-1) + es, h0.begin() + t * es);
    nessi_batch *b = nullptr;
    check(nessi_gpu_batch_create(&b, &d, 1, NESSI_PREC_FP64));
    int rc = nessi_gpu_set_H(b, 0, h0.data());
    if (!rc) rc = nessi_gpu_set_sigma(b, 0, nullptr, nullptr, nullptr, Sigma.matptr(0));
    if (!rc) rc = nessi_gpu_dyson_mat_method(b, method, force_hermitian ? 1 : 0);
    if (!rc) rc = nessi_gpu_get_G(b, 0, nullptr, nullptr, nullptr, G.matptr(0));
    nessi_gpu_batch_destroy(b);
    check(rc);
}

// cntr::dyson(G, mu, H, Sigma, beta, h, SolveOrder, matsubara_method, force_hermitian)
// (cntr_dyson_decl.hpp:95-98, cntr_dyson_impl.hpp:1725-1734): dyson_mat, dyson_start and every
// time step k+1..nt on the device from one upload, then all of G comes back.  G.nt() >= 0.
template <class HM, class FN>
void dyson(HM &G, double mu, FN &H, HM &Sigma, double beta, double h, int SolveOrder = 5,
           int matsubara_method = MAT_FIXPOINT, bool force_hermitian = true) {
    require_device_method(matsubara_method);
    Batch<HM, FN> b;
    b.add(G, H, mu, beta, h, SolveOrder);
    b.build(Sigma);
    b.dyson_mat(matsubara_method, force_hermitian);
    b.dyson_start();
    for (int n = SolveOrder + 1; n <= G.nt(); n++) b.dyson_timestep(n);
    b.download_all();
}

// cntr::extrapolate_timestep(n, G, SolveOrder) (cntr_utilities_decl.hpp:23,
// cntr_utilities_impl.hpp:22-130): time step n+1 of G predicted from n-k..n; n >= SolveOrder
template <class HM> void extrapolate_timestep(int n, HM &G, int SolveOrder = 5) {
    if (n + 1 > G.nt() || n < SolveOrder)  // where libcntr aborts (cntr_utilities_impl.hpp:35-39)
        throw std::invalid_argument("cntr_gpu::extrapolate_timestep: n out of range");
    nessi_problem_desc d;
    d.nt = G.nt(); d.ntau = G.ntau(); d.size1 = G.size1(); d.sig = G.sig();
    d.solve_order = SolveOrder; d.sigma_group = 0; d.beta = 1.0; d.h = 1.0; d.mu = 0.0;
    nessi_batch *b = nullptr;
    check(nessi_gpu_batch_create(&b, &d, 1, NESSI_PREC_FP64));
    int rc = nessi_gpu_set_G(b, 0, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0));
    if (!rc) rc = nessi_gpu_extrapolate_timestep(b, n);
    std::vector<std::complex<double>> s(slice_len(G, n + 1));
    if (!rc) rc = nessi_gpu_get_timestep(b, 0, n + 1, s.data());
    nessi_gpu_batch_destroy(b);
    check(rc);
    const long es = (long)G.size1() * G.size1(), n1 = n + 2, M = G.ntau() + 1;
    std::copy(s.begin(), s.begin() + n1 * es, G.retptr(n + 1, 0));
    std::copy(s.begin() + n1 * es, s.begin() + (n1 + M) * es, G.tvptr(n + 1, 0));
    std::copy(s.begin() + (n1 + M) * es, s.end(), G.lesptr(0, n + 1));
}

// ---- VIE2 single-problem drop-ins (cntr_vie2_decl.hpp:63-90) --------------------------------
// one-problem VIE2 batch of order k holding F, Fcc, Q and (optionally all of) G
template <class HM> nessi_batch *vie2_batch(HM &G, HM &F, HM &Fcc, HM &Q, double beta, double h, int k, bool whole_G) {
    nessi_problem_desc d;
    d.nt = G.nt(); d.ntau = G.ntau(); d.size1 = G.size1(); d.sig = G.sig();
    d.solve_order = k; d.sigma_group = 0; d.beta = beta; d.h = h; d.mu = 0.0;
    nessi_batch *b = nullptr;
    check(nessi_gpu_batch_create(&b, &d, 1, NESSI_PREC_FP64));
    int rc = whole_G ? nessi_gpu_set_G(b, 0, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0))
                     : nessi_gpu_set_G(b, 0, nullptr, nullptr, nullptr, G.matptr(0));
    if (!rc) rc = nessi_gpu_set_F(b, 0, F.retptr(0, 0), F.lesptr(0, 0), F.tvptr(0, 0), F.matptr(0), Fcc.retptr(0, 0),
                                  Fcc.lesptr(0, 0));
    if (!rc) rc = nessi_gpu_set_Fcc_mat(b, 0, Fcc.matptr(0));
    if (!rc) rc = nessi_gpu_set_Q(b, 0, Q.retptr(0, 0), Q.lesptr(0, 0), Q.tvptr(0, 0), Q.matptr(0));
    if (rc) {
        nessi_gpu_batch_destroy(b);
        check(rc);
    }
    return b;
}

// cntr::vie2_mat(G, F, Fcc, Q, beta, SolveOrder, method) (cntr_vie2_decl.hpp:63): G^mat
// (only the Matsubara branches take part, so the matrices may hold it alone, nt = -1)
template <class HM>
void vie2_mat(HM &G, HM &F, HM &Fcc, HM &Q, double beta, int SolveOrder = 5, int method = MAT_FIXPOINT) {
    require_device_method(method, true);
    nessi_problem_desc d;
    d.nt = SolveOrder; d.ntau = G.ntau(); d.size1 = G.size1(); d.sig = G.sig();
    d.solve_order = SolveOrder; d.sigma_group = 0; d.beta = beta; d.h = 1.0; d.mu = 0.0;
    nessi_batch *b = nullptr;
    check(nessi_gpu_batch_create(&b, &d, 1, NESSI_PREC_FP64));
    int rc = nessi_gpu_set_F(b, 0, nullptr, nullptr, nullptr, F.matptr(0), nullptr, nullptr);
    if (!rc && method == MAT_CG) rc = nessi_gpu_set_Fcc_mat(b, 0, Fcc.matptr(0));  // steepest descent reads Fcc^mat
    if (!rc) rc = nessi_gpu_set_Q(b, 0, nullptr, nullptr, nullptr, Q.matptr(0));
    if (!rc) rc = nessi_gpu_vie2_mat_method(b, method);
    if (!rc) rc = nessi_gpu_get_G(b, 0, nullptr, nullptr, nullptr, G.matptr(0));
    nessi_gpu_batch_destroy(b);
    check(rc);
}

// cntr::vie2(G, F, Fcc, Q, beta, h, SolveOrder, matsubara_method) (cntr_vie2_decl.hpp:85-86):
// vie2_mat, vie2_start and every time step on the device from one upload.
template <class HM>
void vie2(HM &G, HM &F, HM &Fcc, HM &Q, double beta, double h, int SolveOrder = 5, int matsubara_method = MAT_FIXPOINT) {
    require_device_method(matsubara_method, true);
    nessi_batch *b = vie2_batch(G, F, Fcc, Q, beta, h, SolveOrder, false);
    int rc = nessi_gpu_vie2_mat_method(b, matsubara_method);
    if (!rc) rc = nessi_gpu_vie2_start(b);
    for (int n = SolveOrder + 1; n <= G.nt() && !rc; n++) rc = nessi_gpu_vie2_timestep(b, n);
    if (!rc) rc = nessi_gpu_get_G(b, 0, G.retptr(0, 0), G.lesptr(0, 0), G.tvptr(0, 0), G.matptr(0));
    nessi_gpu_batch_destroy(b);
    check(rc);
}

// copy time step n (n >= 0) of problem 0 of a batch into G
template <class HM> int fetch_timestep(nessi_batch *b, HM &G, int n) {
    std::vector<std::complex<double>> s(slice_len(G, n));
    int rc = nessi_gpu_get_timestep(b, 0, n, s.data());
    if (rc) return rc;
    const long es = (long)G.size1() * G.size1(), n1 = n + 1, M = G.ntau() + 1;
    std::copy(s.begin(), s.begin() + n1 * es, G.retptr(n, 0));
    std::copy(s.begin() + n1 * es, s.begin() + (n1 + M) * es, G.tvptr(n, 0));
    std::copy(s.begin() + (n1 + M) * es, s.end(), G.lesptr(0, n));
    return NESSI_OK;
}

// cntr::vie2_start(G, F, Fcc, Q, beta, h, SolveOrder) (cntr_vie2_decl.hpp:67): time steps 0..k
template <class HM>
void vie2_start(HM &G, HM &F, HM &Fcc, HM &Q, double beta, double h, int SolveOrder = 5) {
    nessi_batch *b = vie2_batch(G, F, Fcc, Q, beta, h, SolveOrder, false);
    int rc = nessi_gpu_vie2_start(b);
    for (int n = 0; n <= SolveOrder && !rc; n++) rc = fetch_timestep(b, G, n);
    nessi_gpu_batch_destroy(b);
    check(rc);
}

// cntr::vie2_timestep(n, G, F, Fcc, Q, beta, h, SolveOrder, matsubara_method)
// (cntr_vie2_decl.hpp:72, cntr_vie2_impl.hpp:1597-1640): n = -1 gives vie2_mat and
// 1 <= n <= SolveOrder a vie2_start of order n (time steps 0..n), as the reference dispatches;
// n = 0, an order-0 start, is not available
template <class HM>
void vie2_timestep(int n, HM &G, HM &F, HM &Fcc, HM &Q, double beta, double h, int SolveOrder = 5,
                   int matsubara_method = MAT_FIXPOINT) {
    if (n == -1) {
        vie2_mat(G, F, Fcc, Q, beta, SolveOrder, matsubara_method);
        return;
    }
    if (n <= SolveOrder) {
        if (n == 0) throw std::invalid_argument("cntr_gpu::vie2_timestep: an order-0 start (n = 0) is not available");
        vie2_start(G, F, Fcc, Q, beta, h, n);
        return;
    }
    nessi_batch *b = vie2_batch(G, F, Fcc, Q, beta, h, SolveOrder, true);
    int rc = nessi_gpu_vie2_timestep(b, n);
    if (!rc) rc = fetch_timestep(b, G, n);
    nessi_gpu_batch_destroy(b);
    check(rc);
}

// ---- vie2_timestep_sin (cntr_vie2_decl.hpp:58, cntr_vie2_impl.hpp:1779-1838) ------------------
namespace detail {
typedef std::complex<double> cplx;
// z = a b for s x s row-major blocks (z must not alias a or b)
inline void mat_mul(int s, cplx *z, const cplx *a, const cplx *b) {
    for (int i = 0; i < s; i++)
        for (int j = 0; j < s; j++) {
            cplx x = 0;
            for (int l = 0; l < s; l++) x += a[i * s + l] * b[l * s + j];
            z[i * s + j] = x;
        }
}
// inv = a^-1 by Gauss-Jordan elimination with partial pivoting; false if a is singular
inline bool mat_inverse(int s, const cplx *a, cplx *inv) {
    std::vector<cplx> m(a, a + s * s);
    for (int i = 0; i < s * s; i++) inv[i] = (i / s == i % s) ? 1.0 : 0.0;
    for (int c = 0; c < s; c++) {
        int p = c;
        for (int r = c + 1; r < s; r++)
            if (std::abs(m[r * s + c]) > std::abs(m[p * s + c])) p = r;
        if (std::abs(m[p * s + c]) == 0.0) return false;
        for (int j = 0; j < s; j++) {
            std::swap(m[c * s + j], m[p * s + j]);
            std::swap(inv[c * s + j], inv[p * s + j]);
        }
        const cplx d = 1.0 / m[c * s + c];
        for (int j = 0; j < s; j++) { m[c * s + j] *= d; inv[c * s + j] *= d; }
        for (int r = 0; r < s; r++) {
            if (r == c) continue;
            const cplx f = m[r * s + c];
            for (int j = 0; j < s; j++) { m[r * s + j] -= f * m[c * s + j]; inv[r * s + j] -= f * inv[c * s + j]; }
        }
    }
    return true;
}
// herm_matrix::left_multiply / right_multiply at time step t with f given as blocks f(-1), f(0), ...
// (cntr_herm_matrix_impl.hpp:2955-2995, 3206-3246)
template <class HM> void left_multiply(HM &X, int t, const cplx *f) {
    const int s = X.size1(), es = s * s;
    std::vector<cplx> z(es);
    auto fp = [&](int tt) { return f + (long)(tt + 1) * es; };
    auto app = [&](cplx *e, const cplx *fa) { mat_mul(s, z.data(), fa, e); std::copy(z.begin(), z.end(), e); };
    if (t == -1) {
        for (int m = 0; m <= X.ntau(); m++) app(X.matptr(m), fp(-1));
        return;
    }
    for (int m = 0; m <= t; m++) app(X.retptr(t, m), fp(t));
    for (int m = 0; m <= X.ntau(); m++) app(X.tvptr(t, m), fp(t));
    for (int m = 0; m <= t; m++) app(X.lesptr(m, t), fp(m));
}
template <class HM> void right_multiply(HM &X, int t, const cplx *f) {
    const int s = X.size1(), es = s * s;
    std::vector<cplx> z(es);
    auto fp = [&](int tt) { return f + (long)(tt + 1) * es; };
    auto app = [&](cplx *e, const cplx *fa) { mat_mul(s, z.data(), e, fa); std::copy(z.begin(), z.end(), e); };
    if (t == -1) {
        for (int m = 0; m <= X.ntau(); m++) app(X.matptr(m), fp(-1));
        return;
    }
    for (int m = 0; m <= t; m++) app(X.retptr(t, m), fp(m));
    for (int m = 0; m <= X.ntau(); m++) app(X.tvptr(t, m), fp(-1));
    for (int m = 0; m <= t; m++) app(X.lesptr(m, t), fp(t));
}
// X(t) -= Y(t) on time step t
template <class HM> void decr_timestep(HM &X, HM &Y, int t) {
    const long es = (long)X.size1() * X.size1();
    auto sub = [&](cplx *x, const cplx *y, long n) { for (long i = 0; i < n; i++) x[i] -= y[i]; };
    if (t == -1) { sub(X.matptr(0), Y.matptr(0), (X.ntau() + 1) * es); return; }
    sub(X.retptr(t, 0), Y.retptr(t, 0), (t + 1) * es);
    sub(X.tvptr(t, 0), Y.tvptr(t, 0), (X.ntau() + 1) * es);
    sub(X.lesptr(0, t), Y.lesptr(0, t), (t + 1) * es);
}
}  // namespace detail

// [1 + F] G = Q where F, Q and G carry instantaneous parts Fsin, Qsin, Gsin: the time-local
// algebra on the host as in the reference (Finv = (1 + Fsin)^-1, Gsin = Finv Qsin, F -> Finv F,
// Fcc -> Fcc Finv, Q -> Finv Q - (Finv F) Gsin on t = -1..max(n, k)), then vie2_timestep's
// dispatch on the device.  HM must be copyable (libcntr's herm_matrix is).
template <class HM, class FN>
void vie2_timestep_sin(int n, HM &G, FN &Gsin, HM &F, HM &Fcc, FN &Fsin, HM &Q, FN &Qsin, double beta, double h,
                       int SolveOrder = 5) {
    if (n == 0) throw std::invalid_argument("cntr_gpu::vie2_timestep_sin: an order-0 start (n = 0) is not available");
    const int s = G.size1(), es = s * s;
    const int n2 = (n >= 0 && n <= SolveOrder) ? SolveOrder : n;
    std::vector<detail::cplx> finv((long)(n2 + 2) * es), gsin((long)(n2 + 2) * es), a(es);
    for (int t = -1; t <= n2; t++) {
        const detail::cplx *fs = Fsin.ptr(t);
        for (int i = 0; i < es; i++) a[i] = fs[i] + ((i / s == i % s) ? 1.0 : 0.0);
        detail::cplx *fi = finv.data() + (long)(t + 1) * es, *gs = gsin.data() + (long)(t + 1) * es;
        if (!detail::mat_inverse(s, a.data(), fi))
            throw std::runtime_error("cntr_gpu::vie2_timestep_sin: 1 + Fsin is singular");
        detail::mat_mul(s, gs, fi, Qsin.ptr(t));
        std::copy(gs, gs + es, Gsin.ptr(t));
    }
    HM tF(F), tFcc(Fcc), tQ(Q);
    for (int t = -1; t <= n2; t++) {
        detail::left_multiply(tF, t, finv.data());
        detail::right_multiply(tFcc, t, finv.data());
        detail::left_multiply(tQ, t, finv.data());
    }
    HM tF1(tF);
    for (int t = -1; t <= n2; t++) {
        detail::right_multiply(tF1, t, gsin.data());
        detail::decr_timestep(tQ, tF1, t);
    }
    vie2_timestep(n, G, tF, tFcc, tQ, beta, h, SolveOrder);
}

// ---- convolution_timestep / convolution (cntr_convolution_decl.hpp:59-68) ----------------
template <class HM> inline nessi_hm_ptrs hm_ptrs(HM &X) {
    nessi_hm_ptrs q;
    q.ret = X.retptr(0, 0); q.les = X.lesptr(0, 0); q.tv = X.tvptr(0, 0); q.mat = X.matptr(0);
    return q;
}
template <class HM>
void convolution_timestep(int n, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, double beta, double h, int SolveOrder = 5) {
    nessi_hm_ptrs c = hm_ptrs(C), a = hm_ptrs(A), acc = hm_ptrs(Acc), b = hm_ptrs(B), bcc = hm_ptrs(Bcc);
    check(nessi_gpu_convolution_timestep_host(n, &c, &a, &acc, &b, &bcc, C.nt(), C.ntau(), C.size1(), A.sig(), B.sig(),
                                              SolveOrder, beta, h));
}
// hermitian A and B (:64-65): Acc = A, Bcc = B
template <class HM> void convolution_timestep(int n, HM &C, HM &A, HM &B, double beta, double h, int SolveOrder = 5) {
    convolution_timestep(n, C, A, A, B, B, beta, h, SolveOrder);
}
// every time step, convolution_matsubara then n = 0..nt (:66-68, cntr_convolution_impl.hpp:1805-1812)
template <class HM>
void convolution(HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, double beta, double h, int SolveOrder = 5) {
    nessi_hm_ptrs c = hm_ptrs(C), a = hm_ptrs(A), acc = hm_ptrs(Acc), b = hm_ptrs(B), bcc = hm_ptrs(Bcc);
    check(nessi_gpu_convolution_host(&c, &a, &acc, &b, &bcc, C.nt(), C.ntau(), C.size1(), A.sig(), B.sig(), SolveOrder,
                                     beta, h));
}
template <class HM> void convolution(HM &C, HM &A, HM &B, double beta, double h, int SolveOrder = 5) {
    convolution(C, A, A, B, B, beta, h, SolveOrder);
}

// ---- the element-parallel routines of libcntr's OpenMP path ----------------------------------
// omp_num_threads is accepted for the signature and ignored: every element is a GPU thread.
//
// incr_convolution(tstp, alpha, C, A, Acc, f0, ft, B, Bcc, I, beta, h)
// (cntr_convolution_impl.hpp:4786-4807): C(tstp) += alpha A * F * B; F is a cntr::function
// (F(-1) as f0, F(t) as ft); the overload without F takes F = 1 (f0 = ft = NULL in the reference).
namespace detail {
template <class HM>
void incr_convolution_raw(int tstp, std::complex<double> alpha, HM &C, HM &A, HM &Acc, const void *fdata, HM &B,
                          HM &Bcc, double beta, double h, int SolveOrder) {
    nessi_hm_ptrs c = hm_ptrs(C), a = hm_ptrs(A), acc = hm_ptrs(Acc), b = hm_ptrs(B), bcc = hm_ptrs(Bcc);
    check(nessi_gpu_incr_convolution_timestep_host(tstp, alpha.real(), alpha.imag(), &c, &a, &acc, fdata, &b, &bcc,
                                                   C.nt(), C.ntau(), C.size1(), A.sig(), B.sig(), SolveOrder, beta, h));
}
}  // namespace detail
template <class HM, class FN>
void incr_convolution(int tstp, std::complex<double> alpha, HM &C, HM &A, HM &Acc, FN &F, HM &B, HM &Bcc, double beta,
                      double h, int SolveOrder = 5) {
    detail::incr_convolution_raw(tstp, alpha, C, A, Acc, (const void *)F.ptr(-1), B, Bcc, beta, h, SolveOrder);
}
template <class HM>
void incr_convolution(int tstp, std::complex<double> alpha, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, double beta,
                      double h, int SolveOrder = 5) {
    detail::incr_convolution_raw(tstp, alpha, C, A, Acc, nullptr, B, Bcc, beta, h, SolveOrder);
}
// convolution_timestep_new (:4916-4976) and convolution_timestep_omp (:5808-5851): C's time step
// tstp zeroed, then incr_convolution with alpha = 1
template <class HM>
void convolution_timestep_new(int tstp, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, double beta, double h,
                              int SolveOrder = 5) {
    const long es = (long)C.size1() * C.size1();
    if (tstp < 0) {
        std::fill(C.matptr(0), C.matptr(0) + (C.ntau() + 1) * es, std::complex<double>(0.0));
    } else {  // C.set_timestep_zero(tstp): ret row, tv row, les column
        std::fill(C.retptr(tstp, 0), C.retptr(tstp, 0) + (tstp + 1) * es, std::complex<double>(0.0));
        std::fill(C.tvptr(tstp, 0), C.tvptr(tstp, 0) + (C.ntau() + 1) * es, std::complex<double>(0.0));
        std::fill(C.lesptr(0, tstp), C.lesptr(0, tstp) + (tstp + 1) * es, std::complex<double>(0.0));
    }
    detail::incr_convolution_raw(tstp, 1.0, C, A, Acc, nullptr, B, Bcc, beta, h, SolveOrder);
}
template <class HM>
void convolution_timestep_omp(int omp_num_threads, int tstp, HM &C, HM &A, HM &Acc, HM &B, HM &Bcc, double beta,
                              double h, int SolveOrder = 5) {
    (void)omp_num_threads;
    convolution_timestep_new(tstp, C, A, Acc, B, Bcc, beta, h, SolveOrder);
}
template <class HM>
void convolution_timestep_omp(int omp_num_threads, int tstp, HM &C, HM &A, HM &B, double beta, double h,
                              int SolveOrder = 5) {
    convolution_timestep_omp(omp_num_threads, tstp, C, A, A, B, B, beta, h, SolveOrder);
}

// cntr::dyson_timestep_omp(omp_num_threads, n, G, lam0, H, Sigma, beta, h, SolveOrder)
// (cntr_dyson_omp_decl.hpp, cntr_dyson_omp_impl.hpp:577-605): the OpenMP solver's
// discretization of the step, on the device; requires SolveOrder + 1 <= n
template <class HM, class FN>
void dyson_timestep_omp(int omp_num_threads, int n, HM &G, double lam0, FN &H, HM &Sigma, double beta, double h,
                        int SolveOrder = 5) {
    (void)omp_num_threads;
    nessi_hm_ptrs g = hm_ptrs(G), s = hm_ptrs(Sigma);
    check(nessi_gpu_dyson_timestep_omp_host(n, &g, &s, H.ptr(-1), lam0, G.nt(), G.ntau(), G.size1(), G.sig(),
                                            SolveOrder, beta, h));
}

// cntr::vie2_timestep_omp(omp_num_threads, tstp, G, F, Fcc, Q, beta, h, SolveOrder, matsubara_method)
// (cntr_vie2_impl.hpp:2125-2190): tstp = -1 vie2_mat, tstp <= SolveOrder a vie2_start of order
// tstp (as vie2_timestep above), else the element-parallel step
template <class HM>
void vie2_timestep_omp(int omp_num_threads, int tstp, HM &G, HM &F, HM &Fcc, HM &Q, double beta, double h,
                       int SolveOrder = 5, int matsubara_method = MAT_FIXPOINT) {
    (void)omp_num_threads;
    if (tstp <= SolveOrder) {
        vie2_timestep(tstp, G, F, Fcc, Q, beta, h, SolveOrder, matsubara_method);
        return;
    }
    nessi_hm_ptrs g = hm_ptrs(G), f = hm_ptrs(F), fcc = hm_ptrs(Fcc), q = hm_ptrs(Q);
    check(nessi_gpu_vie2_timestep_omp_host(tstp, &g, &f, &fcc, &q, G.nt(), G.ntau(), G.size1(), G.sig(), SolveOrder,
                                           beta, h));
}

}  // namespace cntr_gpu
