// A libcntr-style program on include/cntr_gpu.hpp, for tests/test_gpu_whole_cxx.py: a
// herm_matrix / function pair with libcntr's accessors and layout, filled from raw files
// (complex128, libcntr layout), one cntr_gpu call, the result written back.
//
//   cxx_frontend <mode> <dir>      mode: echo | algebra | mat | dyson | steps | correct | vie2 | sin | conv
//
// Files in <dir>: dims.txt ("nt ntau size1 sig k beta h mu"), and <name>.{ret,les,tv,mat}
// for the herm_matrix operands (H.fn for the function).  The result is G (or C).
#include <complex>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "cntr_gpu.hpp"

typedef std::complex<double> cplx;

struct HM {
    int nt_, ntau_, s_, sig_;
    std::vector<cplx> r_, l_, t_, m_;
    HM(int nt, int ntau, int s, int sig)
        : nt_(nt), ntau_(ntau), s_(s), sig_(sig), r_((long)(nt + 1) * (nt + 2) / 2 * s * s), l_(r_.size()),
          t_((long)(nt + 1) * (ntau + 1) * s * s), m_((long)(ntau + 1) * s * s) {}
    int nt() const { return nt_; }
    int ntau() const { return ntau_; }
    int size1() const { return s_; }
    int sig() const { return sig_; }
    cplx *retptr(int i, int j) { return r_.data() + ((long)i * (i + 1) / 2 + j) * s_ * s_; }
    cplx *lesptr(int i, int j) { return l_.data() + ((long)j * (j + 1) / 2 + i) * s_ * s_; }
    cplx *tvptr(int i, int m) { return t_.data() + ((long)i * (ntau_ + 1) + m) * s_ * s_; }
    cplx *matptr(int m) { return m_.data() + (long)m * s_ * s_; }
};

struct FN {
    int nt_, s_;
    std::vector<cplx> d_;
    FN(int nt, int s) : nt_(nt), s_(s), d_((long)(nt + 2) * s * s) {}
    cplx *ptr(int t) { return d_.data() + (long)(t + 1) * s_ * s_; }
};

static void load(std::vector<cplx> &v, const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    f.read((char *)v.data(), (std::streamsize)(v.size() * sizeof(cplx)));
    if (f.gcount() != (std::streamsize)(v.size() * sizeof(cplx))) throw std::runtime_error("short file " + path);
}

static void save(const std::vector<cplx> &v, const std::string &path) {
    std::ofstream f(path, std::ios::binary);
    f.write((const char *)v.data(), (std::streamsize)(v.size() * sizeof(cplx)));
    if (!f) throw std::runtime_error("cannot write " + path);
}

static void load_hm(HM &G, const std::string &base) {
    load(G.r_, base + ".ret");
    load(G.l_, base + ".les");
    load(G.t_, base + ".tv");
    load(G.m_, base + ".mat");
}

static void save_hm(const HM &G, const std::string &base) {
    save(G.r_, base + ".ret");
    save(G.l_, base + ".les");
    save(G.t_, base + ".tv");
    save(G.m_, base + ".mat");
}

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s echo|algebra|mat|dyson|steps|correct|vie2|sin|omp|conv <dir>\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[1], dir = std::string(argv[2]) + "/";
    int nt, ntau, s, sig, k;
    double beta, h, mu;
    {
        std::ifstream f(dir + "dims.txt");
        if (!(f >> nt >> ntau >> s >> sig >> k >> beta >> h >> mu)) {
            std::fprintf(stderr, "bad dims.txt\n");
            return 2;
        }
    }
    try {
        HM G(nt, ntau, s, sig);
        if (mode == "echo") {  // the file handling alone (no device)
            load_hm(G, dir + "A");
            save_hm(G, dir + "out");
        } else if (mode == "algebra") {  // the host algebra of vie2_timestep_sin (no device)
            HM L(nt, ntau, s, sig), R(nt, ntau, s, sig);
            FN f(nt, s), inv(nt, s);
            load_hm(L, dir + "A");
            load_hm(R, dir + "A");
            load(f.d_, dir + "f.fn");
            for (int t = -1; t <= nt; t++) {
                cntr_gpu::detail::left_multiply(L, t, f.ptr(-1));
                cntr_gpu::detail::right_multiply(R, t, f.ptr(-1));
                std::vector<cplx> a(f.ptr(t), f.ptr(t) + s * s);
                for (int i = 0; i < s; i++) a[i * s + i] += 1.0;
                if (!cntr_gpu::detail::mat_inverse(s, a.data(), inv.ptr(t))) throw std::runtime_error("singular");
            }
            cntr_gpu::detail::decr_timestep(L, R, 2);
            save_hm(L, dir + "out");
            save_hm(R, dir + "outR");
            save(inv.d_, dir + "inv.fn");
        } else if (mode == "mat") {  // cntr::dyson_mat, also for a Matsubara-only G (nt = -1)
            HM Sigma(nt, ntau, s, sig);
            FN H(nt, s);
            load_hm(Sigma, dir + "Sigma");
            load(H.d_, dir + "H.fn");
            cntr_gpu::dyson_mat(G, mu, H, Sigma, beta, k);
            save_hm(G, dir + "out");
        } else if (mode == "dyson" || mode == "steps") {
            HM Sigma(nt, ntau, s, sig);
            FN H(nt, s);
            load_hm(Sigma, dir + "Sigma");
            load(H.d_, dir + "H.fn");
            if (mode == "dyson") {
                cntr_gpu::dyson(G, mu, H, Sigma, beta, h, k);
            } else {  // the single-call forms, one time step at a time
                cntr_gpu::dyson_mat(G, mu, H, Sigma, beta, k);
                cntr_gpu::dyson_start(G, mu, H, Sigma, beta, h, k);
                for (int n = k + 1; n <= nt; n++) cntr_gpu::dyson_timestep(n, G, mu, H, Sigma, beta, h, k);
            }
            save_hm(G, dir + "out");
        } else if (mode == "correct") {  // the single-call step in a predictor-corrector loop
            HM Sigma(nt, ntau, s, sig);
            FN H(nt, s);
            load_hm(Sigma, dir + "Sigma");
            load(H.d_, dir + "H.fn");
            cntr_gpu::dyson_mat(G, mu, H, Sigma, beta, k);
            cntr_gpu::dyson_start(G, mu, H, Sigma, beta, h, k);
            const long es = (long)s * s;
            long long first = -1, most = 0;
            for (int n = k + 1; n <= nt; n++) {
                // Sigma's time step n is recomputed between the calls (here: scaled copies of it)
                std::vector<cplx> r0(Sigma.retptr(n, 0), Sigma.retptr(n, 0) + (n + 1) * es);
                std::vector<cplx> t0(Sigma.tvptr(n, 0), Sigma.tvptr(n, 0) + (ntau + 1) * es);
                std::vector<cplx> l0(Sigma.lesptr(0, n), Sigma.lesptr(0, n) + (n + 1) * es);
                for (int it = 0; it < 3; it++) {
                    const double f = 1.0 + 0.001 * (it - 1);
                    for (size_t i = 0; i < r0.size(); i++) Sigma.retptr(n, 0)[i] = f * r0[i];
                    for (size_t i = 0; i < t0.size(); i++) Sigma.tvptr(n, 0)[i] = f * t0[i];
                    for (size_t i = 0; i < l0.size(); i++) Sigma.lesptr(0, n)[i] = f * l0[i];
                    const long long before = cntr_gpu::transfer_bytes();
                    cntr_gpu::dyson_timestep(n, G, mu, H, Sigma, beta, h, k);
                    const long long moved = cntr_gpu::transfer_bytes() - before;
                    if (first < 0) first = moved; else if (moved > most) most = moved;
                }
            }
            std::ofstream(dir + "bytes.txt") << first << " " << most << "\n";
            save_hm(G, dir + "out");
        } else if (mode == "vie2") {
            HM F(nt, ntau, s, sig), Fcc(nt, ntau, s, sig), Q(nt, ntau, s, sig);
            load_hm(F, dir + "F");
            load_hm(Fcc, dir + "Fcc");
            load_hm(Q, dir + "Q");
            cntr_gpu::vie2_timestep(-1, G, F, Fcc, Q, beta, h, k);  // vie2_mat
            cntr_gpu::vie2_start(G, F, Fcc, Q, beta, h, k);
            for (int n = k + 1; n <= nt; n++) cntr_gpu::vie2_timestep(n, G, F, Fcc, Q, beta, h, k);
            save_hm(G, dir + "out");
        } else if (mode == "sin") {  // vie2_timestep_sin through a propagation
            HM F(nt, ntau, s, sig), Fcc(nt, ntau, s, sig), Q(nt, ntau, s, sig);
            FN Fsin(nt, s), Qsin(nt, s), Gsin(nt, s);
            load_hm(F, dir + "F");
            load_hm(Fcc, dir + "Fcc");
            load_hm(Q, dir + "Q");
            load(Fsin.d_, dir + "Fsin.fn");
            load(Qsin.d_, dir + "Qsin.fn");
            cntr_gpu::vie2_timestep_sin(-1, G, Gsin, F, Fcc, Fsin, Q, Qsin, beta, h, k);
            for (int n = k; n <= nt; n++) cntr_gpu::vie2_timestep_sin(n, G, Gsin, F, Fcc, Fsin, Q, Qsin, beta, h, k);
            save_hm(G, dir + "out");
            save(Gsin.d_, dir + "out.fn");
        } else if (mode == "omp") {  // the OpenMP-path drop-ins: dyson_timestep_omp, vie2_timestep_omp
            HM Sigma(nt, ntau, s, sig), F(nt, ntau, s, sig), Fcc(nt, ntau, s, sig), G0(nt, ntau, s, sig);
            HM A(nt, ntau, s, sig), B(nt, ntau, s, sig), C(nt, ntau, s, sig);
            FN H(nt, s);
            load_hm(Sigma, dir + "Sigma");
            load(H.d_, dir + "H.fn");
            load_hm(G, dir + "G");  // bootstrap (mat and steps 0..k) of the Dyson problem
            for (int n = k + 1; n <= nt; n++) cntr_gpu::dyson_timestep_omp(4, n, G, mu, H, Sigma, beta, h, k);
            save_hm(G, dir + "out");
            // vie2_timestep_omp for every step -1..nt (the reference dispatches n <= k)
            load_hm(F, dir + "F");
            load_hm(Fcc, dir + "Fcc");
            load_hm(G0, dir + "Q");
            HM V(nt, ntau, s, sig);
            for (int n = -1; n <= nt; n++) {
                if (n == 0) continue;  // vie2_start of order n for 1 <= n <= k writes steps 0..n
                cntr_gpu::vie2_timestep_omp(4, n, V, F, Fcc, G0, beta, h, k);
            }
            save_hm(V, dir + "outV");
            // convolution_timestep_omp of the step k + 3
            load_hm(A, dir + "Sigma");
            load_hm(B, dir + "Q");
            cntr_gpu::convolution_timestep_omp(4, k + 3, C, A, B, beta, h, k);
            // C += (0.5 - 0.25i) A * F * B at steps -1 and k + 1 with the function F of the case
            FN Ff(nt, s);
            load(Ff.d_, dir + "Ff.fn");
            for (int n : {-1, k + 1})
                cntr_gpu::incr_convolution(n, cplx(0.5, -0.25), C, A, A, Ff, B, B, beta, h, k);
            save_hm(C, dir + "outC");
        } else if (mode == "conv") {
            HM A(nt, ntau, s, sig), Acc(nt, ntau, s, sig), B(nt, ntau, s, sig);
            load_hm(A, dir + "A");
            load_hm(Acc, dir + "Acc");
            load_hm(B, dir + "B");
            cntr_gpu::convolution(G, A, Acc, B, B, beta, h, k);  // B hermitian: Bcc = B
            save_hm(G, dir + "out");
        } else {
            std::fprintf(stderr, "unknown mode %s\n", mode.c_str());
            return 2;
        }
    } catch (const std::exception &e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
