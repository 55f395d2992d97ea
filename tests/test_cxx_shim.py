"""include/cntr_gpu.hpp (the libcntr-side front end) compiles against a herm_matrix-like class
with libcntr's public accessors and links against libnessi_gpu.so (no GPU needed)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MOCK = r'''
#include <complex>
#include <string>
#include <vector>
#include "cntr_gpu.hpp"
typedef std::complex<double> cplx;
struct HM {  // the accessors of cntr::herm_matrix<double> used by cntr_gpu.hpp
    int nt_, ntau_, s_, sig_;
    std::vector<cplx> r_, l_, t_, m_;
    HM(int nt, int ntau, int s, int sig) : nt_(nt), ntau_(ntau), s_(s), sig_(sig),
        r_((nt + 1) * (nt + 2) / 2 * s * s), l_(r_.size()), t_((nt + 1) * (ntau + 1) * s * s), m_((ntau + 1) * s * s) {}
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
    FN(int nt, int s) : nt_(nt), s_(s), d_((nt + 2) * s * s) {}
    cplx *ptr(int t) { return d_.data() + (long)(t + 1) * s_ * s_; }
};
int main(int argc, char **argv) {
    if (argc == 2 && std::string(argv[1]) == "io") {  // text checkpoint round trip, no GPU needed
        HM A(7, 5, 2, 1), B(9, 5, 2, 1);
        for (size_t i = 0; i < A.t_.size(); i++) A.t_[i] = cplx(0.1 * i, -1.0 / (i + 1));
        for (size_t i = 0; i < A.r_.size(); i++) { A.r_[i] = cplx(i, 2.0 / 3); A.l_[i] = cplx(-1.0 / 7, i); }
        for (size_t i = 0; i < A.m_.size(); i++) A.m_[i] = cplx(1e-300 * i, 3.0);
        cntr_gpu::print_to_file(A, "ckpt.txt", 17);
        cntr_gpu::read_from_file(B, 4, "ckpt.txt");
        for (int t = 0; t <= 4; t++)
            for (int j = 0; j <= 5; j++)
                for (int e = 0; e < 4; e++)
                    if (B.tvptr(t, j)[e] != A.tvptr(t, j)[e]) return 3;
        for (int j = 0; j <= 4; j++)
            for (int e = 0; e < 4; e++)
                if (B.retptr(4, j)[e] != A.retptr(4, j)[e] || B.lesptr(j, 4)[e] != A.lesptr(j, 4)[e]) return 4;
        if (B.tvptr(5, 0)[0] != cplx(0, 0)) return 5;  // steps after nt1 untouched
        try {
            cntr_gpu::read_from_file(B, 8, "ckpt.txt");  // nt1 beyond the file
            return 6;
        } catch (const std::runtime_error &) {
        }
        return 0;
    }
    if (argc < 2) return 0;  // link check only
    HM G(12, 10, 2, -1), S(12, 10, 2, -1);
    FN H(12, 2);
    cntr_gpu::dyson_mat(G, 0.0, H, S, 5.0, 5);
    cntr_gpu::dyson_start(G, 0.0, H, S, 5.0, 0.05, 5);
    cntr_gpu::dyson_timestep(6, G, 0.0, H, S, 5.0, 0.05, 5);
    HM F(12, 10, 2, -1), Q(12, 10, 2, -1), C(12, 10, 2, -1);
    cntr_gpu::vie2_start(G, F, F, Q, 5.0, 0.05, 5);
    cntr_gpu::vie2_timestep(6, G, F, F, Q, 5.0, 0.05, 5);
    cntr_gpu::vie2_timestep(-1, G, F, F, Q, 5.0, 0.05, 5);
    cntr_gpu::vie2_timestep(3, G, F, F, Q, 5.0, 0.05);
    cntr_gpu::vie2_mat(G, F, F, Q, 5.0, 5);
    cntr_gpu::vie2(G, F, F, Q, 5.0, 0.05, 5);
    cntr_gpu::dyson(G, 0.0, H, S, 5.0, 0.05, 5);
    cntr_gpu::extrapolate_timestep(7, G, 5);
    cntr_gpu::convolution_timestep(6, C, G, G, S, S, 5.0, 0.05, 5);
    cntr_gpu::convolution_timestep(6, C, G, S, 5.0, 0.05, 5);
    cntr_gpu::convolution(C, G, G, S, S, 5.0, 0.05, 5);
    cntr_gpu::convolution(C, G, S, 5.0, 0.05);
    return 0;
}
'''


def test_cntr_gpu_header_compiles_and_links(tmp_path):
    from nessi_b200 import build
    build.build()
    src = tmp_path / "mock.cpp"
    src.write_text(MOCK)
    exe = tmp_path / "mock"
    libdir = os.path.join(ROOT, "nessi_b200")
    cmd = ["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
           "-L", libdir, "-lnessi_gpu", "-lnessi_io", "-Wl,-rpath," + libdir]
    subprocess.check_call(cmd)
    assert exe.exists()
    # the checkpoint functions of the front end run without a GPU
    assert subprocess.call([str(exe), "io"], cwd=tmp_path) == 0
    assert (tmp_path / "ckpt.txt").read_text().startswith("# 7 5 2  1\n")
