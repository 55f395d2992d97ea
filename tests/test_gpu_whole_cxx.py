"""include/cntr_gpu.hpp used as a libcntr program uses it, on the GPU: tests/cxx_frontend.cpp holds
a herm_matrix / function pair with libcntr's accessors and layout and calls cntr_gpu::dyson,
the single-call dyson_mat / dyson_start / dyson_timestep loop, vie2_timestep (n = -1, then
n > k) with vie2_start, and cntr_gpu::convolution; the results are checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import component_errors, make_H, make_sigma, rel_err, solve_oracle
from test_gpu_conv import _pair
from test_gpu_vie2 import _kernel_pair, _oracle_vie2, _source

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.join(ROOT, "tests")
TOL = 1e-10


def build_frontend(tmp_path):
    # links the libraries as built (no rebuild here: other tests of this process have them loaded)
    libdir = os.path.join(ROOT, "nessi_b200")
    for lib in ("libnessi_gpu.so", "libnessi_io.so"):
        assert os.path.exists(os.path.join(libdir, lib)), lib + " missing: run python -m nessi_b200.build"
    exe = tmp_path / "cxx_frontend"
    subprocess.check_call(["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                           os.path.join(HERE, "cxx_frontend.cpp"), "-o", str(exe), "-L", libdir, "-lnessi_gpu",
                           "-lnessi_io", "-Wl,-rpath," + libdir])
    return exe


def write_case(d, dims, **hms):
    d.mkdir(parents=True, exist_ok=True)
    (d / "dims.txt").write_text(" ".join(str(x) for x in dims) + "\n")
    for name, G in hms.items():
        if isinstance(G, np.ndarray):
            np.ascontiguousarray(G, np.complex128).tofile(str(d / (name + ".fn")))
            continue
        for c in ("ret", "les", "tv", "mat"):
            np.ascontiguousarray(getattr(G, c)).tofile(str(d / ("%s.%s" % (name, c))))


def read_out(d, nt, ntau, s, sig):
    G = herm_matrix(nt, ntau, s, sig)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(G, c)
        a[...] = np.fromfile(str(d / ("out." + c)), np.complex128).reshape(a.shape)
    return G


def run(exe, mode, d):
    r = subprocess.run([str(exe), mode, str(d)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("nt", [6, -1])
def test_file_handling_without_device(tmp_path, nt):
    """The program's own file round trip (mode echo), which needs no GPU."""
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(1)
    A = herm_matrix(nt, 5, 2, -1)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(A, c)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    d = tmp_path / "echo"
    write_case(d, (nt, 5, 2, -1, 5, 1.0, 0.1, 0.0), A=A)
    run(exe, "echo", d)
    B = read_out(d, nt, 5, 2, -1)
    for c in ("ret", "les", "tv", "mat"):
        assert np.array_equal(getattr(A, c), getattr(B, c))


def test_vie2_sin_host_algebra_without_device(tmp_path):
    """The host half of cntr_gpu::vie2_timestep_sin (mode algebra, no GPU): left and right
    multiplication by a function at every time step, the inverses of 1 + f(t), and the slice
    subtraction, against the Python herm_matrix and numpy."""
    from nessi_b200 import function
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(5)
    nt, ntau, s = 6, 4, 3
    A = herm_matrix(nt, ntau, s, -1)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(A, c)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    f = function(nt, s)
    f.data[...] = 0.4 * (rng.normal(size=f.data.shape) + 1j * rng.normal(size=f.data.shape))
    d = tmp_path / "algebra"
    write_case(d, (nt, ntau, s, -1, 5, 1.0, 0.1, 0.0), A=A, f=f.data)
    run(exe, "algebra", d)
    L, R = A.copy(), A.copy()
    for t in range(-1, nt + 1):
        L.left_multiply(t, f)
        R.right_multiply(t, f)
    L.incr_timestep(2, R, -1.0)
    got_R = herm_matrix(nt, ntau, s, -1)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(got_R, c)
        a[...] = np.fromfile(str(d / ("outR." + c)), np.complex128).reshape(a.shape)
    got_L = read_out(d, nt, ntau, s, -1)
    for c in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(got_L, c), getattr(L, c)) < 1e-14, c
        assert rel_err(getattr(got_R, c), getattr(R, c)) < 1e-14, c
    inv = np.fromfile(str(d / "inv.fn"), np.complex128).reshape(f.data.shape)
    assert rel_err(inv, np.linalg.inv(np.eye(s) + f.data)) < 1e-13


@pytest.mark.gpu
def test_vie2_timestep_sin_through_the_cxx_frontend(oracle, tmp_path):
    from nessi_b200 import function
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(59)
    nt, ntau, s, beta, h, k = 14, 12, 2, 3.0, 0.05, 5
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    Fsin, Qsin = function(nt, s), function(nt, s)
    Fsin.data[...] = 0.3 * (rng.normal(size=Fsin.data.shape) + 1j * rng.normal(size=Fsin.data.shape))
    Qsin.data[...] = rng.normal(size=Qsin.data.shape) + 1j * rng.normal(size=Qsin.data.shape)
    R, Rsin = herm_matrix(nt, ntau, s, -1), function(nt, s)
    for n in [-1] + list(range(k, nt + 1)):
        oracle.vie2_timestep_sin(n, R, Rsin, F, Fcc, Fsin, Q, Qsin, beta, h, k)
    d = tmp_path / "sin"
    write_case(d, (nt, ntau, s, -1, k, beta, h, 0.0), F=F, Fcc=Fcc, Q=Q, Fsin=Fsin.data, Qsin=Qsin.data)
    run(exe, "sin", d)
    G = read_out(d, nt, ntau, s, -1)
    Gsin = np.fromfile(str(d / "out.fn"), np.complex128).reshape(Rsin.data.shape)
    assert rel_err(Gsin, Rsin.data) < 1e-13
    for c in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(G, c), getattr(R, c)) < TOL, c


@pytest.mark.gpu
def test_dyson_mat_of_a_matsubara_only_matrix(oracle, tmp_path):
    """cntr_gpu::dyson_mat on herm_matrix(-1, ntau, 2, -1), as libcntr programs call it for the
    equilibrium alone."""
    from nessi_b200 import function
    from builders import rand_herm
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(53)
    ntau, s, beta, k, mu = 100, 2, 5.0, 5, 0.1
    Sig = herm_matrix(-1, ntau, s, -1)
    oracle.green_from_H(Sig, 0.0, rand_herm(rng, s, 0.7), beta, 1.0)
    Sig.smul(-1, 0.3)
    H = function(-1, s)
    H.set_value(-1, rand_herm(rng, s, 0.8))
    ref = herm_matrix(-1, ntau, s, -1)
    oracle.dyson_mat(ref, Sig, mu, H, beta, k)
    d = tmp_path / "mat"
    write_case(d, (-1, ntau, s, -1, k, beta, 1.0, mu), Sigma=Sig, H=H.data)
    run(exe, "mat", d)
    G = read_out(d, -1, ntau, s, -1)
    assert rel_err(G.mat, ref.mat) < TOL


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["dyson", "steps"])
def test_dyson_through_the_cxx_frontend(oracle, tmp_path, mode):
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(41)
    nt, ntau, s, beta, h, k, mu = 20, 16, 2, 3.0, 0.05, 5, 0.1
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    H = make_H(rng, nt, s, h)
    ref, _ = solve_oracle(oracle, herm_matrix(nt, ntau, s, -1), H, Sig, mu, beta, h, k)
    d = tmp_path / mode
    write_case(d, (nt, ntau, s, -1, k, beta, h, mu), Sigma=Sig, H=getattr(H, "data", H))
    run(exe, mode, d)
    G = read_out(d, nt, ntau, s, -1)
    assert rel_err(G.mat, ref.mat) < TOL
    e = component_errors(G, ref, 0, nt)
    assert max(e.values()) < TOL, e


@pytest.mark.gpu
def test_single_call_step_in_a_corrector_loop(oracle, tmp_path):
    """cntr_gpu::dyson_timestep called three times per time step with Sigma's time step n changed
    between the calls (a predictor-corrector driver): the device copy is kept, each call after
    the first moves O(n) data (Sigma's and G's slice n and H), and G equals the oracle's run of
    the same call sequence."""
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(43)
    nt, ntau, s, beta, h, k, mu = 50, 16, 2, 3.0, 0.05, 5, 0.1
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    H = make_H(rng, nt, s, h)
    d = tmp_path / "correct"
    write_case(d, (nt, ntau, s, -1, k, beta, h, mu), Sigma=Sig, H=getattr(H, "data", H))
    run(exe, "correct", d)
    G = read_out(d, nt, ntau, s, -1)
    ref = herm_matrix(nt, ntau, s, -1)
    oracle.dyson_mat(ref, Sig, mu, H, beta, k)
    oracle.dyson_start(ref, mu, H, Sig, beta, h, k)
    S = Sig.copy()
    for n in range(k + 1, nt + 1):
        orig = S.get_timestep(n).copy()
        for it in range(3):
            S.set_timestep_data(n, orig * (1.0 + 0.001 * (it - 1)))
            oracle.dyson_timestep(n, ref, mu, H, S, beta, h, k)
    e = component_errors(G, ref, 0, nt)
    assert max(e.values()) < TOL, e
    first, most = (int(x) for x in open(d / "bytes.txt").read().split())
    slice_bytes = 16 * (2 * (nt + 1) + ntau + 1) * s * s
    assert most <= 2 * slice_bytes + 16 * (nt + 2) * s * s, (first, most)
    assert first > 20 * most


@pytest.mark.gpu
def test_vie2_through_the_cxx_frontend(oracle, tmp_path):
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(43)
    nt, ntau, s, beta, h, k = 20, 16, 2, 4.0, 0.05, 5
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    ref, _ = _oracle_vie2(oracle, F, Fcc, Q, beta, h, k)
    d = tmp_path / "vie2"
    write_case(d, (nt, ntau, s, -1, k, beta, h, 0.0), F=F, Fcc=Fcc, Q=Q)
    run(exe, "vie2", d)
    G = read_out(d, nt, ntau, s, -1)
    assert rel_err(G.mat, ref.mat) < TOL
    e = component_errors(G, ref, 0, nt)
    assert max(e.values()) < TOL, e


@pytest.mark.gpu
def test_convolution_through_the_cxx_frontend(oracle, tmp_path):
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(47)
    nt, ntau, s, beta, h, k = 12, 10, 2, 2.0, 0.05, 5
    A, Acc = _pair(oracle, rng, nt, ntau, s, -1, beta, h, k)
    B = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.8)
    R = herm_matrix(nt, ntau, s, -1)
    for n in range(-1, nt + 1):
        oracle.convolution_timestep(n, R, A, Acc, B, B, beta, h, k)
    d = tmp_path / "conv"
    write_case(d, (nt, ntau, s, -1, k, beta, h, 0.0), A=A, Acc=Acc, B=B)
    run(exe, "conv", d)
    C = read_out(d, nt, ntau, s, -1)
    for c in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(C, c), getattr(R, c)) < TOL, c


def _read_prefix(d, prefix, nt, ntau, s, sig):
    G = herm_matrix(nt, ntau, s, sig)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(G, c)
        a[...] = np.fromfile(str(d / ("%s.%s" % (prefix, c))), np.complex128).reshape(a.shape)
    return G


@pytest.mark.gpu
def test_omp_dropins_through_the_cxx_frontend(oracle, tmp_path):
    """cntr_gpu::dyson_timestep_omp (n = k+1..nt), cntr_gpu::vie2_timestep_omp (n = -1, 1..nt, with
    the reference's dispatch of n <= k), cntr_gpu::convolution_timestep_omp and
    cntr_gpu::incr_convolution with a function F from a libcntr-style program, against the
    oracle's restatement of the OpenMP path."""
    exe = build_frontend(tmp_path)
    rng = np.random.default_rng(53)
    nt, ntau, s, beta, h, k, mu = 22, 14, 2, 3.0, 0.05, 4, 0.1
    Sigma = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.6)
    H = make_H(rng, nt, s, h)
    G = herm_matrix(nt, ntau, s, -1)
    oracle.dyson_mat(G, Sigma, mu, H, beta, k)
    oracle.dyson_start(G, mu, H, Sigma, beta, h, k)
    F, Fcc = _kernel_pair(oracle, rng, nt, ntau, s, beta, h, k)
    Q = _source(oracle, rng, nt, ntau, s, beta, h)
    Ff = np.zeros((nt + 2, s, s), np.complex128)
    x = rng.normal(0, 0.4, (s, s)) + 1j * rng.normal(0, 0.4, (s, s))
    for t in range(-1, nt + 1):
        Ff[t + 1] = np.eye(s) + np.sin(0.2 * t) * x
    d = tmp_path / "omp"
    write_case(d, (nt, ntau, s, -1, k, beta, h, mu), Sigma=Sigma, G=G, F=F, Fcc=Fcc, Q=Q, H=H.data, Ff=Ff)
    run(exe, "omp", d)
    refG = G.copy()
    for n in range(k + 1, nt + 1):
        oracle.dyson_timestep_omp(n, refG, mu, H, Sigma, beta, h, k)
    refV = herm_matrix(nt, ntau, s, -1)
    for n in range(-1, nt + 1):
        if n != 0:
            oracle.vie2_timestep_omp(n, refV, F, Fcc, Q, beta, h, k)
    refC = herm_matrix(nt, ntau, s, -1)
    oracle.convolution_timestep_new(k + 3, refC, Sigma, Sigma, Q, Q, beta, h, k)
    for n in (-1, k + 1):
        oracle.incr_convolution(n, 0.5 - 0.25j, refC, Sigma, Sigma, Q, Q, beta, h, k, ft=Ff)
    for prefix, ref in (("out", refG), ("outV", refV), ("outC", refC)):
        got = _read_prefix(d, prefix, nt, ntau, s, -1)
        for c in ("ret", "les", "tv", "mat"):
            assert rel_err(getattr(got, c), getattr(ref, c)) < TOL, (prefix, c)
