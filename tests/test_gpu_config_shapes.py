"""Parity at the full shapes of the benchmark configurations (the parity tests elsewhere use short
histories).  FP64 within 1e-10 and mixed precision within 1e-8 of the oracle, max|x - x_ref| /
max|x_ref| per component over every time step:

* config 0: the impurity quench end to end on the device (Matsubara solve, bootstrap and all
  steps) against the oracle run in the test;
* config 1: three k-points of the 2-band chain at its full shape (size1 2, nt 1000, ntau 600),
  every element against the oracle run in the test (OpenMP over the k-points);
* config 3: a size1 = 5 and a size1 = 8 problem at nt 500, ntau 400, and config 4: a 2 x 3
  k-subset of the lattice at its full per-k shape (nt 2000, ntau 800, 3 correctors), against
  golden projections of every time-step slice from the oracle (tests/golden/make_config_golden.py:
  its oracle runs take minutes).  A projection error bounds the slice error from below."""
import os

import numpy as np
import pytest

from builders import boot_to_full, component_errors, config3_problem, fingerprint_errors, fingerprints
from nessi_b200 import herm_matrix, workloads

pytestmark = pytest.mark.gpu
TOL64, TOLMIX = 1e-10, 1e-8
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_shapes.npz")


def _golden(case):
    d = np.load(GOLDEN)
    out = {}
    for key in d.files:
        c, name = key.split(".")
        if c == case:
            v = d[key]
            out[name] = float(v) if v.ndim == 0 else v
    return out


@pytest.mark.parametrize("prec", [0, 1])
def test_config0_impurity(oracle, prec):
    """Config 0 end to end on the device (dyson_mat, dyson_start, dyson_timestep n = 6..200)
    against the oracle's dyson_mat / dyson_start / dyson_timestep on the same Sigma and H."""
    from nessi_b200 import function, gpu
    W = workloads.config0()
    d = W.descs[0]
    nt, ntau, k = d["nt"], d["ntau"], W.k
    H = function(nt, 1)
    for t in range(-1, nt + 1):
        H.set_value(t, W.H[0, t + 1])
    ref = herm_matrix(nt, ntau, 1, -1)
    oracle.dyson_mat(ref, W.sigma, d["mu"], H, d["beta"], k)
    oracle.dyson_start(ref, d["mu"], H, W.sigma, d["beta"], d["h"], k)
    for n in range(k + 1, nt + 1):
        oracle.dyson_timestep(n, ref, d["mu"], H, W.sigma, d["beta"], d["h"], k)
    b = gpu.Batch(W.descs, precision=prec)
    b.set_sigma(0, W.sigma)
    b.set_H(0, H)
    b.dyson_mat()
    b.dyson_start()
    for n in range(k + 1, nt + 1):
        b.dyson_timestep(n)
    G = herm_matrix(nt, ntau, 1, -1)
    b.get_G(0, G)
    b.close()
    e = component_errors(G, ref, 0, nt)
    e["mat"] = float(np.max(np.abs(G.mat - ref.mat)) / np.max(np.abs(ref.mat)))
    assert max(e.values()) < (TOL64 if prec == 0 else TOLMIX), e


def test_config1_shape(oracle):
    from nessi_b200 import gpu
    W = workloads.chain(256, 1000, 600, 20.0, 0.01, 2, kslice=slice(37, 256, 101))
    d = W.descs[0]
    nt, k = d["nt"], W.k
    ref = [boot_to_full(W.boot[p], d) for p in range(W.nprob)]
    oracle.dyson_timestep_batch(k + 1, nt, ref, d["mu"], W.H, W.sigma, d["beta"], d["h"], k)
    for prec, tol in ((gpu.PREC_FP64, TOL64), (gpu.PREC_MIXED, TOLMIX)):
        b = gpu.Batch(W.descs, precision=prec)
        workloads.upload(b, W)
        for n in range(k + 1, nt + 1):
            b.dyson_timestep(n)
        for p in range(W.nprob):
            G = herm_matrix(nt, d["ntau"], 2, -1)
            b.get_G(p, G)
            e = component_errors(G, ref[p], k + 1, nt)
            assert max(e.values()) < tol, (prec, p, e)
        b.close()


@pytest.mark.parametrize("prec,pp", [(0, -1), (0, 100), (1, 0)])
def test_config3_large_orbitals(monkeypatch, prec, pp):
    """size1 5 and 8 in one batch (two Sigma groups): FP64 with the one-problem Volterra kernels
    and with the cluster recursion, and mixed precision with the autotuner's choice."""
    from nessi_b200 import gpu
    if pp:
        monkeypatch.setenv("NESSI_VOLTERRA_PP", str(pp))
    probs = [config3_problem(5, 500, 5005), config3_problem(8, 500, 8008)]
    descs = []
    for desc, H, Sig, boot in probs:
        desc = dict(desc, sigma_group=desc["size1"])
        descs.append(desc)
    b = gpu.Batch(descs, precision=prec)
    for p, (desc, H, Sig, boot) in enumerate(probs):
        b.set_sigma(desc["size1"], Sig)
        b.set_H(p, H)
        b.set_timestep(p, -1, boot.mat)
        for t in range(desc["solve_order"] + 1):
            b.set_timestep(p, t, boot.get_timestep(t))
    k = descs[0]["solve_order"]
    for n in range(k + 1, 501):
        b.dyson_timestep(n)
    tol = TOL64 if prec == 0 else TOLMIX
    for p, d in enumerate(descs):
        G = herm_matrix(d["nt"], d["ntau"], d["size1"], -1)
        b.get_G(p, G)
        e = fingerprint_errors(fingerprints(G, d["nt"]), _golden("c3_s%d" % d["size1"]))
        assert max(e.values()) < tol, (d["size1"], e)
    b.close()


@pytest.mark.parametrize("prec", [0, 1])
def test_config4_lattice_subset(prec):
    from nessi_b200 import gpu
    W = workloads.lattice2b(2, 3, 2000, 800, 20.0, 0.01)
    d = W.descs[0]
    b = gpu.Batch(W.descs, precision=prec)
    workloads.upload(b, W)
    b.lattice_2b_start(max_iter=8, tol=0.0)
    for n in range(W.k + 1, d["nt"] + 1):
        b.lattice_2b_timestep(n, W.ncorr)
    L = herm_matrix(d["nt"], d["ntau"], 1, -1)
    b.get_gloc(0, L)
    G0 = herm_matrix(d["nt"], d["ntau"], 1, -1)
    b.get_G(0, G0)
    b.close()
    tol = TOL64 if prec == 0 else TOLMIX
    for case, G in (("c4_gloc", L), ("c4_g0", G0)):
        e = fingerprint_errors(fingerprints(G, d["nt"]), _golden(case))
        assert max(e.values()) < tol, (case, e)
