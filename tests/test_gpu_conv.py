"""GPU parity of convolution_timestep on device-resident herm_matrix data through the C ABI
(cntr_convolution_impl.hpp:594-1803): C = A * B at every time step n = -1..nt (including the
start region n < k and the Acc/Bcc continuations), batched over problems, against the oracle at
1e-10; and the known-answer identity of libcntr/test/convolution.cpp (free propagators,
A * B = (A - B)/(wa - wb)) computed on the GPU at the reference's tolerance."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import rand_herm, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-10


class DevHM:
    """A herm_matrix copied to device memory (torch tensors hold the allocation)."""

    def __init__(self, G):
        import torch
        self.G = G
        self.t = {c: torch.from_numpy(np.ascontiguousarray(getattr(G, c))).cuda() for c in ("ret", "les", "tv", "mat")}

    def ptrs(self):
        return tuple(self.t[c].data_ptr() if self.t[c].numel() else 0 for c in ("ret", "les", "tv", "mat"))

    def host(self):
        out = herm_matrix(self.G.nt, self.G.ntau, self.G.size1, self.G.sig)
        for c in ("ret", "les", "tv", "mat"):
            getattr(out, c)[...] = self.t[c].cpu().numpy()
        return out


def make_sigma(O, rng, nt, ntau, s, sig, beta, h, lam):
    """lam^2 times the free propagator of a random hermitian level matrix; bosons get levels
    shifted above the chemical potential so that their occupations stay finite."""
    G = herm_matrix(nt, ntau, s, sig)
    O.green_from_H(G, -3.0 if sig == 1 else 0.0, rand_herm(rng, s, 0.7) + np.diag(rng.uniform(-1, 1, s)), beta, h)
    for t in range(-1, nt + 1):
        G.smul(t, lam * lam)
    return G


def _pair(O, rng, nt, ntau, s, sig, beta, h, k):
    """A non-hermitian A = X * Y with its partner Acc = Y * X."""
    X = make_sigma(O, rng, nt, ntau, s, sig, beta, h, lam=0.7)
    Y = make_sigma(O, rng, nt, ntau, s, sig, beta, h, lam=0.6)
    A, Acc = herm_matrix(nt, ntau, s, sig), herm_matrix(nt, ntau, s, sig)
    O.convolution_matsubara(A, X, Y, beta, k)
    O.convolution_matsubara(Acc, Y, X, beta, k)
    for t in range(nt + 1):
        O.convolution_timestep(t, A, X, X, Y, Y, beta, h, k)
        O.convolution_timestep(t, Acc, Y, Y, X, X, beta, h, k)
    return A, Acc


@pytest.mark.parametrize("s,sig,k", [(1, -1, 5), (2, -1, 5), (3, 1, 4), (5, -1, 5), (2, 1, 2)])
def test_convolution_matches_oracle(oracle, s, sig, k):
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(300 + 10 * s + k)
    nt, ntau, beta, h = 14, 12, 3.0, 0.05
    probs = []
    for _ in range(3):
        A, Acc = _pair(oracle, rng, nt, ntau, s, sig, beta, h, k)
        B = make_sigma(oracle, rng, nt, ntau, s, sig, beta, h, lam=0.9)
        probs.append((A, Acc, B))
    dev = [(DevHM(herm_matrix(nt, ntau, s, sig)), DevHM(A), DevHM(Acc), DevHM(B)) for A, Acc, B in probs]
    for n in range(-1, nt + 1):
        gpu.convolution_timestep_dev(n, [d[0].ptrs() for d in dev], [d[1].ptrs() for d in dev],
                                     [d[2].ptrs() for d in dev], [d[3].ptrs() for d in dev],
                                     [d[3].ptrs() for d in dev], nt, ntau, s, sig, sig, k, beta, h)
    torch.cuda.synchronize()
    for (A, Acc, B), d in zip(probs, dev):
        R = herm_matrix(nt, ntau, s, sig)
        for n in range(-1, nt + 1):
            oracle.convolution_timestep(n, R, A, Acc, B, B, beta, h, k)
        C = d[0].host()
        for comp in ("ret", "les", "tv", "mat"):
            assert rel_err(getattr(C, comp), getattr(R, comp)) < TOL, comp


@pytest.mark.parametrize("sig", [-1, 1])
def test_convolution_free_propagators_on_gpu(oracle, sig):
    """libcntr/test/convolution.cpp: for free propagators A, B of levels wa, wb,
    A * B = (A - B)/(wa - wb); the reference accepts a summed distance of 4e-6."""
    import torch
    from nessi_b200 import gpu
    O = oracle
    nt, ntau, beta, h, wa, wb, k = 7, 500, 5.0, 0.01, 1.123, 0.345, 5
    A, B = herm_matrix(nt, ntau, 1, sig), herm_matrix(nt, ntau, 1, sig)
    O.green_from_H(A, 0.0, np.array([[wa]]), beta, h)
    O.green_from_H(B, 0.0, np.array([[wb]]), beta, h)
    X = A.copy()
    for t in range(-1, nt + 1):
        X.incr_timestep(t, B, -1.0)
        X.smul(t, 1.0 / (wa - wb))
    dC, dA, dB = DevHM(herm_matrix(nt, ntau, 1, sig)), DevHM(A), DevHM(B)
    for t in range(-1, nt + 1):
        gpu.convolution_timestep_dev(t, [dC.ptrs()], [dA.ptrs()], [dA.ptrs()], [dB.ptrs()], [dB.ptrs()], nt, ntau, 1,
                                     sig, sig, k, beta, h)
    torch.cuda.synchronize()
    C = dC.host()
    err = sum(O.distance_norm2(t, X, C) for t in range(-1, nt + 1))
    assert err < 1e-6 * 4, err


def test_convolution_rejects_bad_arguments():
    from nessi_b200 import gpu
    with pytest.raises(gpu.NessiGpuError):
        gpu.convolution_timestep_dev(3, [(0, 0, 0, 0)], [(0, 0, 0, 0)], [(0, 0, 0, 0)], [(0, 0, 0, 0)],
                                     [(0, 0, 0, 0)], 10, 8, 1, -1, -1, 5, 3.0, 0.05)
    with pytest.raises(gpu.NessiGpuError):
        gpu.convolution_timestep_dev(11, [], [], [], [], [], 10, 8, 1, -1, -1, 5, 3.0, 0.05)


def test_convolution_host_dropin(oracle):
    """gpu.convolution_timestep with libcntr's signature on host herm_matrix objects."""
    from nessi_b200 import gpu
    rng = np.random.default_rng(9)
    nt, ntau, beta, h, k, s = 10, 8, 2.0, 0.05, 5, 2
    A, Acc = _pair(oracle, rng, nt, ntau, s, -1, beta, h, k)
    B = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h, lam=0.8)
    C, R = herm_matrix(nt, ntau, s, -1), herm_matrix(nt, ntau, s, -1)
    for n in range(-1, nt + 1):
        gpu.convolution_timestep(n, C, A, Acc, B, B, beta, h, k)
        oracle.convolution_timestep(n, R, A, Acc, B, B, beta, h, k)
    for comp in ("ret", "les", "tv", "mat"):
        assert rel_err(getattr(C, comp), getattr(R, comp)) < TOL, comp

