"""nessi_gpu_dyson_mat_noalloc: dyson_mat for one problem on caller-owned device memory with
scratch in a fixed device array.  Callers whose device memory belongs to another allocator (a
framework's memory pool, an arena sized at start-up), or that must not take the device-wide
synchronisation a cudaMalloc / cudaFree can bring, cannot let the library allocate; this entry
point serves them.  Its output must equal the oracle's dyson_mat (the CPU restatement of
cntr::dyson_mat, fixpoint method) within the tolerance of the GPU tests, and the batch API's
dyson_mat, on two calls in a row (the second call reuses the scratch the first one left)."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix, function
from nessi_b200.equilibrium import green_from_H

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _problem(seed, s, ntau, beta, sig):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.7, (s, s)) + 1j * rng.normal(0, 0.7, (s, s))
    Sig = herm_matrix(-1, ntau, s, sig)
    green_from_H(Sig, 0.0 if sig < 0 else -4.0, (x + x.conj().T) / 2, beta, 0.05)
    Sig.mat *= 0.3
    y = rng.normal(0, 0.8, (s, s)) + 1j * rng.normal(0, 0.8, (s, s))
    H0 = (y + y.conj().T) / 2
    if sig > 0:  # bosons: levels well above the chemical potential
        H0 = H0 + 4.0 * np.eye(s)
    return Sig, H0


def _batch_api(Sig, H0, s, ntau, beta, mu, k, sig):
    from nessi_b200 import gpu
    b = gpu.Batch([dict(nt=k, ntau=ntau, size1=s, sig=sig, solve_order=k, beta=beta, h=0.05, mu=mu)])
    S = herm_matrix(k, ntau, s, sig)
    S.mat[...] = Sig.mat
    b.set_sigma(0, S)
    H = np.zeros((k + 2, s, s), np.complex128)
    H[:] = H0
    b.set_H(0, H)
    b.dyson_mat()
    G = herm_matrix(k, ntau, s, sig)
    b.get_G(0, G)
    b.close()
    return G.mat


def _oracle(O, Sig, H0, s, ntau, beta, mu, k, sig):
    S = herm_matrix(k, ntau, s, sig)
    S.mat[...] = Sig.mat
    H = function(k, s)
    for t in range(-1, k + 1):
        H.set_value(t, H0)
    G = herm_matrix(k, ntau, s, sig)
    O.dyson_mat(G, S, mu, H, beta, k)
    return G.mat


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("s,sig", [(1, -1), (2, -1), (2, 1)])
def test_dyson_mat_noalloc_matches_oracle(oracle, s, sig):
    import torch
    from nessi_b200 import gpu
    ntau, beta, k = 40, 5.0, 5
    for call, (seed, mu) in enumerate([(1, 0.1), (2, -0.3)]):
        Sig, H0 = _problem(seed + 10 * s, s, ntau, beta, sig)
        ref = _oracle(oracle, Sig, H0, s, ntau, beta, mu, k, sig)
        api = _batch_api(Sig, H0, s, ntau, beta, mu, k, sig)
        H_d = torch.from_numpy(H0.reshape(1, s, s).copy()).cuda()
        S_d = torch.from_numpy(Sig.mat.copy()).cuda()
        G_d = torch.zeros((ntau + 1, s, s), dtype=torch.complex128, device="cuda")
        gpu.dyson_mat_noalloc(ntau, s, sig, k, beta, mu, H_d.data_ptr(), S_d.data_ptr(), G_d.data_ptr(), 0)
        torch.cuda.synchronize()
        out = G_d.cpu().numpy()
        assert _rel(out, ref) < TOL, (call, _rel(out, ref))
        assert _rel(out, api) < TOL, (call, _rel(out, api))


def test_dyson_mat_noalloc_rejects_oversize():
    import torch
    from nessi_b200 import gpu
    G_d = torch.zeros(4, dtype=torch.complex128, device="cuda")
    # scratch: 6 (ntau+1) + 2 ntau complex values beyond the fixed array
    with pytest.raises(gpu.NessiGpuError) as e:
        gpu.dyson_mat_noalloc(200000, 1, -1, 5, 5.0, 0.0, G_d.data_ptr(), G_d.data_ptr(), G_d.data_ptr(), 0)
    assert e.value.code == 1
    # fits the scratch array, but its 2 ntau twiddle factors (32 ntau bytes) exceed the shared
    # memory a block may use; rejected before anything is launched
    with pytest.raises(gpu.NessiGpuError) as e:
        gpu.dyson_mat_noalloc(16000, 1, -1, 5, 5.0, 0.0, G_d.data_ptr(), G_d.data_ptr(), G_d.data_ptr(), 0)
    assert e.value.code == 1
