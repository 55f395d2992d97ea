"""nessi_gpu_dyson_mat_noalloc: dyson_mat for one problem on caller-owned device memory with
scratch in a fixed device array.  Callers that run under stream capture, or whose device memory
belongs to another allocator, cannot let the library call cudaMalloc; this entry point serves
them.  Its output must equal the batch API's dyson_mat within the tolerance of the GPU tests,
on two calls in a row (the second call reuses the scratch the first one left)."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from nessi_b200.equilibrium import green_from_H

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _problem(seed, s, ntau, beta):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.7, (s, s)) + 1j * rng.normal(0, 0.7, (s, s))
    Sig = herm_matrix(-1, ntau, s, -1)
    green_from_H(Sig, 0.0, (x + x.conj().T) / 2, beta, 0.05)
    Sig.mat *= 0.3
    y = rng.normal(0, 0.8, (s, s)) + 1j * rng.normal(0, 0.8, (s, s))
    return Sig, (y + y.conj().T) / 2


def _reference(Sig, H0, s, ntau, beta, mu, k):
    from nessi_b200 import gpu
    b = gpu.Batch([dict(nt=k, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=0.05, mu=mu)])
    S = herm_matrix(k, ntau, s, -1)
    S.mat[...] = Sig.mat
    b.set_sigma(0, S)
    H = np.zeros((k + 2, s, s), np.complex128)
    H[:] = H0
    b.set_H(0, H)
    b.dyson_mat()
    G = herm_matrix(k, ntau, s, -1)
    b.get_G(0, G)
    b.close()
    return G.mat


def test_dyson_mat_noalloc_matches_batch_api():
    import torch
    from nessi_b200 import gpu
    s, ntau, beta, k = 2, 40, 5.0, 5
    for call, (seed, mu) in enumerate([(1, 0.1), (2, -0.3)]):
        Sig, H0 = _problem(seed, s, ntau, beta)
        ref = _reference(Sig, H0, s, ntau, beta, mu, k)
        H_d = torch.from_numpy(H0.reshape(1, s, s).copy()).cuda()
        S_d = torch.from_numpy(Sig.mat.copy()).cuda()
        G_d = torch.zeros((ntau + 1, s, s), dtype=torch.complex128, device="cuda")
        gpu.dyson_mat_noalloc(ntau, s, -1, k, beta, mu, H_d.data_ptr(), S_d.data_ptr(), G_d.data_ptr(), 0)
        torch.cuda.synchronize()
        out = G_d.cpu().numpy()
        err = np.max(np.abs(out - ref)) / np.max(np.abs(ref))
        assert err < TOL, (call, err)


def test_dyson_mat_noalloc_rejects_oversize():
    import torch
    from nessi_b200 import gpu
    G_d = torch.zeros(4, dtype=torch.complex128, device="cuda")
    with pytest.raises(gpu.NessiGpuError):
        gpu.dyson_mat_noalloc(200000, 1, -1, 5, 5.0, 0.0, G_d.data_ptr(), G_d.data_ptr(), G_d.data_ptr(), 0)
