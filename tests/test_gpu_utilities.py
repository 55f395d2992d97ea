"""nessi_gpu_distance_norm2 (cntr::distance_norm2, cntr_utilities_impl.hpp:607-650) on device
herm_matrix data against the oracle's restatement, for every kind of time step."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix

pytestmark = pytest.mark.gpu


def _random_hm(rng, nt, ntau, s):
    G = herm_matrix(nt, ntau, s, -1)
    for comp in ("ret", "les", "tv", "mat"):
        a = getattr(G, comp)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    return G


@pytest.mark.parametrize("s", [1, 3])
def test_distance_norm2_matches_oracle(oracle, s):
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(90 + s)
    nt, ntau = 9, 7
    A, B = _random_hm(rng, nt, ntau, s), _random_hm(rng, nt, ntau, s)
    keep = []

    def dev(G):
        ptrs = []
        for comp in ("ret", "les", "tv", "mat"):
            t = torch.from_numpy(getattr(G, comp).copy()).cuda()
            keep.append(t)
            ptrs.append(t.data_ptr())
        return gpu.HmPtrs(*ptrs)

    da, db = dev(A), dev(B)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for tstp in (-1, 0, 4, nt):
        gpu.distance_norm2_dev(tstp, da, db, nt, ntau, s, out.data_ptr())
        torch.cuda.synchronize()
        ref = oracle.distance_norm2(tstp, A, B)
        assert abs(float(out.item()) - ref) <= 1e-12 * ref, (tstp, float(out.item()), ref)
