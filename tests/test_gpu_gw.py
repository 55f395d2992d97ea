"""The GW self-energy diagrams on the device (nessi_gpu_gw_polarization_timestep /
nessi_gpu_gw_sigma_timestep; examples/programs/gw_selfene_impl.cpp:114-153) against the oracle's
element-index restatement with the reference's k-point arithmetic, for every momentum and every
kind of time step, size1 1 and 2 (the element-by-element rule of the example)."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _random_hm(rng, nt, ntau, s, sig):
    G = herm_matrix(nt, ntau, s, sig)
    for comp in ("ret", "les", "tv", "mat"):
        a = getattr(G, comp)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    return G


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _table(hms, keep):
    """Device copies of the herm_matrix components (appended to keep, 4 per matrix) and a device
    table of their addresses in nessi_hm_ptrs order."""
    import torch
    rows = []
    for G in hms:
        ptrs = []
        for comp in ("ret", "les", "tv", "mat"):
            t = torch.from_numpy(getattr(G, comp).copy()).cuda()
            keep.append(t)
            ptrs.append(t.data_ptr())
        rows.append(ptrs)
    return torch.tensor(rows, dtype=torch.int64, device="cuda")  # nk x 4 device pointers


@pytest.mark.parametrize("s", [1, 2])
def test_gw_polarization_and_sigma_match_oracle(oracle, s):
    import torch
    from nessi_b200 import gpu
    rng = np.random.default_rng(1200 + s)
    nk, nt, ntau = 5, 7, 6
    Gs = [_random_hm(rng, nt, ntau, s, -1) for _ in range(nk)]
    Ws = [_random_hm(rng, nt, ntau, s, 1) for _ in range(nk)]
    w = rng.uniform(0.1, 0.3, nk)
    keep = []
    Gtab = _table(Gs, keep)
    Wtab = _table(Ws, keep)
    Ps = [herm_matrix(nt, ntau, s, 1) for _ in range(nk)]
    Ss = [herm_matrix(nt, ntau, s, -1) for _ in range(nk)]
    Pdev, Sdev = [], []
    Ptab = _table(Ps, Pdev)
    Stab = _table(Ss, Sdev)
    wd = torch.from_numpy(w).cuda()
    for tstp in (-1, 0, 3, nt):
        gpu.gw_polarization_timestep_dev(tstp, nk, Gtab.data_ptr(), Ptab.data_ptr(), wd.data_ptr(), nt, ntau, s, -1)
        gpu.gw_sigma_timestep_dev(tstp, nk, Gtab.data_ptr(), Wtab.data_ptr(), Stab.data_ptr(), wd.data_ptr(), nt, ntau, s)
        torch.cuda.synchronize()
        for q in range(nk):
            ref = herm_matrix(nt, ntau, s, 1)
            oracle.gw_polarization_timestep(tstp, ref, q, Gs, w)
            dev = Pdev[4 * q:4 * q + 4]
            got = herm_matrix(nt, ntau, s, 1)
            for i, comp in enumerate(("ret", "les", "tv", "mat")):
                getattr(got, comp)[...] = dev[i].cpu().numpy()
            a, b = got.get_timestep(tstp), ref.get_timestep(tstp)
            assert _rel(a, b) < TOL, ("P", q, tstp, _rel(a, b))
        for kk in range(nk):
            ref = herm_matrix(nt, ntau, s, -1)
            oracle.gw_sigma_timestep(tstp, ref, kk, Gs, Ws, w)
            dev = Sdev[4 * kk:4 * kk + 4]
            got = herm_matrix(nt, ntau, s, -1)
            for i, comp in enumerate(("ret", "les", "tv", "mat")):
                getattr(got, comp)[...] = dev[i].cpu().numpy()
            a, b = got.get_timestep(tstp), ref.get_timestep(tstp)
            assert _rel(a, b) < TOL, ("Sigma", kk, tstp, _rel(a, b))
