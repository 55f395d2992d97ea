"""The tv row's two kernels for size1 <= 4: k_tv_stream (history read into shared memory by bulk
copies; NESSI_TV_KERNEL=stream) against k_tv (register loads, the default) on the same inputs, and
the bounded-wait path of the stream kernel.  The two kernels sum the same terms in a different
order, so they agree to rounding: max|x - y| / max|y| < 1e-12 per component.  Parity of the default
path with the oracle is in test_gpu_dyson.py / test_gpu_vie2.py / test_gpu_config_shapes.py."""
import numpy as np
import pytest

from builders import make_H, make_sigma, rel_err
from nessi_b200 import herm_matrix, workloads

pytestmark = pytest.mark.gpu


def _propagate(oracle, monkeypatch, kernel, s, nprob, nt, ntau, prec, seed, nts=None):
    from nessi_b200 import gpu
    monkeypatch.setenv("NESSI_TV_KERNEL", kernel)
    rng = np.random.default_rng(seed)
    beta, h, k, mu = 5.0, 0.04, 5, 0.1
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    nts = nts or [nt] * nprob
    b = gpu.Batch([dict(nt=t, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h, mu=mu) for t in nts],
                  precision=prec)
    b.set_sigma(0, Sig)
    for p in range(nprob):
        H = make_H(rng, nts[p], s, h)
        b.set_H(p, H)
        boot = workloads.bootstrap_free(H.get_value(-1), mu, beta, h, k, ntau)  # any ntau, odd included
        b.set_timestep(p, -1, boot.mat)
        for t in range(k + 1):
            b.set_timestep(p, t, boot.get_timestep(t))
    for n in range(k + 1, nt + 1):
        b.dyson_timestep(n)
    b.synchronize()
    out = []
    for p in range(nprob):
        G = herm_matrix(nts[p], ntau, s, -1)
        b.get_G(p, G)
        out.append(G)
    b.close()
    return out


@pytest.mark.parametrize("s,nprob,nt,ntau", [(1, 3, 30, 300), (1, 160, 16, 101), (2, 5, 24, 60), (3, 2, 20, 41),
                                             (4, 3, 18, 32)])
@pytest.mark.parametrize("prec", [0, 1])
def test_stream_matches_register_kernel(oracle, monkeypatch, s, nprob, nt, ntau, prec):
    """Odd and even ntau + 1 (odd: FP32 segments that start 8 bytes past a 16-byte boundary), one
    chunk per problem (160 problems) and several, FP64 and mixed precision; the bootstrap is the
    free propagator of H(-1)."""
    a = _propagate(oracle, monkeypatch, "stream", s, nprob, nt, ntau, prec, seed=s)
    r = _propagate(oracle, monkeypatch, "regs", s, nprob, nt, ntau, prec, seed=s)
    for p in range(nprob):
        for comp in ("ret", "les", "tv", "mat"):
            e = rel_err(getattr(a[p], comp), getattr(r[p], comp))
            assert e < 1e-12, (p, comp, e)


def test_stream_uneven_batch(oracle, monkeypatch):
    """Problems with different nt in one group: only the first nact (nt >= n) are items."""
    nts = [22, 17, 9, 22]
    a = _propagate(oracle, monkeypatch, "stream", 2, 4, 22, 45, 1, seed=9, nts=nts)
    r = _propagate(oracle, monkeypatch, "regs", 2, 4, 22, 45, 1, seed=9, nts=nts)
    for p in range(4):
        assert rel_err(a[p].tv, r[p].tv) < 1e-12


def test_stream_wait_timeout_is_reported(oracle, monkeypatch):
    """A wait bound of 0 makes the stream kernel's waits give up at once: the kernel waits for its
    copies in flight, returns, and the next synchronize reports NESSI_ERR_TIMEOUT once."""
    from nessi_b200 import gpu
    monkeypatch.setenv("NESSI_TV_KERNEL", "stream")
    rng = np.random.default_rng(3)
    nt, ntau, beta, h, k = 12, 20, 5.0, 0.04, 5
    Sig = make_sigma(oracle, rng, nt, ntau, 1, -1, beta, h)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=1, sig=-1, solve_order=k, beta=beta, h=h, mu=0.0)] * 2)
    b.set_sigma(0, Sig)
    for p in range(2):
        H = make_H(rng, nt, 1, h)
        b.set_H(p, H)
        boot = workloads.bootstrap_free(H.get_value(-1), 0.0, beta, h, k, ntau)
        b.set_timestep(p, -1, boot.mat)
        for t in range(k + 1):
            b.set_timestep(p, t, boot.get_timestep(t))
    b.synchronize()
    b.set_wait_limit(0)
    b.dyson_timestep(k + 1)
    with pytest.raises(gpu.NessiGpuError) as ei:
        b.synchronize()
    assert ei.value.code == 5
    b.synchronize()  # the condition was cleared
    b.set_wait_limit(2_000_000_000)
    b.dyson_timestep(k + 1)
    b.synchronize()
    b.close()
