"""Mixed-precision path (NESSI_PREC_MIXED): the G^tv history older than the k+1 backward-
difference rows is streamed from an FP32 copy, every sum and solve stays FP64.  Bound stated
by the workload: max relative error <= 1e-8 per component against the FP64 oracle."""
import numpy as np
import pytest

from builders import make_H, make_sigma, solve_oracle, component_errors
from nessi_b200 import herm_matrix

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-8


def _run(oracle, s, nt, ntau, npb, precision, seed, beta=10.0, h=0.02, k=5, mu=0.0):
    from nessi_b200 import gpu
    rng = np.random.default_rng(seed)
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    Hs, Go, G0 = [], [], []
    for _ in range(npb):
        H = make_H(rng, nt, s, h)
        G = herm_matrix(nt, ntau, s, -1)
        Gf, Gb = solve_oracle(oracle, G, H, Sig, mu, beta, h, k)
        Hs.append(H); Go.append(Gf); G0.append(Gb)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h, mu=mu)] * npb,
                  precision=precision)
    b.set_sigma(0, Sig)
    for p in range(npb):
        b.set_G(p, G0[p])
        b.set_H(p, Hs[p])
    for n in range(k + 1, nt + 1):
        b.dyson_timestep(n)
    b.synchronize()
    out = []
    for p in range(npb):
        Gg = herm_matrix(nt, ntau, s, -1)
        b.get_G(p, Gg)
        out.append(component_errors(Gg, Go[p], k + 1, nt))
    b.close()
    return out


@pytest.mark.parametrize("s,nt,ntau", [(1, 300, 100), (2, 120, 60), (4, 60, 30)])
def test_mixed_precision_within_bound(oracle, s, nt, ntau):
    from nessi_b200 import gpu
    errs = _run(oracle, s, nt, ntau, 2, gpu.PREC_MIXED, seed=40 + s)
    worst = {c: max(e[c] for e in errs) for c in errs[0]}
    print("mixed s=%d nt=%d: max rel err %s" % (s, nt, worst))
    for c, v in worst.items():
        assert v < MIXED_TOL, (c, v)


def test_fp64_long_run_parity(oracle):
    from nessi_b200 import gpu
    errs = _run(oracle, 1, 300, 100, 2, gpu.PREC_FP64, seed=41)
    worst = {c: max(e[c] for e in errs) for c in errs[0]}
    print("fp64 s=1 nt=300: max rel err %s" % worst)
    for c, v in worst.items():
        assert v < 1e-10, (c, v)
