"""Checkpoint and restart of a device batch in libcntr's text format (nessi_b200.hm_file): a batch
propagated to nt1 is checkpointed (download + print_to_file at precision 17), a new batch reads
time steps 0..nt1 back (read_from_file(nt1) + upload) and continues to nt; every problem equals
the uninterrupted propagation and the oracle."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import component_errors, make_H, make_sigma, rel_err, solve_oracle

pytestmark = pytest.mark.gpu


def restart_run(O, batch_cls, hm_file, tmp_path, nt=40, ntau=20, s=2, k=5, nt1=22, beta=3.0, h=0.05, mu=0.1):
    rng = np.random.default_rng(77)
    Sig = make_sigma(O, rng, nt, ntau, s, -1, beta, h)
    Hs, Go, Gb = [], [], []
    for _ in range(2):
        H = make_H(rng, nt, s, h)
        full, boot = solve_oracle(O, herm_matrix(nt, ntau, s, -1), H, Sig, mu, beta, h, k)
        Hs.append(H); Go.append(full); Gb.append(boot)
    descs = [dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h, mu=mu)] * 2

    def batch(start):
        b = batch_cls(descs)
        b.set_sigma(0, Sig)
        for p in range(2):
            b.set_H(p, Hs[p])
            b.set_G(p, start[p])
        return b

    whole = batch(Gb)
    for n in range(k + 1, nt + 1):
        whole.dyson_timestep(n)
    ref = [herm_matrix(nt, ntau, s, -1) for _ in range(2)]
    for p in range(2):
        whole.get_G(p, ref[p])
    whole.close()

    first = batch(Gb)
    for n in range(k + 1, nt1 + 1):
        first.dyson_timestep(n)
    files = [tmp_path / ("G%d.txt" % p) for p in range(2)]
    for p in range(2):
        hm_file.checkpoint(first, p, files[p])
    first.close()

    blank = [herm_matrix(nt, ntau, s, -1) for _ in range(2)]
    second = batch(blank)
    for p in range(2):
        hm_file.restart(second, p, nt1, files[p])
    for n in range(nt1 + 1, nt + 1):
        second.dyson_timestep(n)
    out = [herm_matrix(nt, ntau, s, -1) for _ in range(2)]
    for p in range(2):
        second.get_G(p, out[p])
    second.close()
    return out, ref, Go


def test_checkpoint_restart_continues_the_propagation(oracle, tmp_path):
    from nessi_b200 import gpu, hm_file
    out, ref, Go = restart_run(oracle, gpu.Batch, hm_file, tmp_path)
    for p in range(2):
        for c in ("ret", "les", "tv", "mat"):
            # the two batches may pick other (equally exact) Volterra kernels: rounding-level
            assert rel_err(getattr(out[p], c), getattr(ref[p], c)) < 1e-12, c
        e = component_errors(out[p], Go[p], 6, 40)
        assert max(e.values()) < 1e-10, e
