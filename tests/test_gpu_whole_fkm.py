"""The GPU time stepping against libcntr's own output: the Falicov-Kimball Bethe-lattice quench of
libcntr/test/fkm_bethe_quench.cpp with the Matsubara solution and the bootstrap from the oracle
and every time step t = 6..50 on the GPU: G0 and G1 are one batch sharing Sigma = Delta; per
step the host extrapolates Delta (the predictor), uploads it with nessi_gpu_set_sigma_timestep,
and three times runs nessi_gpu_dyson_timestep, downloads the two slices and uploads the new
Delta(t) = (G0(t) + G1(t)) / 2.  The densities must equal libcntr's (the golden values of
fkm_bethe_quench.h5) as closely as the oracle does."""
import numpy as np
import pytest

from test_oracle_fkm import BETA, H, ITER_RTIME, KT, NT, NTAU, ERRMAX, fkm_equilibrium_and_bootstrap, golden

pytestmark = pytest.mark.gpu


def propagate(O, batch_cls):
    s = fkm_equilibrium_and_bootstrap(O)
    desc = dict(nt=NT, ntau=NTAU, size1=1, sig=-1, solve_order=KT, beta=BETA, h=H, mu=s.mu)
    b = batch_cls([desc, desc])
    b.set_G(0, s.G0)
    b.set_G(1, s.G1)
    b.set_H(0, s.f0)
    b.set_H(1, s.f1)
    b.set_sigma(0, s.Delta)
    for t in range(KT + 1, NT + 1):
        O.extrapolate_timestep(t - 1, s.Delta, KT)
        b.set_sigma_timestep(0, t, s.Delta.get_timestep(t))
        for _ in range(ITER_RTIME):
            b.dyson_timestep(t)
            for p, Gp in ((0, s.G0), (1, s.G1)):
                out = np.zeros((2 * (t + 1) + NTAU + 1, 1, 1), np.complex128)
                b.get_timestep(p, t, out)
                Gp.set_timestep_data(t, out)
            s.mix(t)
            s.Delta.set_timestep(t, s.G)
            b.set_sigma_timestep(0, t, s.Delta.get_timestep(t))
    b.close()
    return s.densities()


def test_fkm_time_stepping_on_gpu_matches_libcntr(oracle):
    from nessi_b200 import gpu
    ref = golden()
    d0, d1 = propagate(oracle, gpu.Batch)
    e0, e1 = np.abs(d0 - ref["den0"]), np.abs(d1 - ref["den1"])
    assert np.sum(e0 ** 2) < ERRMAX and np.sum(e1 ** 2) < ERRMAX   # fkm_bethe_quench.cpp:145-151
    assert max(e0.max(), e1.max()) < 1e-11                         # as close as the oracle (4.8e-13)
