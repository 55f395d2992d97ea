"""CUDA-graph replay of the per-step launch sequence: a recorded propagation replays to the same
numbers as the eagerly launched one (and as the oracle), for Dyson batches and for the
self-consistent lattice."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from builders import make_H, make_lattice, make_sigma, rel_err, solve_oracle, component_errors, u_matrices

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("s,pp", [(2, None), (4, 101)])
def test_graph_replay_dyson(oracle, monkeypatch, s, pp):
    """pp = 101: the whole-GPU Volterra recursion, a cooperative launch with its barrier reset,
    inside the graph."""
    from nessi_b200 import gpu
    if pp is not None:
        monkeypatch.setenv("NESSI_VOLTERRA_PP", str(pp))
    rng = np.random.default_rng(21)
    nt, ntau, beta, h, k, mu = 60, 20, 4.0, 0.05, 5, 0.1
    Sig = make_sigma(oracle, rng, nt, ntau, s, -1, beta, h)
    Hs, Go, G0 = [], [], []
    for _ in range(3):
        H = make_H(rng, nt, s, h)
        Gf, Gb = solve_oracle(oracle, herm_matrix(nt, ntau, s, -1), H, Sig, mu, beta, h, k)
        Hs.append(H); Go.append(Gf); G0.append(Gb)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, beta=beta, h=h, mu=mu)] * 3)
    b.set_sigma(0, Sig)
    for p in range(3):
        b.set_G(p, G0[p])
        b.set_H(p, Hs[p])
    for n in range(k + 1, nt + 1):
        b.dyson_timestep(n)
    eager = [herm_matrix(nt, ntau, s, -1) for _ in range(3)]
    for p in range(3):
        b.get_G(p, eager[p])
    b.graph_record(b.GRAPH_DYSON, k + 1, nt)
    for _ in range(2):
        for p in range(3):                      # wipe the propagated steps, keep the bootstrap
            b.set_G(p, G0[p])
        b.graph_launch()
        b.synchronize()
        for p in range(3):
            Gg = herm_matrix(nt, ntau, s, -1)
            b.get_G(p, Gg)
            assert max(component_errors(Gg, eager[p], k + 1, nt).values()) < 1e-14
            assert max(component_errors(Gg, Go[p], k + 1, nt).values()) < 1e-10
    b.close()


def test_graph_replay_lattice(oracle):
    from nessi_b200 import gpu
    nt, ntau, beta, h, k = 30, 20, 5.0, 0.02, 5
    Gs, Hs, U = make_lattice(oracle, 3, 2, nt, ntau, beta, h, u_max=2.0, t_ramp=0.2)
    nk = len(Gs)
    b = gpu.Batch([dict(nt=nt, ntau=ntau, size1=1, sig=-1, solve_order=k, beta=beta, h=h)] * nk)
    for p in range(nk):
        b.set_G(p, Gs[p])
        b.set_H(p, Hs[p])
    b.set_sigma(0, herm_matrix(nt, ntau, 1, -1))
    b.set_U(0, U)
    b.lattice_2b_start(max_iter=6, tol=0.0)
    for n in range(k + 1, nt + 1):
        b.lattice_2b_timestep(n, 3)
    L_eager = herm_matrix(nt, ntau, 1, -1)
    b.get_gloc(0, L_eager)
    b.graph_record(b.GRAPH_LATTICE, k + 1, nt, 3)
    b.graph_launch()
    b.synchronize()
    L = herm_matrix(nt, ntau, 1, -1)
    b.get_gloc(0, L)
    b.close()
    assert max(component_errors(L, L_eager, 0, nt).values()) < 1e-14


def test_graph_launch_without_recording():
    from nessi_b200 import gpu
    b = gpu.Batch([dict(nt=10, ntau=8, size1=1, sig=-1, solve_order=5, beta=3.0, h=0.05)])
    with pytest.raises(gpu.NessiGpuError):
        b.graph_launch()
    b.close()
