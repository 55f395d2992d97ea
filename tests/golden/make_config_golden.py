"""Golden fingerprints of the oracle at the full shapes of the benchmark configurations, for
GPU parity tests whose oracle runs would take minutes (tests/test_gpu_config_shapes.py):

* config 3 (uneven batch): one problem of size1 = 5 and one of size1 = 8, nt = 500, ntau = 400,
  beta = 10, h = 0.01 (tests/builders.py:config3_problem), propagated from the free bootstrap;
* config 4 (self-consistent lattice): a 2 x 3 k-subset of the square lattice with config 4's
  per-k shape (nt = 2000, ntau = 800, beta = 20, h = 0.01, U ramped to 2, 3 correctors), the
  bootstrap iterated 9 times (nessi_b200/workloads.py:lattice2b).

The oracle (oracle/, the CPU restatement of libcntr's serial path) solves each case; the file
keeps the slice projections of tests/builders.py:fingerprints (G of the config-3 problems, G_loc
and G of the first k-point of the lattice) and the per-component maxima.

    python tests/golden/make_config_golden.py        # writes tests/golden/config_shapes.npz
"""
import os
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

import oracle as O  # noqa: E402
from builders import boot_to_full, config3_problem, fingerprints, u_matrices  # noqa: E402
from nessi_b200 import herm_matrix, workloads  # noqa: E402

CONFIG3 = [(5, 500, 5005), (8, 500, 8008)]   # (size1, nt, seed)
LATTICE = dict(nkx=2, nky=3, nt=2000, ntau=800, beta=20.0, h=0.01, max_iter=8)


def run_config3(s, nt, seed, out):
    desc, H, Sig, boot = config3_problem(s, nt, seed)
    G = boot_to_full(boot, desc)
    k = desc["solve_order"]
    for n in range(k + 1, nt + 1):
        O.dyson_timestep(n, G, desc["mu"], H, Sig, desc["beta"], desc["h"], k)
    out["c3_s%d" % s] = fingerprints(G, nt)


def run_lattice(out):
    L = LATTICE
    W = workloads.lattice2b(L["nkx"], L["nky"], L["nt"], L["ntau"], L["beta"], L["h"])
    d0 = W.descs[0]
    Gs = [boot_to_full(W.boot[p], d0) for p in range(W.nprob)]
    Gloc = herm_matrix(d0["nt"], d0["ntau"], 1, -1)
    Sig = herm_matrix(d0["nt"], d0["ntau"], 1, -1)
    Um = u_matrices(W.U)
    O.lattice2b_start(Gs, Gloc, Sig, Um, 0.0, W.H, L["beta"], L["h"], W.k, max_iter=L["max_iter"], tol=0.0)
    for n in range(W.k + 1, d0["nt"] + 1):
        O.lattice2b_timestep(n, Gs, Gloc, Sig, Um, 0.0, W.H, L["beta"], L["h"], W.k, ncorr=W.ncorr)
    out["c4_gloc"] = fingerprints(Gloc, d0["nt"])
    out["c4_g0"] = fingerprints(Gs[0], d0["nt"])


def main(path=os.path.join(HERE, "config_shapes.npz")):
    out = {}
    t0 = time.time()
    threads = [threading.Thread(target=run_config3, args=(s, nt, seed, out)) for s, nt, seed in CONFIG3]
    threads.append(threading.Thread(target=run_lattice, args=(out,)))
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    flat = {}
    for case, fp in out.items():
        for key, val in fp.items():
            flat["%s.%s" % (case, key)] = np.asarray(val)
    np.savez_compressed(path, **flat)
    print("wrote %s (%d arrays) in %.0f s" % (path, len(flat), time.time() - t0))


if __name__ == "__main__":
    main()
