"""Golden vectors for libcntr's herm_matrix text format: a small herm_matrix with closed-form
entries (hm_text_values below) is written by nessi_b200.hm_file.print_to_file (precision 17)
into tests/golden/hm_text_small.txt, and that file is parsed by the reference's own Python reader,
libcntr/python3/ReadCNTR.py:read_gf, whose arrays go to tests/golden/hm_text_small.json.
tests/test_hm_file.py then checks the writer against the text and the reader against read_gf.

ReadCNTR.py uses np.int, which numpy 2 no longer has; the script supplies it as the builtin int
for the duration of the call (the reference file itself is not touched).

    NESSI_REFERENCE_ROOT=<reference checkout> python tests/golden/make_text_format_golden.py [path/to/libcntr/python3]
"""
import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# default source: under NESSI_REFERENCE_ROOT, the reference checkout (the directory holding
# libcntr/); a path given as the first argument overrides it
DEFAULT_SRC = os.path.join(os.environ.get("NESSI_REFERENCE_ROOT", "."), "libcntr/python3")
TXT = os.path.join(HERE, "hm_text_small.txt")
JSN = os.path.join(HERE, "hm_text_small.json")
NT, NTAU, S, SIG = 3, 2, 2, -1


def hm_text_values():
    """The herm_matrix of the fixture: entries from a closed formula with signs, zeros and a
    wide range of magnitudes, so that the number formatting is exercised."""
    sys.path.insert(0, ROOT)
    from nessi_b200 import herm_matrix
    G = herm_matrix(NT, NTAU, S, SIG)
    for c, arr in (("ret", G.ret), ("les", G.les), ("tv", G.tv), ("mat", G.mat)):
        flat = arr.reshape(-1)
        for i in range(flat.size):
            x = (i + 1) * (1 + len(c))
            flat[i] = complex((-1) ** i * x / 7.0 * 10.0 ** (i % 5 - 2), (i % 3 - 1) * 3.0 ** (-i))
    return G


def main(src):
    sys.path.insert(0, ROOT)
    from nessi_b200 import hm_file
    G = hm_text_values()
    hm_file.print_to_file(G, TXT, precision=17)
    spec = importlib.util.spec_from_file_location("ReadCNTR", os.path.join(src, "ReadCNTR.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    had = hasattr(np, "int")
    np.int = int
    try:
        d = mod.read_gf(TXT)
    finally:
        if not had:
            del np.int
    out = {"source": "libcntr/python3/ReadCNTR.py read_gf of hm_text_small.txt",
           "nt": int(d.nt), "ntau": int(d.ntau), "dim": int(d.dim), "sig": int(d.foo)}
    for c in ("ret", "les", "tv", "mat"):
        a = np.asarray(getattr(d, c))
        out[c] = {"shape": list(a.shape), "re": a.real.reshape(-1).tolist(), "im": a.imag.reshape(-1).tolist()}
    with open(JSN, "w") as fh:
        json.dump(out, fh)
    print("wrote", TXT, JSN)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC)
