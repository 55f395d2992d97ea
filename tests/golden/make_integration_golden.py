"""Extract the reference's hard-coded integration tables into a JSON fixture.

libcntr ships the Gregory start/sigma/omega weights, the backward-differentiation
weights and the Matsubara boundary correction ``rcorr`` as decimal literals in
``libcntr/cntr/integration.cpp`` (``read_gregory_weights`` :152-808,
``read_bd_weights`` :815-900, ``read_rcorr`` :905-1180).  This script reads that
file as text and writes ``integration_tables.json`` beside itself, assembled the
way ``read_gregory_weights`` lays them out for the ``Integrator`` class
(integration.cpp:794-806): a (2k+2) x (2k+2) row-major matrix whose rows m < k+1
are the start weights and rows k+1..2k+1 hold sigma followed by omega.

The fixture is the golden data that pins ``nessi_b200.tables`` (exact-rational
derivation used by the CUDA library) and the oracle's own derivation.

Usage:  NESSI_REFERENCE_ROOT=<reference checkout> python tests/golden/make_integration_golden.py [path/to/integration.cpp]
"""
import json
import os
import re
import sys

# default source: under NESSI_REFERENCE_ROOT, the reference checkout (the directory holding
# libcntr/); a path given as the first argument overrides it
DEFAULT_SRC = os.path.join(os.environ.get("NESSI_REFERENCE_ROOT", "."), "libcntr/cntr/integration.cpp")


def _cases(body):
    """Split a switch body into {case_number: text}."""
    parts = re.split(r"\bcase\s+(\d+)\s*:", body)
    out = {}
    for i in range(1, len(parts), 2):
        out[int(parts[i])] = parts[i + 1]
    return out


def _assignments(text, name):
    vals = {}
    for m in re.finditer(name + r"\[\s*([0-9+\s]+)\s*\]\s*=\s*([-+0-9.eE]+)\s*;", text):
        idx = eval(m.group(1))  # indices look like "16+3"
        vals[idx] = m.group(2)
    return vals


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC
    text = open(src).read()
    g0 = text.index("void read_gregory_weights(int k,double *w)")
    b0 = text.index("void read_bd_weights(int k,double *w)")
    r0 = text.index("void read_rcorr(int k,double *w)")
    greg_body, bd_body, rc_body = text[g0:b0], text[b0:r0], text[r0:]

    gregory = {}
    for k, t in _cases(greg_body).items():
        k1 = k + 1
        k2 = 2 * k1
        start = _assignments(t, "start")
        sigma = _assignments(t, "sigma")
        omega = _assignments(t, "omega")
        w = [["0"] * k2 for _ in range(k2)]
        for n in range(k1):
            for i in range(k1):
                w[n][i] = start.get(k1 * n + i, "0")
        for n in range(k1):
            for i in range(k1):
                w[k1 + n][i] = sigma[k1 * n + i]
            for i in range(k1, k1 + n + 1):
                w[k1 + n][i] = omega[k1 + n - i]
        gregory[str(k)] = {"weights": w, "omega": [omega[j] for j in range(k1)]}

    bd = {}
    for k, t in _cases(bd_body).items():
        a = _assignments(t, "alpha")
        bd[str(k)] = [a[i] for i in range(len(a))]

    rcorr = {}
    for k, t in _cases(rc_body).items():
        a = _assignments(t, "w")
        rcorr[str(k)] = [a[i] for i in range(len(a))]

    out = {
        "source": "libcntr/cntr/integration.cpp (read_gregory_weights, read_bd_weights, read_rcorr)",
        "note": "decimal strings exactly as written in the reference; gregory rows laid out as in "
                "integration.cpp:794-806; rcorr index (m-1)*(k+1)^2 + j*(k+1) + l",
        "gregory": gregory,
        "bd": bd,
        "rcorr": rcorr,
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "integration_tables.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", dst)


if __name__ == "__main__":
    main()
