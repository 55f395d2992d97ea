"""libcntr's text herm_matrix format (nessi_b200.hm_file, libnessi_io.so) on CPU: the exact text
print_to_file writes (cntr_herm_matrix_impl.hpp:1308-1361), round trips, the read_from_file(nt1)
semantics (:1469-1560), the errors libcntr aborts on, and a restart from a checkpoint that
reproduces the uninterrupted propagation bit for bit."""
import numpy as np
import pytest

from nessi_b200 import herm_matrix
from nessi_b200 import hm_file
from builders import make_H, make_sigma, solve_oracle


@pytest.fixture(scope="module", autouse=True)
def _built():
    from nessi_b200 import build
    build.build_io()


def _random(rng, nt, ntau, s, sig):
    G = herm_matrix(nt, ntau, s, sig)
    for c in ("ret", "les", "tv", "mat"):
        a = getattr(G, c)
        a[...] = rng.normal(size=a.shape) + 1j * rng.normal(size=a.shape)
    return G


def test_text_is_the_reference_format(tmp_path):
    """Layout of print_to_file: header '# nt ntau size1  sig', mat lines and a blank line, then
    ret rows, tv rows and les columns, each block followed by a blank line and each component by
    one more; numbers as std::ostream prints them at the precision (16 by default)."""
    G = herm_matrix(1, 1, 1, -1)
    G.mat[:, 0, 0] = [0.5 - 0.25j, 2.0 + 1e-3j]
    G.ret[:, 0, 0] = [1.0 / 3.0, complex(-0.0, 0.0), 123456789012345678.0]
    G.tv[:, :, 0, 0] = [[1 + 1j, 2 + 2j], [3 + 3j, 4 + 4j]]
    G.les[:, 0, 0] = [-1j, 0.125, 7.0]
    f = tmp_path / "g.txt"
    hm_file.print_to_file(G, f)
    want = ("# 1 1 1  -1\n"
            "mat: 0 0.5 -0.25\n"
            "mat: 1 2 0.001\n"
            "\n"
            "ret: 0 0 0.3333333333333333 0\n"
            "\n"
            "ret: 1 0 -0 0\n"
            "ret: 1 1 1.234567890123457e+17 0\n"
            "\n"
            "\n"
            "tv: 0 0 1 1\n"
            "tv: 0 1 2 2\n"
            "\n"
            "tv: 1 0 3 3\n"
            "tv: 1 1 4 4\n"
            "\n"
            "\n"
            "les: 0 0 -0 -1\n"
            "\n"
            "les: 0 1 0.125 0\n"
            "les: 1 1 7 0\n"
            "\n"
            "\n")
    assert f.read_text() == want


@pytest.mark.parametrize("nt,s,sig", [(7, 2, 1), (0, 1, -1), (-1, 3, -1), (5, 3, -1)])
def test_round_trip(tmp_path, nt, s, sig):
    rng = np.random.default_rng(nt + 10 * s)
    G = _random(rng, nt, 6, s, sig)
    f = tmp_path / "g.txt"
    hm_file.print_to_file(G, f, precision=17)
    assert hm_file.file_header(f) == (nt, 6, s, sig)
    R = hm_file.read_from_file(f)
    for c in ("ret", "les", "tv", "mat"):
        assert np.array_equal(getattr(R, c), getattr(G, c)), c
    assert R.sig == sig
    hm_file.print_to_file(G, f)  # libcntr's default precision 16: within a unit of the 16th digit
    R = hm_file.read_from_file(f)
    for c in ("ret", "les", "tv", "mat"):
        a, b = getattr(R, c), getattr(G, c)
        assert np.all(np.abs(a - b) <= 2e-15 * np.abs(b) + 1e-300), c


def test_read_from_file_into_a_larger_matrix(tmp_path):
    """read_from_file(file) into a herm_matrix with more time steps: steps 0..nt_file are read,
    the others keep their values, and the sign comes from the file."""
    rng = np.random.default_rng(3)
    G = _random(rng, 4, 5, 2, 1)
    f = tmp_path / "g.txt"
    hm_file.print_to_file(G, f, 17)
    T = _random(rng, 9, 5, 2, -1)
    before = T.copy()
    hm_file.read_from_file(f, T)
    assert T.sig == 1
    for t in range(5):
        assert np.array_equal(T.get_timestep(t), G.get_timestep(t))
    assert np.array_equal(T.mat, G.mat)
    assert np.array_equal(T.ret_row(7), before.ret_row(7)) and np.array_equal(T.tv[9], before.tv[9])
    with pytest.raises(hm_file.HmFileError):
        hm_file.read_from_file(f, herm_matrix(3, 5, 2, 1))   # fewer time steps than the file
    with pytest.raises(hm_file.HmFileError):
        hm_file.read_from_file(f, herm_matrix(9, 4, 2, 1))   # other ntau


def test_read_from_file_nt1(tmp_path):
    rng = np.random.default_rng(4)
    G = _random(rng, 8, 5, 2, -1)
    f = tmp_path / "g.txt"
    hm_file.print_to_file(G, f, 17)
    nt1 = 4
    T = _random(rng, 10, 5, 2, 1)
    before = T.copy()
    hm_file.read_from_file_nt1(T, nt1, f)
    assert T.sig == 1  # the nt1 variant leaves the sign alone
    assert np.array_equal(T.mat, G.mat)
    for t in range(nt1 + 1):
        assert np.array_equal(T.ret_row(t), G.ret_row(t))
        assert np.array_equal(T.tv[t], G.tv[t])
        assert np.array_equal(T.les_col(t), G.les_col(t))
    for t in range(nt1 + 1, 11):
        assert np.array_equal(T.ret_row(t), before.ret_row(t))
        assert np.array_equal(T.tv[t], before.tv[t])
        assert np.array_equal(T.les_col(t), before.les_col(t))
    for bad in (9, 11):   # nt1 above the file's nt, above the matrix's nt
        with pytest.raises(hm_file.HmFileError):
            hm_file.read_from_file_nt1(herm_matrix(10, 5, 2, -1), bad, f)
    with pytest.raises(hm_file.HmFileError):
        hm_file.read_from_file_nt1(herm_matrix(10, 5, 1, -1), 3, f)


def test_malformed_files_raise(tmp_path):
    rng = np.random.default_rng(5)
    G = _random(rng, 3, 4, 1, -1)
    f = tmp_path / "g.txt"
    hm_file.print_to_file(G, f)
    text = f.read_text()
    cut = tmp_path / "cut.txt"
    cut.write_text(text[:text.index("tv: 2 1")])
    with pytest.raises(hm_file.HmFileError, match=r"error at tv \(2,1\)"):
        hm_file.read_from_file(cut)
    bad = tmp_path / "bad.txt"
    bad.write_text(text.replace("les: 1 2", "les: 1 2 x", 1))
    with pytest.raises(hm_file.HmFileError, match="error at les"):
        hm_file.read_from_file(bad)
    empty = tmp_path / "empty.txt"
    empty.write_text("")
    with pytest.raises(hm_file.HmFileError, match="error in file"):
        hm_file.read_from_file(empty)
    with pytest.raises(hm_file.HmFileError):
        hm_file.read_from_file(tmp_path / "missing.txt")


def test_restart_reproduces_the_propagation(oracle, tmp_path):
    """Propagate to nt1, checkpoint at precision 17, read the steps up to nt1 into a fresh
    herm_matrix and continue: every component equals the uninterrupted propagation exactly."""
    O = oracle
    rng = np.random.default_rng(6)
    nt, ntau, s, beta, h, k, mu, nt1 = 24, 12, 2, 3.0, 0.05, 5, 0.1, 13
    Sig = make_sigma(O, rng, nt, ntau, s, -1, beta, h)
    H = make_H(rng, nt, s, h)
    G = herm_matrix(nt, ntau, s, -1)
    full, boot = solve_oracle(O, G, H, Sig, mu, beta, h, k)
    part = boot.copy()
    for n in range(k + 1, nt1 + 1):
        O.dyson_timestep(n, part, mu, H, Sig, beta, h, k)
    f = tmp_path / "ckpt.txt"
    hm_file.print_to_file(part, f, precision=17)
    R = hm_file.read_from_file_nt1(herm_matrix(nt, ntau, s, -1), nt1, f)
    for n in range(nt1 + 1, nt + 1):
        O.dyson_timestep(n, R, mu, H, Sig, beta, h, k)
    for c in ("ret", "les", "tv", "mat"):
        assert np.array_equal(getattr(R, c), getattr(full, c)), c


def test_reference_read_write_cases(oracle, tmp_path):
    """libcntr/test/herm_matrix_member.cpp:472-506: a free 2 x 2 propagator (nt = 100, ntau = 50,
    beta = 5, h = 0.01) printed at precision 12 and read back whole, and up to nt1 = 50; the
    summed distance_norm2 stays below the reference's 1e-7."""
    from nessi_b200.herm_matrix import distance_norm2
    nt, ntau, s, beta, h = 100, 50, 2, 5.0, 0.01
    h0 = np.array([[-0.4, 0.1j], [-0.1j, 0.6]])
    G1 = herm_matrix(nt, ntau, s, -1)
    oracle.green_from_H(G1, 0.0, h0, beta, h)
    f = tmp_path / "herm_matrix_plain.dat"
    hm_file.print_to_file(G1, f, 12)
    G2 = hm_file.read_from_file(f, herm_matrix(nt, ntau, s, -1))
    assert sum(distance_norm2(t, G1, G2) for t in range(-1, nt + 1)) < 1e-7
    G3 = hm_file.read_from_file_nt1(herm_matrix(nt, ntau, s, -1), 50, f)
    assert sum(distance_norm2(t, G1, G3) for t in range(-1, 51)) < 1e-7


def test_format_against_the_reference_reader(tmp_path):
    """tests/golden/hm_text_small.{txt,json} (tests/golden/make_text_format_golden.py): the writer
    reproduces the committed text byte for byte, and the reader returns exactly what the
    reference's own Python reader (libcntr/python3/ReadCNTR.py read_gf) parsed from it."""
    import json
    import os
    import sys
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, golden)
    from make_text_format_golden import hm_text_values
    G = hm_text_values()
    f = tmp_path / "g.txt"
    hm_file.print_to_file(G, f, precision=17)
    txt = os.path.join(golden, "hm_text_small.txt")
    assert f.read_bytes() == open(txt, "rb").read()
    ref = json.load(open(os.path.join(golden, "hm_text_small.json")))

    def arr(c):
        return (np.array(ref[c]["re"]) + 1j * np.array(ref[c]["im"])).reshape(ref[c]["shape"])
    R = hm_file.read_from_file(txt)
    assert (R.nt, R.ntau, R.size1, R.sig) == (ref["nt"], ref["ntau"], ref["dim"], ref["sig"])
    assert np.array_equal(R.mat, arr("mat")) and np.array_equal(R.tv, arr("tv"))
    ret, les = arr("ret"), arr("les")
    for i in range(R.nt + 1):
        for j in range(i + 1):
            assert np.array_equal(R.get_ret(i, j), ret[i, j])
            assert np.array_equal(R.get_les(j, i), les[j, i])
    for c in ("ret", "les", "tv", "mat"):  # and both equal the values written
        assert np.array_equal(getattr(R, c), getattr(G, c))
