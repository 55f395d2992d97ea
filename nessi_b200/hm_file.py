"""libcntr's plain-text herm_matrix files (herm_matrix::print_to_file / read_from_file,
cntr_herm_matrix_impl.hpp:1308-1560) for checkpoint and restart of a propagation.

The format is the reference's, so a file written here is read by libcntr and its Python tools
and vice versa; the work is done by libnessi_io.so (nessi_b200/csrc/hm_text_io.cpp).  A device
batch is checkpointed by downloading a problem's G and printing it, and restarted by reading
its time steps up to nt1 (``read_from_file(nt1, file)`` semantics) and uploading them; the
propagation then continues at nt1 + 1.  Precision 17 makes the text round trip exact, so a
restarted propagation reproduces the uninterrupted one bit for bit; libcntr's default is 16.
"""
import ctypes
import os

import numpy as np

from .herm_matrix import herm_matrix

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libnessi_io.so")
_lib = None

EXPORTS = {
    "nessi_io_last_error": (ctypes.c_char_p, []),
    "nessi_hm_print_to_file": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4 +
                               [ctypes.c_int]),
    "nessi_hm_file_header": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.POINTER(ctypes.c_int)] * 4),
    "nessi_hm_read_from_file": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 3 +
                                [ctypes.POINTER(ctypes.c_int)] + [ctypes.c_void_p] * 4),
    "nessi_hm_read_from_file_nt1": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4),
}


class HmFileError(RuntimeError):
    pass


def load_library(path=None):
    global _lib
    if _lib is None:
        p = path or _LIB_PATH
        if not os.path.exists(p):
            raise HmFileError("%s is missing: run `python -m nessi_b200.build`" % p)
        L = ctypes.CDLL(p)
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise HmFileError(load_library().nessi_io_last_error().decode())


def _p(a):
    if a is None or a.size == 0:
        return None
    if a.dtype != np.complex128 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous complex128")
    return a.ctypes.data


def _name(file):
    return os.fsencode(file)


def print_to_file(G, file, precision=16):
    """G.print_to_file(file, precision)."""
    _check(load_library().nessi_hm_print_to_file(_name(file), G.nt, G.ntau, G.size1, G.sig, _p(G.ret), _p(G.les),
                                                 _p(G.tv), _p(G.mat), precision))


def file_header(file):
    """(nt, ntau, size1, sig) of a file written by print_to_file."""
    v = [ctypes.c_int() for _ in range(4)]
    _check(load_library().nessi_hm_file_header(_name(file), *[ctypes.byref(x) for x in v]))
    return tuple(x.value for x in v)


def read_from_file(file, G=None):
    """G.read_from_file(file): with G None, a herm_matrix of the file's size is returned; a given G
    must hold the file (nt >= the file's, equal ntau and size1) and receives its sign."""
    if G is None:
        nt, ntau, s, sig = file_header(file)
        G = herm_matrix(nt, ntau, s, sig)
    sig = ctypes.c_int()
    _check(load_library().nessi_hm_read_from_file(_name(file), G.nt, G.ntau, G.size1, ctypes.byref(sig), _p(G.ret),
                                                  _p(G.les), _p(G.tv), _p(G.mat)))
    G.sig = sig.value
    return G


def read_from_file_nt1(G, nt1, file):
    """G.read_from_file(nt1, file): mat and time steps 0..nt1; the rest of G is left as it is."""
    _check(load_library().nessi_hm_read_from_file_nt1(_name(file), nt1, G.nt, G.ntau, G.size1, _p(G.ret), _p(G.les),
                                                      _p(G.tv), _p(G.mat)))
    return G


def _problem_shape(batch, p):
    d = batch.descs[p]
    return d["nt"], d["ntau"], d.get("size1", 1), d.get("sig", -1)


def checkpoint(batch, p, file, precision=17):
    """Download problem p of a device batch and print it (all time steps the batch holds)."""
    G = herm_matrix(*_problem_shape(batch, p))
    batch.get_G(p, G)
    print_to_file(G, file, precision)
    return G


def restart(batch, p, nt1, file):
    """Read mat and time steps 0..nt1 of a checkpoint into problem p of a device batch; the
    propagation continues with time step nt1 + 1."""
    G = herm_matrix(*_problem_shape(batch, p))
    read_from_file_nt1(G, nt1, file)
    batch.set_G(p, G)
    return G


__all__ = ["print_to_file", "file_header", "read_from_file", "read_from_file_nt1", "checkpoint", "restart",
           "HmFileError"]
