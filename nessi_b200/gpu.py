"""Python host API over libnessi_gpu.so (C ABI in include/nessi_gpu.h).

``Batch`` advances many problems ("k-points") sharing a self-energy on one GPU.  The
cntr-style functions at the bottom (``dyson_timestep`` ...) mirror libcntr's signatures
(libcntr/cntr/cntr_dyson_decl.hpp:92) for single problems.

There is no CPU fallback: if the CUDA library is missing or no device is present every
call raises ``NessiGpuError``.
"""
import ctypes
import os

import numpy as np

from .herm_matrix import herm_matrix, function

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libnessi_gpu.so")
_lib = None
_inited = False

PREC_FP64 = 0
PREC_MIXED = 1

_ERRNAMES = {1: "NESSI_ERR_ARG", 2: "NESSI_ERR_OOM", 3: "NESSI_ERR_CUDA", 4: "NESSI_ERR_SINGULAR",
             5: "NESSI_ERR_TIMEOUT"}


class NessiGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (_ERRNAMES.get(code, str(code)), msg))
        self.code = code


class ProblemDesc(ctypes.Structure):
    _fields_ = [("nt", ctypes.c_int), ("ntau", ctypes.c_int), ("size1", ctypes.c_int), ("sig", ctypes.c_int),
                ("solve_order", ctypes.c_int), ("sigma_group", ctypes.c_int),
                ("beta", ctypes.c_double), ("h", ctypes.c_double), ("mu", ctypes.c_double)]


class HmPtrs(ctypes.Structure):
    """Device pointers of one herm_matrix (nessi_hm_ptrs)."""
    _fields_ = [("ret", ctypes.c_void_p), ("les", ctypes.c_void_p), ("tv", ctypes.c_void_p), ("mat", ctypes.c_void_p)]


EXPORTS = {
    "nessi_gpu_init": (ctypes.c_int, [ctypes.c_int]),
    "nessi_gpu_last_error": (ctypes.c_char_p, []),
    "nessi_gpu_finalize": (ctypes.c_int, []),
    "nessi_gpu_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ProblemDesc),
                                              ctypes.c_int, ctypes.c_int]),
    "nessi_gpu_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_batch_bytes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "nessi_gpu_set_G": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4),
    "nessi_gpu_get_G": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4),
    "nessi_gpu_get_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_set_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_set_H": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_set_sigma": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4),
    "nessi_gpu_set_sigma_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_dyson_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nessi_gpu_dyson_mat": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_dyson_start": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_dyson_mat_method": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "nessi_gpu_vie2_mat_method": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nessi_gpu_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_set_wait_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "nessi_gpu_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "nessi_gpu_dyson_mat_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                   ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p]),
    "nessi_gpu_set_F": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 6),
    "nessi_gpu_set_Fcc_mat": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_set_F_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_void_p]),
    "nessi_gpu_set_Q": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4),
    "nessi_gpu_set_Q_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_vie2_start": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_vie2_mat": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_vie2_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nessi_gpu_set_U": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "nessi_gpu_extrapolate_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nessi_gpu_gloc_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "nessi_gpu_sigma_2b_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "nessi_gpu_get_gloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4),
    "nessi_gpu_get_sigma": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 4),
    "nessi_gpu_gloc_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int] + [ctypes.POINTER(ctypes.c_void_p)] * 4),
    "nessi_gpu_lattice_2b_start": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                  ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]),
    "nessi_gpu_lattice_2b_timestep": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "nessi_gpu_convolution_timestep": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 5 +
                                       [ctypes.c_int] * 6 + [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    "nessi_gpu_convolution_timestep_host": (ctypes.c_int, [ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 5 +
                                            [ctypes.c_int] * 6 + [ctypes.c_double, ctypes.c_double]),
    "nessi_gpu_convolution_host": (ctypes.c_int, [ctypes.POINTER(HmPtrs)] * 5 + [ctypes.c_int] * 6 +
                                   [ctypes.c_double, ctypes.c_double]),
    "nessi_gpu_incr_convolution_timestep": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double] +
                                            [ctypes.POINTER(HmPtrs)] * 3 + [ctypes.c_void_p] +
                                            [ctypes.POINTER(HmPtrs)] * 2 + [ctypes.c_int] * 6 +
                                            [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    "nessi_gpu_incr_convolution_component": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                                            ctypes.c_double, ctypes.c_double] +
                                             [ctypes.POINTER(HmPtrs)] * 3 + [ctypes.c_void_p] +
                                             [ctypes.POINTER(HmPtrs)] * 2 + [ctypes.c_int] * 6 +
                                             [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    "nessi_gpu_convolution_timestep_new": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 3 +
                                           [ctypes.c_void_p] + [ctypes.POINTER(HmPtrs)] * 2 + [ctypes.c_int] * 6 +
                                           [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    "nessi_gpu_dyson_timestep_omp": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 2 +
                                     [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 5 +
                                     [ctypes.c_double, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]),
    "nessi_gpu_vie2_timestep_omp": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 4 +
                                    [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                                          ctypes.c_void_p]),
    "nessi_gpu_incr_convolution_timestep_host": (ctypes.c_int, [ctypes.c_int, ctypes.c_double, ctypes.c_double] +
                                                 [ctypes.POINTER(HmPtrs)] * 3 + [ctypes.c_void_p] +
                                                 [ctypes.POINTER(HmPtrs)] * 2 + [ctypes.c_int] * 6 +
                                                 [ctypes.c_double, ctypes.c_double]),
    "nessi_gpu_dyson_timestep_omp_host": (ctypes.c_int, [ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 2 +
                                          [ctypes.c_void_p, ctypes.c_double] + [ctypes.c_int] * 5 +
                                          [ctypes.c_double, ctypes.c_double]),
    "nessi_gpu_vie2_timestep_omp_host": (ctypes.c_int, [ctypes.c_int] + [ctypes.POINTER(HmPtrs)] * 4 +
                                         [ctypes.c_int] * 5 + [ctypes.c_double, ctypes.c_double]),
    "nessi_gpu_distance_norm2": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(HmPtrs), ctypes.POINTER(HmPtrs)] +
                                 [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_void_p]),
    "nessi_gpu_gw_polarization_timestep": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p] + [ctypes.c_int] * 4 + [ctypes.c_void_p]),
    "nessi_gpu_gw_sigma_timestep": (ctypes.c_int, [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4 +
                                    [ctypes.c_int] * 3 + [ctypes.c_void_p]),
    "nessi_gpu_get_volterra_choice": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                                     ctypes.POINTER(ctypes.c_int)]),
    "nessi_gpu_graph_record": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_int] * 4),
    "nessi_gpu_graph_launch": (ctypes.c_int, [ctypes.c_void_p]),
    "nessi_gpu_set_profiling": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "nessi_gpu_read_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                              ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_double)]),
}

KERNELS = ["prep", "ret", "tv", "les_operands", "gemm", "les", "matop", "lattice"]


def load_library(path=None):
    """Load libnessi_gpu.so and declare its exports (no device needed)."""
    global _lib
    if _lib is None:
        p = path or _LIB_PATH
        if not os.path.exists(p):
            raise NessiGpuError(3, "%s is missing: run `python -m nessi_b200.build`" % p)
        L = ctypes.CDLL(p)
        for name, (res, args) in EXPORTS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise NessiGpuError(rc, load_library().nessi_gpu_last_error().decode())


def init(device=0):
    global _inited
    L = load_library()
    _check(L.nessi_gpu_init(device))
    _inited = True


def finalize():
    """nessi_gpu_finalize: every batch must be closed first."""
    global _inited
    _check(load_library().nessi_gpu_finalize())
    _inited = False


def _ptr(a):
    if a is None or a.size == 0:
        return None
    if a.dtype != np.complex128 or not a.flags["C_CONTIGUOUS"]:
        raise ValueError("arrays must be C-contiguous complex128")
    return a.ctypes.data


class Batch:
    """Problems advanced together on one GPU; problems with equal ``sigma_group`` share Sigma."""

    def __init__(self, descs, precision=PREC_FP64):
        if not _inited:
            init(0)
        arr = (ProblemDesc * len(descs))()
        for i, d in enumerate(descs):
            arr[i] = ProblemDesc(d["nt"], d["ntau"], d.get("size1", 1), d.get("sig", -1), d.get("solve_order", 5),
                                 d.get("sigma_group", 0), d["beta"], d["h"], d.get("mu", 0.0))
        self.descs = [dict(d) for d in descs]
        h = ctypes.c_void_p()
        _check(load_library().nessi_gpu_batch_create(ctypes.byref(h), arr, len(descs), precision))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            load_library().nessi_gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def nbytes(self):
        v = ctypes.c_longlong()
        _check(load_library().nessi_gpu_batch_bytes(self._h, ctypes.byref(v)))
        return v.value

    def set_G(self, p, G):
        _check(load_library().nessi_gpu_set_G(self._h, p, _ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat)))

    def get_G(self, p, G):
        _check(load_library().nessi_gpu_get_G(self._h, p, _ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat)))

    def get_timestep(self, p, tstp, out):
        _check(load_library().nessi_gpu_get_timestep(self._h, p, tstp, _ptr(out)))

    def set_timestep(self, p, tstp, data):
        _check(load_library().nessi_gpu_set_timestep(self._h, p, tstp, _ptr(np.ascontiguousarray(data))))

    def set_H(self, p, H):
        a = H.data if isinstance(H, function) else H
        _check(load_library().nessi_gpu_set_H(self._h, p, _ptr(np.ascontiguousarray(a, np.complex128))))

    def set_sigma(self, group, S):
        _check(load_library().nessi_gpu_set_sigma(self._h, group, _ptr(S.ret), _ptr(S.les), _ptr(S.tv), _ptr(S.mat)))

    def set_sigma_timestep(self, group, tstp, data):
        _check(load_library().nessi_gpu_set_sigma_timestep(self._h, group, tstp,
                                                           _ptr(np.ascontiguousarray(data, np.complex128))))

    def dyson_timestep(self, n):
        _check(load_library().nessi_gpu_dyson_timestep(self._h, n))

    def dyson_mat(self, method=2, force_hermitian=True):
        """G^mat of every problem (cntr::dyson_mat; method 0 = Fourier, 1 = steepest descent,
        2 = fixpoint, the default)."""
        _check(load_library().nessi_gpu_dyson_mat_method(self._h, int(method), int(bool(force_hermitian))))

    def dyson_start(self):
        """Time steps 0..k of every problem (cntr::dyson_start)."""
        _check(load_library().nessi_gpu_dyson_start(self._h))

    def synchronize(self):
        _check(load_library().nessi_gpu_synchronize(self._h))

    def set_wait_limit(self, ns):
        """Bound (device nanoseconds) of every mbarrier wait in this batch's kernels."""
        _check(load_library().nessi_gpu_set_wait_limit(self._h, int(ns)))

    # ---- VIE2: [1 + F] G = Q ---------------------------------------------------------
    def set_F(self, group, F, Fcc):
        """Kernel F of a group (and its partner Fcc); makes the group a VIE2 group."""
        _check(load_library().nessi_gpu_set_F(self._h, group, _ptr(F.ret), _ptr(F.les), _ptr(F.tv), _ptr(F.mat),
                                              _ptr(Fcc.ret), _ptr(Fcc.les)))
        if Fcc.mat is not None and Fcc.mat.size:  # Fcc^mat: the steepest-descent vie2_mat reads it
            _check(load_library().nessi_gpu_set_Fcc_mat(self._h, group, _ptr(Fcc.mat)))

    def set_F_timestep(self, group, tstp, F_slice, Fcc_slice=None):
        fs = np.ascontiguousarray(F_slice, np.complex128)
        cs = None if Fcc_slice is None else np.ascontiguousarray(Fcc_slice, np.complex128)
        _check(load_library().nessi_gpu_set_F_timestep(self._h, group, tstp, _ptr(fs), _ptr(cs)))

    def set_Q(self, p, Q):
        _check(load_library().nessi_gpu_set_Q(self._h, p, _ptr(Q.ret), _ptr(Q.les), _ptr(Q.tv), _ptr(Q.mat)))

    def set_Q_timestep(self, p, tstp, data):
        _check(load_library().nessi_gpu_set_Q_timestep(self._h, p, tstp, _ptr(np.ascontiguousarray(data,
                                                                                                    np.complex128))))

    def vie2_mat(self, method=2):
        """G^mat of every VIE2 problem (cntr::vie2_mat; method 0 = Fourier, 2 = fixpoint, the default)."""
        _check(load_library().nessi_gpu_vie2_mat_method(self._h, int(method)))

    def vie2_start(self):
        """Time steps 0..k of every VIE2 problem (cntr::vie2_start)."""
        _check(load_library().nessi_gpu_vie2_start(self._h))

    def vie2_timestep(self, n):
        """cntr::vie2_timestep(n, ...) for every VIE2 problem."""
        _check(load_library().nessi_gpu_vie2_timestep(self._h, n))

    # ---- CUDA graphs ------------------------------------------------------------------
    GRAPH_DYSON, GRAPH_VIE2, GRAPH_LATTICE = 0, 1, 2

    def graph_record(self, kind, n0, n1, corrector_steps=3):
        """Record the launches of steps n0..n1 into a CUDA graph (nothing runs)."""
        _check(load_library().nessi_gpu_graph_record(self._h, kind, n0, n1, corrector_steps))

    def volterra_choice(self, group=0):
        """(ret, les) Volterra kernels of a group: -1 one problem per CTA, 2/4/8 problems per CTA."""
        r, l = ctypes.c_int(), ctypes.c_int()
        _check(load_library().nessi_gpu_get_volterra_choice(self._h, group, ctypes.byref(r), ctypes.byref(l)))
        return r.value, l.value

    def graph_launch(self):
        _check(load_library().nessi_gpu_graph_launch(self._h))

    # ---- self-consistent lattice ----------------------------------------------------
    def set_U(self, group, U):
        """Diagonal local interaction of a group: array (nt+2, size1), t = -1 first."""
        _check(load_library().nessi_gpu_set_U(self._h, group, _ptr(np.ascontiguousarray(U, np.complex128))))

    def extrapolate_timestep(self, n):
        """cntr::extrapolate_timestep(n, G, SolveOrder) of every problem: step n+1 from n-k..n."""
        _check(load_library().nessi_gpu_extrapolate_timestep(self._h, n))

    def gloc_timestep(self, group, tstp):
        _check(load_library().nessi_gpu_gloc_timestep(self._h, group, tstp))

    def sigma_2b_timestep(self, group, tstp):
        _check(load_library().nessi_gpu_sigma_2b_timestep(self._h, group, tstp))

    def get_gloc(self, group, G):
        _check(load_library().nessi_gpu_get_gloc(self._h, group, _ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat)))

    def get_sigma(self, group, S):
        _check(load_library().nessi_gpu_get_sigma(self._h, group, _ptr(S.ret), _ptr(S.les), _ptr(S.tv), _ptr(S.mat)))

    def group_shape(self, group):
        """(ntmax, ntau, size1, solve_order, number of problems) of a sigma group."""
        m = [d for d in self.descs if d.get("sigma_group", 0) == group]
        if not m:
            raise NessiGpuError(1, "no problem in sigma group %d" % group)
        return max(d["nt"] for d in m), m[0]["ntau"], m[0].get("size1", 1), m[0].get("solve_order", 5), len(m)

    def gloc_views(self, group):
        """{component: torch float64 tensor} aliasing the group's G_loc in device memory (no copy;
        libcntr layout, real and imaginary parts interleaved), valid while the batch lives."""
        ntmax, ntau, s, _, _ = self.group_shape(group)
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        _check(load_library().nessi_gpu_gloc_device(self._h, group, *[ctypes.byref(q) for q in ptrs]))
        s2, N, M = s * s, ntmax + 1, ntau + 1
        sizes = {"ret": N * (N + 1) // 2 * s2, "les": N * (N + 1) // 2 * s2, "tv": N * M * s2, "mat": M * s2}
        return {c: _device_f64(q.value, 2 * sizes[c]) for c, q in zip(("ret", "les", "tv", "mat"), ptrs)}

    def lattice_2b_start(self, max_iter=20, tol=1e-12):
        """Bootstrap of the lattice; returns (iterations, last distance)."""
        it, err = ctypes.c_int(), ctypes.c_double()
        _check(load_library().nessi_gpu_lattice_2b_start(self._h, max_iter, tol, ctypes.byref(it), ctypes.byref(err)))
        return it.value, err.value

    def lattice_2b_timestep(self, n, corrector_steps=3):
        _check(load_library().nessi_gpu_lattice_2b_timestep(self._h, n, corrector_steps))

    def set_stream(self, stream_handle):
        """Use a caller-owned cudaStream_t (an int handle, e.g. torch.cuda.Stream().cuda_stream)."""
        _check(load_library().nessi_gpu_set_stream(self._h, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def set_profiling(self, on=True):
        _check(load_library().nessi_gpu_set_profiling(self._h, int(on)))

    def read_profile(self):
        """{kernel: (device ms, launches, algorithmic bytes or flops)} since the last read."""
        out = {}
        for i, name in enumerate(KERNELS):
            ms, nl, by = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_double()
            _check(load_library().nessi_gpu_read_profile(self._h, i, ctypes.byref(ms), ctypes.byref(nl),
                                                         ctypes.byref(by)))
            out[name] = (ms.value, nl.value, by.value)
        return out


class _DeviceBuffer:
    """Device memory of the library described by the CUDA array interface (read by torch)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 2}


def _device_f64(ptr, n):
    import torch
    if not ptr:
        raise NessiGpuError(3, "null device pointer")
    return torch.as_tensor(_DeviceBuffer(ptr, n), device="cuda")


def dyson_mat_noalloc(ntau, size1, sig, solve_order, beta, mu, H_ptr, sigma_mat_ptr, gmat_ptr, stream=0):
    """nessi_gpu_dyson_mat_noalloc on caller-owned device pointers (integers); allocates
    nothing.  For callers that cannot let the library allocate device memory."""
    _check(load_library().nessi_gpu_dyson_mat_noalloc(ntau, size1, sig, solve_order, beta, mu, ctypes.c_void_p(H_ptr),
                                                       ctypes.c_void_p(sigma_mat_ptr), ctypes.c_void_p(gmat_ptr),
                                                       ctypes.c_void_p(stream) if stream else None))


def distance_norm2_dev(tstp, g1, g2, nt, ntau, size1, out_ptr, stream=0):
    """nessi_gpu_distance_norm2 on device herm_matrix data: g1, g2 are HmPtrs (device pointers,
    libcntr layout); the result is written to the device double at out_ptr."""
    _check(load_library().nessi_gpu_distance_norm2(tstp, ctypes.byref(g1), ctypes.byref(g2), nt, ntau, size1,
                                                    ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream) if stream else None))


def gw_polarization_timestep_dev(tstp, nk, G_table, P_table, w_ptr, nt, ntau, size1, sig_g=-1, stream=0):
    """nessi_gpu_gw_polarization_timestep: the tables are device addresses of nk HmPtrs (and of nk
    float64 weights)."""
    _check(load_library().nessi_gpu_gw_polarization_timestep(tstp, nk, ctypes.c_void_p(G_table), ctypes.c_void_p(P_table),
                                                              ctypes.c_void_p(w_ptr), nt, ntau, size1, sig_g,
                                                              ctypes.c_void_p(stream) if stream else None))


def gw_sigma_timestep_dev(tstp, nk, G_table, W_table, S_table, w_ptr, nt, ntau, size1, stream=0):
    """nessi_gpu_gw_sigma_timestep on device tables (see gw_polarization_timestep_dev)."""
    _check(load_library().nessi_gpu_gw_sigma_timestep(tstp, nk, ctypes.c_void_p(G_table), ctypes.c_void_p(W_table),
                                                       ctypes.c_void_p(S_table), ctypes.c_void_p(w_ptr), nt, ntau,
                                                       size1, ctypes.c_void_p(stream) if stream else None))


def convolution_timestep_dev(n, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h, stream=0):
    """cntr::convolution_timestep(n, C, A, Acc, B, Bcc, beta, h, SolveOrder) for len(C) problems on
    device memory.  Each of C, A, Acc, B, Bcc is a list of (ret, les, tv, mat) device pointers
    (integers, libcntr layout).  Queued on ``stream``; allocates nothing."""
    if not _inited:
        init(0)
    cnt = len(C)

    def arr(lst):
        a = (HmPtrs * max(cnt, 1))()
        for i, t in enumerate(lst):
            a[i] = HmPtrs(*[ctypes.c_void_p(x) if x else None for x in t])
        return a
    _check(load_library().nessi_gpu_convolution_timestep(n, cnt, arr(C), arr(A), arr(Acc), arr(B), arr(Bcc), nt, ntau,
                                                         size1, sig_a, sig_b, solve_order, beta, h,
                                                         ctypes.c_void_p(stream) if stream else None))


def _hm_array(lst):
    a = (HmPtrs * max(len(lst), 1))()
    for i, t in enumerate(lst):
        a[i] = HmPtrs(*[ctypes.c_void_p(x) if x else None for x in t])
    return a


def _ptr_array(lst):
    """host array of device pointers (integers, 0 = none), or None for no list"""
    if lst is None:
        return None
    a = (ctypes.c_void_p * max(len(lst), 1))()
    for i, x in enumerate(lst):
        a[i] = ctypes.c_void_p(x) if x else None
    return a


def _stream(stream):
    return ctypes.c_void_p(stream) if stream else None


def incr_convolution_dev(tstp, alpha, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h, ft=None,
                         stream=0):
    """incr_convolution (cntr_convolution_impl.hpp:4786-4807): C(tstp) += alpha A * ft * B for len(C)
    problems on device memory; C, A, Acc, B, Bcc are lists of (ret, les, tv, mat) device pointers,
    ft None or a list of device pointers to function data (F(-1) first).  Allocates nothing."""
    if not _inited:
        init(0)
    alpha = complex(alpha)
    _check(load_library().nessi_gpu_incr_convolution_timestep(
        tstp, len(C), alpha.real, alpha.imag, _hm_array(C), _hm_array(A), _hm_array(Acc), _ptr_array(ft), _hm_array(B),
        _hm_array(Bcc), nt, ntau, size1, sig_a, sig_b, solve_order, beta, h, _stream(stream)))


def incr_convolution_component_dev(which, tstp, mask_ptr, alpha, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b,
                                   solve_order, beta, h, ft=None, stream=0):
    """One component of incr_convolution (0 mat, 1 ret, 2 tv, 3 les) for the output indices whose
    byte in the device array at mask_ptr is nonzero (0 = all)."""
    if not _inited:
        init(0)
    alpha = complex(alpha)
    _check(load_library().nessi_gpu_incr_convolution_component(
        which, tstp, ctypes.c_void_p(mask_ptr) if mask_ptr else None, len(C), alpha.real, alpha.imag, _hm_array(C),
        _hm_array(A), _hm_array(Acc), _ptr_array(ft), _hm_array(B), _hm_array(Bcc), nt, ntau, size1, sig_a, sig_b,
        solve_order, beta, h, _stream(stream)))


def convolution_timestep_new_dev(tstp, C, A, Acc, B, Bcc, nt, ntau, size1, sig_a, sig_b, solve_order, beta, h, ft=None,
                                 stream=0):
    """convolution_timestep_new / convolution_timestep_omp (cntr_convolution_impl.hpp:4811-4976,
    5596-5812): C's time step zeroed, then incr_convolution with alpha = 1."""
    if not _inited:
        init(0)
    _check(load_library().nessi_gpu_convolution_timestep_new(
        tstp, len(C), _hm_array(C), _hm_array(A), _hm_array(Acc), _ptr_array(ft), _hm_array(B), _hm_array(Bcc), nt,
        ntau, size1, sig_a, sig_b, solve_order, beta, h, _stream(stream)))


def dyson_timestep_omp_dev(n, G, Sigma, H, mu, nt, ntau, size1, sig, solve_order, beta, h, status_ptr=0, stream=0):
    """cntr::dyson_timestep_omp (cntr_dyson_omp_impl.hpp:37-605) for len(G) problems on device
    memory: G, Sigma lists of (ret, les, tv, mat) device pointers, H device pointers to function
    data (H(-1) first), mu a list of floats; status_ptr an optional device int set on a singular
    step matrix."""
    if not _inited:
        init(0)
    mus = (ctypes.c_double * max(len(G), 1))(*[float(x) for x in mu])
    _check(load_library().nessi_gpu_dyson_timestep_omp(
        n, len(G), _hm_array(G), _hm_array(Sigma), _ptr_array(H), mus, nt, ntau, size1, sig, solve_order, beta, h,
        ctypes.c_void_p(status_ptr) if status_ptr else None, _stream(stream)))


def vie2_timestep_omp_dev(n, G, F, Fcc, Q, nt, ntau, size1, sig, solve_order, beta, h, status_ptr=0, stream=0):
    """cntr::vie2_timestep_omp (cntr_vie2_impl.hpp:1851-2190) for n > solve_order on device memory."""
    if not _inited:
        init(0)
    _check(load_library().nessi_gpu_vie2_timestep_omp(
        n, len(G), _hm_array(G), _hm_array(F), _hm_array(Fcc), _hm_array(Q), nt, ntau, size1, sig, solve_order, beta,
        h, ctypes.c_void_p(status_ptr) if status_ptr else None, _stream(stream)))


# ---- cntr-style single-problem entry points ---------------------------------------------
def convolution_timestep(n, C, A, Acc, B, Bcc, beta, h, SolveOrder=5):
    """cntr::convolution_timestep(n, C, A, Acc, B, Bcc, beta, h, SolveOrder) on host herm_matrix
    objects (cntr_convolution_decl.hpp:61): writes C's time step n (mat for n = -1) in place."""
    if not _inited:
        init(0)

    def hp(G):
        return ctypes.byref(HmPtrs(_ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat)))
    _check(load_library().nessi_gpu_convolution_timestep_host(n, hp(C), hp(A), hp(Acc), hp(B), hp(Bcc), C.nt, C.ntau,
                                                              C.size1, A.sig, B.sig, SolveOrder, beta, h))


def _hp(G):
    return ctypes.byref(HmPtrs(_ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat)))


def _fn_data(F):
    """cntr::function-like object (or its (nt+2, s, s) array) as a contiguous complex128 array"""
    a = F.data if hasattr(F, "data") and not isinstance(F, np.ndarray) else F
    return np.ascontiguousarray(a, dtype=np.complex128)


def incr_convolution(tstp, alpha, C, A, Acc, B, Bcc, beta, h, SolveOrder=5, ft=None):
    """incr_convolution (cntr_convolution_impl.hpp:4786-4807) on host herm_matrix objects:
    C(tstp) += alpha A * ft * B, written in place (ft: cntr::function or None)."""
    if not _inited:
        init(0)
    alpha = complex(alpha)
    fd = None if ft is None else _fn_data(ft)
    _check(load_library().nessi_gpu_incr_convolution_timestep_host(
        tstp, alpha.real, alpha.imag, _hp(C), _hp(A), _hp(Acc), None if fd is None else fd.ctypes.data, _hp(B),
        _hp(Bcc), C.nt, C.ntau, C.size1, A.sig, B.sig, SolveOrder, beta, h))


def convolution_timestep_omp(omp_num_threads, tstp, C, A, Acc, B, Bcc, beta, h, SolveOrder=5):
    """cntr::convolution_timestep_omp / convolution_timestep_new (cntr_convolution_impl.hpp:4916-4976,
    5596-5812) on host herm_matrix objects: C's time step zeroed, then incr_convolution with alpha = 1;
    omp_num_threads is ignored (every element is a GPU thread)."""
    if tstp == -1:
        C.mat[...] = 0
    else:
        C.ret[C.ret_index(tstp, 0):C.ret_index(tstp, tstp) + 1] = 0
        C.tv[tstp] = 0
        C.les[C.les_index(0, tstp):C.les_index(tstp, tstp) + 1] = 0
    incr_convolution(tstp, 1.0, C, A, Acc, B, Bcc, beta, h, SolveOrder)


def dyson_timestep_omp(omp_num_threads, n, G, mu, H, Sigma, beta, h, SolveOrder=5):
    """cntr::dyson_timestep_omp (cntr_dyson_omp_impl.hpp:577-605) on host herm_matrix objects: time
    step n (> SolveOrder) of G in place, in the OpenMP solver's discretization."""
    if not _inited:
        init(0)
    hd = _fn_data(H)
    _check(load_library().nessi_gpu_dyson_timestep_omp_host(n, _hp(G), _hp(Sigma), hd.ctypes.data, mu, G.nt, G.ntau,
                                                            G.size1, G.sig, SolveOrder, beta, h))


def vie2_timestep_omp(omp_num_threads, n, G, F, Fcc, Q, beta, h, SolveOrder=5, matsubara_method=2):
    """cntr::vie2_timestep_omp (cntr_vie2_impl.hpp:2125-2190) on host herm_matrix objects: n = -1
    vie2_mat, n <= SolveOrder vie2_start of order n (as the reference dispatches), else the
    element-parallel step on the GPU."""
    if n <= SolveOrder:
        if n == 0:
            raise NessiGpuError(1, "vie2_timestep_omp: an order-0 start (n = 0) is not available")
        b = Batch([dict(nt=G.nt, ntau=G.ntau, size1=G.size1, sig=G.sig, solve_order=SolveOrder if n < 0 else n,
                        beta=beta, h=h)])
        try:
            b.set_F(0, F, Fcc)
            b.set_Q(0, Q)
            b.set_G(0, G)
            if n < 0:
                b.vie2_mat(matsubara_method)
            else:
                b.vie2_start()
            b.get_G(0, G)
        finally:
            b.close()
        return
    if not _inited:
        init(0)
    _check(load_library().nessi_gpu_vie2_timestep_omp_host(n, _hp(G), _hp(F), _hp(Fcc), _hp(Q), G.nt, G.ntau, G.size1,
                                                           G.sig, SolveOrder, beta, h))


def convolution(C, A, Acc, B, Bcc, beta, h, SolveOrder=5):
    """cntr::convolution(C, A, Acc, B, Bcc, beta, h, SolveOrder) (cntr_convolution_decl.hpp:66-68):
    C = A * B at every time step, -1..nt; the operands are copied to the device once.  For
    hermitian operands pass A as Acc and B as Bcc (the reference's short form)."""
    if not _inited:
        init(0)

    def hp(G):
        return ctypes.byref(HmPtrs(_ptr(G.ret), _ptr(G.les), _ptr(G.tv), _ptr(G.mat)))
    _check(load_library().nessi_gpu_convolution_host(hp(C), hp(A), hp(Acc), hp(B), hp(Bcc), C.nt, C.ntau, C.size1,
                                                     A.sig, B.sig, SolveOrder, beta, h))


def dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder=5):
    """cntr::dyson_timestep(n, G, mu, H, Sigma, beta, h, SolveOrder) on the GPU
    (cntr_dyson_decl.hpp:92): writes G's time step n in place."""
    b = Batch([dict(nt=G.nt, ntau=G.ntau, size1=G.size1, sig=G.sig, solve_order=SolveOrder, beta=beta, h=h,
                    mu=mu)])
    b.set_G(0, G)
    b.set_H(0, H)
    b.set_sigma(0, Sigma)
    b.dyson_timestep(n)
    slc = np.zeros((2 * (n + 1) + G.ntau + 1, G.size1, G.size1), np.complex128)
    b.get_timestep(0, n, slc)
    G.set_timestep_data(n, slc)
    b.close()


def dyson(G, mu, H, Sigma, beta, h, SolveOrder=5, matsubara_method=2, force_hermitian=True):
    """cntr::dyson(G, mu, H, Sigma, beta, h, SolveOrder, matsubara_method, force_hermitian)
    (cntr_dyson_decl.hpp:95-98, cntr_dyson_impl.hpp:1725-1734): dyson_mat (method 0 Fourier or
    2 fixpoint), dyson_start and every time step on the GPU from one upload; all of G is written."""
    b = Batch([dict(nt=G.nt, ntau=G.ntau, size1=G.size1, sig=G.sig, solve_order=SolveOrder, beta=beta, h=h,
                    mu=mu)])
    try:
        b.set_G(0, G)
        b.set_H(0, H)
        b.set_sigma(0, Sigma)
        b.dyson_mat(matsubara_method, force_hermitian)
        b.dyson_start()
        for n in range(SolveOrder + 1, G.nt + 1):
            b.dyson_timestep(n)
        b.get_G(0, G)
    finally:
        b.close()


def vie2(G, F, Fcc, Q, beta, h, SolveOrder=5, matsubara_method=2):
    """cntr::vie2(G, F, Fcc, Q, beta, h, SolveOrder, matsubara_method) (cntr_vie2_decl.hpp:85-86):
    [1 + F] G = Q by vie2_mat (method 0 Fourier or 2 fixpoint), vie2_start and every time step on
    the GPU from one upload."""
    b = Batch([dict(nt=G.nt, ntau=G.ntau, size1=G.size1, sig=G.sig, solve_order=SolveOrder, beta=beta, h=h)])
    try:
        b.set_F(0, F, Fcc)
        b.set_Q(0, Q)
        b.vie2_mat(matsubara_method)
        b.vie2_start()
        for n in range(SolveOrder + 1, G.nt + 1):
            b.vie2_timestep(n)
        b.get_G(0, G)
    finally:
        b.close()


def _value_at_minus1(X, s):
    """The (s, s) value of a cntr::function at t = -1, or a plain matrix."""
    a = X.get_value(-1) if isinstance(X, function) else np.asarray(X, np.complex128)
    return np.ascontiguousarray(a, np.complex128).reshape(s, s)


def dyson_mat(G, mu, H, Sigma, beta, SolveOrder=5, SigmaMF=None, method=2, force_hermitian=True):
    """cntr::dyson_mat(G, mu, H, Sigma, beta, SolveOrder, method, force_hermitian)
    (cntr_dyson_decl.hpp:77-79): writes G^mat; method 0 = Fourier (dyson_mat_fourier_dispatch,
    cntr_dyson_impl.hpp:356-446), 1 = steepest descent (dyson_mat_steep_dispatch, :519-540), 2 =
    fixpoint (the default).  With ``SigmaMF`` (a cntr::function or the (s, s) matrix of its value
    at -1) it is the mean-field overload dyson_mat(G, mu, H, SigmaMF, Sigma, beta, SolveOrder,
    method) (:81-83; cntr_dyson_impl.hpp:472-575, 1270-1298): the Fourier method takes
    H(-1) + SigmaMF(-1) as the one-body part; with G0 the free propagator of H(-1), the fixpoint
    method solves [1 + F] G = G0 with F = -(G0 * Sigma + G0 SigmaMF(-1)), and steepest descent the
    same with Fcc = -(Sigma * G0 + SigmaMF(-1) G0) (:545-572); the convolutions and the solves run
    on the GPU."""
    from .equilibrium import green_from_H
    k, s, ntau, sig = SolveOrder, G.size1, G.ntau, G.sig
    h0 = _value_at_minus1(H, s)
    if SigmaMF is not None and method == 0:
        h0 = h0 + _value_at_minus1(SigmaMF, s)
        SigmaMF = None
    Sk = herm_matrix(k, ntau, s, sig)  # only the Matsubara branch takes part
    Sk.mat[...] = Sigma.mat
    desc = dict(nt=k, ntau=ntau, size1=s, sig=sig, solve_order=k, beta=beta, h=1.0, mu=mu)
    out = herm_matrix(k, ntau, s, sig)
    if SigmaMF is None:
        b = Batch([desc])
        try:
            b.set_H(0, np.broadcast_to(h0, (k + 2, s, s)).copy())
            b.set_sigma(0, Sk)
            b.dyson_mat(method, force_hermitian)
            b.get_G(0, out)
        finally:
            b.close()
        G.mat[...] = out.mat
        return
    mf = _value_at_minus1(SigmaMF, s)
    G0 = herm_matrix(k, ntau, s, sig)
    green_from_H(G0, mu, h0, beta, 1.0)
    C = herm_matrix(k, ntau, s, sig)
    convolution_timestep(-1, C, G0, G0, Sk, Sk, beta, 1.0, k)  # convolution_matsubara(G0, Sigma)
    F = herm_matrix(k, ntau, s, sig)
    F.mat[...] = -(C.mat + G0.mat @ mf)
    Fcc = F
    if method == 1:
        Cc = herm_matrix(k, ntau, s, sig)
        convolution_timestep(-1, Cc, Sk, Sk, G0, G0, beta, 1.0, k)  # convolution_matsubara(Sigma, G0)
        Fcc = herm_matrix(k, ntau, s, sig)
        Fcc.mat[...] = -(Cc.mat + mf @ G0.mat)
    b = Batch([desc])
    try:
        b.set_F(0, F, Fcc)
        b.set_Q(0, G0)
        b.vie2_mat(1 if method == 1 else 2)
        b.get_G(0, out)
    finally:
        b.close()
    if force_hermitian:
        G.mat[...] = 0.5 * (out.mat + out.mat.conj().transpose(0, 2, 1))  # force_matsubara_hermitian
    else:
        G.mat[...] = out.mat


def vie2_timestep_sin(n, G, Gsin, F, Fcc, Fsin, Q, Qsin, beta, h, SolveOrder=5):
    """cntr::vie2_timestep_sin(n, G, Gsin, F, Fcc, Fsin, Q, Qsin, beta, h, SolveOrder)
    (cntr_vie2_decl.hpp:58, cntr_vie2_impl.hpp:1779-1838): [1 + F] G = Q where F, Q and G carry
    instantaneous parts Fsin, Qsin, Gsin (cntr::function).  The time-local algebra runs on the
    host as in the reference: for t = -1..n2 (n2 = max(n, k) in the start region),
    Finv = (1 + Fsin)^-1, Gsin = Finv Qsin, F -> Finv F, Fcc -> Fcc Finv, Q -> Finv Q - (Finv F) Gsin;
    the Volterra solve runs on the GPU: vie2_mat for n = -1, a start of order n for 1 <= n <= k
    (time steps 0..n), vie2_timestep for n > k.  n = 0 (an order-0 start) is not available."""
    k = SolveOrder
    if n == 0:
        raise NessiGpuError(1, "vie2_timestep_sin: n = 0 needs an order-0 start, which is not available")
    if n < -1 or n > G.nt:
        raise NessiGpuError(1, "vie2_timestep_sin: time step %d out of range" % n)
    s, nt, ntau, sig = G.size1, G.nt, G.ntau, G.sig
    n2 = k if 0 <= n <= k else n
    fs = Fsin.data if isinstance(Fsin, function) else np.asarray(Fsin)
    qs = Qsin.data if isinstance(Qsin, function) else np.asarray(Qsin)
    gs = Gsin.data if isinstance(Gsin, function) else Gsin
    finv = np.zeros((nt + 2, s, s), np.complex128)
    finv[:n2 + 2] = np.linalg.inv(np.eye(s) + fs[:n2 + 2])
    gs[:n2 + 2] = finv[:n2 + 2] @ qs[:n2 + 2]
    tF, tFcc, tQ = F.copy(), Fcc.copy(), Q.copy()
    for t in range(-1, n2 + 1):
        tF.left_multiply(t, finv)
        tFcc.right_multiply(t, finv)
        tQ.left_multiply(t, finv)
    tF1 = tF.copy()
    for t in range(-1, n2 + 1):
        tF1.right_multiply(t, gs)
        tQ.incr_timestep(t, tF1, -1.0)
    order = n if 1 <= n <= k else k
    b = Batch([dict(nt=nt, ntau=ntau, size1=s, sig=sig, solve_order=order, beta=beta, h=h)])
    try:
        b.set_G(0, G)
        b.set_F(0, tF, tFcc)
        b.set_Q(0, tQ)
        if n == -1:
            b.vie2_mat()
            steps = [-1]
        elif n <= k:
            b.vie2_start()
            steps = list(range(0, n + 1))
        else:
            b.vie2_timestep(n)
            steps = [n]
        for t in steps:
            out = np.zeros((_slice_len(t, ntau), s, s), np.complex128)
            b.get_timestep(0, t, out)
            G.set_timestep_data(t, out)
    finally:
        b.close()


def _slice_len(t, ntau):
    """Elements of time step t's slice: ret row, tv row and les column, or mat for t = -1."""
    return ntau + 1 if t < 0 else 2 * (t + 1) + ntau + 1
