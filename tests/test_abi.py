"""The C-ABI library loads without a GPU and exports every symbol include/nessi_gpu.h declares."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "nessi_gpu.h")).read()
    return sorted(set(re.findall(r"\b(nessi_gpu_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "nessi_gpu_dyson_timestep" in syms and len(syms) >= 10


def test_library_exports_all_declared_symbols():
    from nessi_b200 import build, gpu
    build.build()
    L = gpu.load_library()
    for s in declared_symbols():
        assert hasattr(L, s), s
        assert s in gpu.EXPORTS, s


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from nessi_b200 import gpu
    with pytest.raises(gpu.NessiGpuError):
        gpu.init(0)


def test_io_library_exports_all_declared_symbols():
    from nessi_b200 import build, hm_file
    build.build_io()
    text = open(os.path.join(ROOT, "include", "nessi_io.h")).read()
    syms = sorted(set(re.findall(r"\b(nessi_(?:hm|io)_\w+)\s*\(", text)))
    assert len(syms) == 5
    L = hm_file.load_library()
    for s in syms:
        assert hasattr(L, s), s
        assert s in hm_file.EXPORTS, s


def test_finalize_without_batches_needs_no_device():
    from nessi_b200 import gpu
    gpu.finalize()   # nothing was set up: returns at once, on a machine without a GPU too


@pytest.mark.parametrize("bad", [dict(nt=-1), dict(size1=9), dict(size1=0), dict(sig=0), dict(solve_order=6),
                                 dict(solve_order=0), dict(ntau=3), dict(h=0.0), dict(beta=-1.0)])
def test_bad_descriptor_is_rejected_before_the_device(bad):
    """Host-side failure detection: descriptors libcntr would assert on come back as
    NESSI_ERR_ARG with a message, before any device call (so also on a machine without a GPU)."""
    import ctypes
    from nessi_b200 import gpu
    d = dict(nt=10, ntau=8, size1=2, sig=-1, solve_order=5, sigma_group=0, beta=2.0, h=0.05, mu=0.0)
    d.update(bad)
    arr = (gpu.ProblemDesc * 1)(gpu.ProblemDesc(d["nt"], d["ntau"], d["size1"], d["sig"], d["solve_order"],
                                                d["sigma_group"], d["beta"], d["h"], d["mu"]))
    h = ctypes.c_void_p()
    L = gpu.load_library()
    assert L.nessi_gpu_batch_create(ctypes.byref(h), arr, 1, gpu.PREC_FP64) == 1
    assert b"bad descriptor" in L.nessi_gpu_last_error()
    assert not h.value
    assert L.nessi_gpu_batch_create(ctypes.byref(h), arr, 1, 7) == 1          # unknown precision
    assert L.nessi_gpu_batch_create(ctypes.byref(h), arr, 0, gpu.PREC_FP64) == 1  # no problems


def test_null_arguments_are_rejected_before_the_device():
    from nessi_b200 import gpu
    L = gpu.load_library()
    assert L.nessi_gpu_dyson_mat_noalloc(10, 1, -1, 5, 2.0, 0.0, None, None, None, None) == 1
    assert L.nessi_gpu_convolution_timestep_host(2, None, None, None, None, None, 10, 8, 1, -1, -1, 5, 2.0, 0.05) == 1
    assert L.nessi_gpu_convolution_host(None, None, None, None, None, 10, 8, 1, -1, -1, 5, 2.0, 0.05) == 1
    assert L.nessi_gpu_set_G(None, 0, None, None, None, None) == 1   # no batch


def test_element_parallel_entries_reject_bad_arguments_before_the_device():
    """incr_convolution, convolution_timestep_new, dyson_timestep_omp and vie2_timestep_omp return
    NESSI_ERR_ARG for null operands, a step the solver does not cover (n <= SolveOrder, which
    libcntr asserts on: cntr_dyson_omp_impl.hpp:595, cntr_vie2_impl.hpp:2150) and bad
    dimensions, without touching a device."""
    import ctypes
    from nessi_b200 import gpu
    L = gpu.load_library()
    z = gpu.HmPtrs(None, None, None, None)
    one = (gpu.HmPtrs * 1)(z)
    mu = (ctypes.c_double * 1)(0.0)
    H = (ctypes.c_void_p * 1)(None)
    assert L.nessi_gpu_incr_convolution_timestep(3, 1, 1.0, 0.0, one, one, one, None, one, one, 10, 8, 1, -1, -1, 5, 2.0,
                                                 0.05, None) == 1
    assert L.nessi_gpu_incr_convolution_component(2, -1, None, 1, 1.0, 0.0, one, one, one, None, one, one, 10, 8, 1,
                                                  -1, -1, 5, 2.0, 0.05, None) == 1     # tv needs tstp >= 0
    assert L.nessi_gpu_convolution_timestep_new(3, 1, one, one, one, None, one, one, 10, 8, 1, -1, -1, 5, 2.0, 0.05,
                                                None) == 1
    assert L.nessi_gpu_dyson_timestep_omp(5, 1, one, one, H, mu, 10, 8, 1, -1, 5, 2.0, 0.05, None, None) == 1
    assert b"must exceed SolveOrder" in L.nessi_gpu_last_error()
    assert L.nessi_gpu_dyson_timestep_omp(7, 1, one, one, H, mu, 10, 8, 1, -1, 5, 2.0, 0.05, None, None) == 1
    assert L.nessi_gpu_vie2_timestep_omp(4, 1, one, one, one, one, 10, 8, 1, -1, 5, 2.0, 0.05, None, None) == 1
    assert L.nessi_gpu_vie2_timestep_omp(7, 1, one, one, one, one, 10, 8, 1, -1, 5, 2.0, 0.05, None, None) == 1
    assert b"null pointer" in L.nessi_gpu_last_error()


def test_vie2_timestep_omp_order0_start_is_refused_without_a_device():
    """The reference dispatches vie2_timestep_omp(0, ...) to an order-0 vie2_start, which this
    library does not provide: the Python drop-in refuses it with NESSI_ERR_ARG before any device
    call."""
    import pytest
    from nessi_b200 import gpu, herm_matrix
    G = herm_matrix(8, 6, 1, -1)
    with pytest.raises(gpu.NessiGpuError) as e:
        gpu.vie2_timestep_omp(4, 0, G, G, G, G, 2.0, 0.05, 5)
    assert e.value.code == 1
