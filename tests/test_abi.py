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
