"""Build recipe for libnessi_gpu.so (in-tree, sm_100a) and libnessi_io.so (host only).

``python -m nessi_b200.build`` compiles nessi_b200/csrc/*.cu with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` into nessi_b200/libnessi_gpu.so, and the text
checkpoint format (csrc/hm_text_io.cpp) with g++ into nessi_b200/libnessi_io.so.
No GPU is needed to build.
"""
import os
import subprocess
import time
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libnessi_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "-ccbin", "/usr/bin/g++"]
SOURCES = ["nessi_gpu.cu"]
IO_LIB = os.path.join(HERE, "libnessi_io.so")
IO_SOURCES = [os.path.join(CSRC, "hm_text_io.cpp"), os.path.join(os.path.dirname(HERE), "include", "nessi_io.h")]
CXX = "/usr/bin/g++"  # the host compiler nvcc uses for the CUDA library


def _inputs():
    out = []
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".inc", ".h")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(os.path.dirname(HERE), "include", "nessi_gpu.h"))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build_io(force=False, verbose=False):
    """libnessi_io.so: libcntr's herm_matrix text format, host code only."""
    if not force and os.path.exists(IO_LIB) and all(os.path.getmtime(f) <= os.path.getmtime(IO_LIB)
                                                    for f in IO_SOURCES):
        return IO_LIB
    tmp = IO_LIB + ".tmp"
    cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-o", tmp, IO_SOURCES[0]]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(tmp, IO_LIB)  # a process that has the old library loaded keeps its copy
    return IO_LIB


def build(force=False, verbose=False):
    build_io(force=force, verbose=verbose)
    if not force and up_to_date():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [NVCC] + FLAGS + ["-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd))
    start = time.time()
    subprocess.check_call(cmd, cwd=CSRC)
    os.replace(tmp, LIB)  # a process that has the old library loaded keeps its copy
    # stamp the library with the time the compile read its sources, so that a source edited
    # while nvcc ran is newer than the library and the next build compiles it
    os.utime(LIB, (start, start))
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print("built", LIB)
