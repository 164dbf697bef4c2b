"""Builds the sm_100a shared library ``libdampm_cuda.so`` in-tree with nvcc.

The FP64 kernels are compiled with ``--fmad=false`` so that every
multiply/add rounds separately, exactly as the reference's C++ evaluates the
same expressions; that is what makes the FP64 path bitwise reproducible
against the CPU restatement.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdampm_cuda.so")
SOURCES = ["step_kernels.cu", "ms_kernels.cu", "slab_kernels.cu", "dampm_api.cu",
           "cfl_noalloc.cu", "batch_api.cu", "data_json.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "dampm_cuda.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "--fmad=false", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-o", LIB + ".tmp"]
    # build options of the kernels (dampm_kernels.h, dampm_device.cuh), e.g.
    # DAMPM_NVCC_DEFS="-DDAMPM_P2G_CAP=384"
    cmd += os.environ.get("DAMPM_NVCC_DEFS", "").split()
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
