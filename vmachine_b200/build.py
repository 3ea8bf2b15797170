"""Build the engine library in-tree: vmachine_b200/libvmc_b200.so (sm_100a).

    python -m vmachine_b200.build [--verbose-ptxas]

nvcc cross-compiles without a GPU, so this runs in the build container; the
resulting .so travels with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvmc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["vmc_engine.cu", "vmc_config.cpp"]
HEADERS = ["vmc_device.cuh", "vmc_kernels.cuh", "vmc_config.hpp"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "vmc_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose_ptxas=False):
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC, "-o", LIB,
           *[os.path.join(CSRC, f) for f in SOURCES]]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv)
    print(LIB)
