"""Build the engine library in-tree: vmachine_b200/libvmc_b200.so (sm_100a).

    python -m vmachine_b200.build [--verbose-ptxas]

nvcc cross-compiles without a GPU, so this runs in the build container; the
resulting .so travels with the source tree.  The translation units compile in
parallel: the host engine, and the FP32 and FP64 kernel instantiations.
"""
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvmc_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["vmc_engine.cu", "vmc_inst_f32.cu", "vmc_inst_f64.cu", "vmc_config.cpp",
           "vmc_noalloc.cu", "vmc_general.cu", "vmc_batch.cu", "vmc_batch_f32.cu", "vmc_batch_f64.cu",
           "vmc_blocking.cu", "vmc_checkpoint.cu", "vmc_density.cu"]
HEADERS = ["vmc_device.cuh", "vmc_kernels.cuh", "vmc_sweep.cuh", "vmc_config.hpp", "vmc_general.hpp",
           "vmc_general_dev.cuh", "vmc_engine.hpp", "vmc_batch_kernels.cuh", "vmc_mlp.cuh",
           "vmc_owner_sweep.cuh"]
FLAGS = ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]


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
    inc = ["-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
    extra = ["-Xptxas=-v"] if verbose_ptxas else []
    with tempfile.TemporaryDirectory(prefix="vmc_build_") as tmp:
        procs, objs = [], []
        for src in SOURCES:
            obj = os.path.join(tmp, src + ".o")
            objs.append(obj)
            cmd = [NVCC, *ARCH, *FLAGS, *extra, *inc, "-c", os.path.join(CSRC, src), "-o", obj]
            procs.append((src, subprocess.Popen(cmd)))
        failed = [src for src, p in procs if p.wait() != 0]
        if failed:
            raise RuntimeError(f"nvcc failed on {failed}")
        subprocess.run([NVCC, *ARCH, "-shared", "-o", LIB, *objs], check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv)
    print(LIB)
