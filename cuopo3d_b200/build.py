"""Build recipe for the in-tree CUDA library cuopo3d_b200/libcuopo3d.so (sm_100a).

    python -m cuopo3d_b200.build          # or __graft_entry__.build()
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcuopo3d.so")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("ssfm_kernels.cu", "opo_host.cu", "noalloc_sums.cu", "batch.cu",
                                                             "init_fields.cu", "serve.cpp", "plane_pass.cu", "ws_pass.cu", "peaks.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("fft_radix.cuh", "opo_internal.h", "pass_body.cuh",
                                                   "solver_internal.h")] + [
    os.path.join(ROOT, "include", "cuopo3d.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-shared",
           "-I" + os.path.join(ROOT, "include"), *SOURCES, "-o", LIB]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
