"""Build recipe for the in-tree CUDA library cuopo3d_b200/libcuopo3d.so (sm_100a).

    python -m cuopo3d_b200.build          # or __graft_entry__.build()
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libcuopo3d.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = [os.path.join(HERE, "csrc", f) for f in ("ssfm_kernels.cu", "opo_host.cu", "noalloc_sums.cu", "batch.cu",
                                                             "init_fields.cu", "serve.cpp", "sweep.cpp", "writer.cpp", "plane_pass.cu", "ws_pass.cu", "tpass_line.cu",
                                                                     "peaks.cu")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in ("fft_radix.cuh", "fft_gain.h", "opo_internal.h", "pass_body.cuh", "tpass_line.cuh",
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


def _compile(src, obj, verbose):
    cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include"),
           "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)


def build(force=False, verbose=False, jobs=None):
    """Compile every source to an object in parallel (one nvcc per file), then link."""
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.splitext(os.path.basename(f))[0] + ".o") for f in SOURCES]
    jobs = jobs or max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        for fut in [ex.submit(_compile, src, obj, verbose) for src, obj in zip(SOURCES, objs)]:
            fut.result()
    subprocess.run([nvcc(), *ARCH, "-shared", *objs, "-o", LIB], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
