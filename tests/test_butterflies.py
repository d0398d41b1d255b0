"""The register butterflies of the pass kernels (cuopo3d_b200/csrc/fft_radix.cuh) are
__host__ __device__: compile them for the host and check them against the DFT
definition for every radix and both signs, in FP64 and FP32.  No GPU needed."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_butterflies_match_dft(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "bfly")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets",
                    os.path.join(HERE, "native", "butterfly_check.cu"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.skipif(shutil.which("nvcc") is None and not os.path.exists("/usr/local/cuda/bin/nvcc"),
                    reason="nvcc not available")
def test_fp32_pair_gain_compensation(tmp_path):
    """The FP32 transform pairs' gain compensation (cuopo3d_b200/csrc/fft_gain.h): its
    squared-magnitude network equals the brute-force row / column norms of the dense
    forward / inverse operators built with the FP32 constants, on radix-2/3/4/8/16 plans,
    and the compensated pair keeps the energy of white inputs to ~1e-10 where the plain
    FP32 pair drains ~1e-7 per application."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "gain")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets",
                    os.path.join(HERE, "native", "gain_check.cu"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
