"""CPU check of the fused kernels' index arithmetic (tests/fused_geometry_check.cu)."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_fused_indices_in_bounds():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "geom")
        subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(HERE, "..", "include"),
                        "-o", exe, os.path.join(HERE, "fused_geometry_check.cu")], check=True, capture_output=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr
