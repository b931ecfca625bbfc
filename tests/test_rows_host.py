"""The row-interval search of the pair generation, compiled for the host
(the functions are __host__ __device__) and compared with testing every cell."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_row_intervals_equal_brute_force(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    exe = str(tmp_path / "rows_check")
    subprocess.run([nvcc, "-O2", "-std=c++17", "-fmad=false", "-Xcompiler", "-ffp-contract=off", "-x", "cu",
                    "-I", os.path.join(ROOT, "shinobi_b200", "csrc"), os.path.join(ROOT, "tests", "cpp", "rows_check.cu"),
                    "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe, "4000"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0 noncontiguous 0" in r.stdout
