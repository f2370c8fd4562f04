"""The bucket-guided EOS axis search returns exactly the bisection's index (CPU):
tests/axis_search_check.cu is compiled with nvcc and run on the host, where the search and the
bisection are ordinary host functions."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "salec-2d-public_b200", "csrc")


def test_axis_search_equals_bisection(tmp_path):
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
    if nvcc is None:
        pytest.skip("no nvcc on this machine")
    exe = str(tmp_path / "axis_search_check")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "-I", CSRC,
                    os.path.join(HERE, "axis_search_check.cu"), "-o", exe], check=True, capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
