"""The adjoint's dual numbers against central differences (CPU): tests/dual_check.cu is compiled
with nvcc and run on the host, where the dual type, the Tillotson EOS, RockStrengthT and the
flux geometry the reverse sweeps differentiate are ordinary host functions."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "salec-2d-public_b200", "csrc")


def test_dual_derivatives_match_central_differences(tmp_path):
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
    if nvcc is None:
        pytest.skip("no nvcc on this machine")
    exe = str(tmp_path / "dual_check")
    res = subprocess.run([nvcc, "-std=c++17", "-O2", "--expt-relaxed-constexpr", "-gencode",
                          "arch=compute_100a,code=sm_100a", "-I", CSRC, os.path.join(HERE, "dual_check.cu"), "-o", exe],
                         capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
