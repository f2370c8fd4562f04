"""Gather maps whose sources include destinations run in one launch over connected components
(k_gather); tests/gather_components_check.cpp checks on the host, for every ghost pattern and
the vertex restriction over all combinations of six boundary options, that component-wise
application equals the all-reads-before-writes semantics bit for bit (CPU, g++)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "salec-2d-public_b200", "csrc")


def test_component_application_equals_two_pass(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no g++ on this machine")
    exe = str(tmp_path / "gather_components_check")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", CSRC, "-I", "/usr/local/cuda/include",
                    os.path.join(HERE, "gather_components_check.cpp"), os.path.join(CSRC, "salec_ghost.cpp"),
                    "-o", exe], check=True, capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("OK"), out.stdout
