"""Build the sm_100a shared library ``libsalec_b200.so`` in-tree with nvcc.

The library has no dependency on torch or Python: it is the C ABI of include/salec_gpu.h.
Flags: ``-gencode arch=compute_100a,code=sm_100a`` (B200 only), ``--fmad=false`` so that no
multiply-add is contracted (the FP64 form keeps the reference's rounding), ``-lineinfo`` for
profiling. Links the system zlib for the output files.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)               # salec-2d-public_b200/
CSRC = os.path.join(ROOT, "csrc")
LIB = os.path.join(PKG, "libsalec_b200.so")
SOURCES = ["salec_step.cu", "salec_runtime.cu", "salec_init.cu", "salec_noalloc.cu", "salec_output.cu",
           "salec_conserve.cu", "salec_adjoint.cu", "salec_ghost.cpp"]
HEADERS = ["salec_device.cuh", "salec_kernels.h", "salec_deck.h", "salec_dual.cuh", "salec_adjoint.h"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-lineinfo",
              "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(ROOT), "include", "salec_gpu.h"))
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not _stale():
        return LIB
    cmd = ([nvcc()] + NVCC_FLAGS + (extra or []) + [os.path.join(CSRC, f) for f in SOURCES] +
           ["-lz", "-o", LIB + ".tmp"])
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
