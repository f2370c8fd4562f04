"""The C ABI library on a machine without a GPU: it loads, exports every entry point that
include/salec_gpu.h declares, answers the host-only queries, and reports a missing device
as an error code with a message instead of crashing or falling back to the CPU."""
import ctypes
import os
import re
import subprocess

import pytest

from salec_b200 import build, capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "salec_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return sorted(set(re.findall(r"\b(salec_[a-z0-9_]+)\s*\(", text)))


def exported_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True, check=True)
    return {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}


def test_header_declares_the_entry_points():
    names = declared_functions()
    for must in ("salec_gpu_create", "salec_gpu_step", "salec_gpu_get_field", "salec_gpu_set_field",
                 "salec_gpu_destroy", "salec_cfl_dt_noalloc", "salec_boundary_map"):
        assert must in names


def test_library_exports_every_declared_symbol():
    capi.lib()
    missing = [n for n in declared_functions() if n not in exported_symbols()]
    assert not missing, "declared in include/salec_gpu.h but not exported: %s" % missing


def test_every_declared_symbol_resolves_through_ctypes():
    L = capi.lib()
    for n in declared_functions():
        assert getattr(L, n) is not None


def test_field_table_lookups():
    for name in ("v_vel", "e_den", "m_vof", "bx_phi", "by_phi", "y_profile", "e_dampref"):
        assert capi.field_index(name) >= 0
    with pytest.raises(KeyError):
        capi.field_index("no_such_field")


def test_strength_function_registry():
    for name in ("RockStrengthT", "Ivanov", "Collins", "SimpleTensile", "Wunnemann", "VonMises1"):
        assert capi.func_index(name) >= 0
    with pytest.raises(ValueError):
        capi.func_index("NotAStrengthModel")


def test_create_without_a_device_is_an_error_code():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    run = capi.RunDesc()
    run.nx, run.ny, run.nmat = 8, 8, 2
    mats = (capi.MaterialDesc * 2)()
    h = ctypes.c_void_p()
    rc = capi.lib().salec_gpu_create(ctypes.byref(run), mats, ctypes.byref(h))
    assert rc == -2
    assert not h.value
    assert capi.lib().salec_gpu_last_error().decode()


def test_bad_arguments_are_rejected_before_any_device_work():
    L = capi.lib()
    h = ctypes.c_void_p()
    assert L.salec_gpu_create(None, None, ctypes.byref(h)) == -1
    out = ctypes.c_double(0.0)
    rc = L.salec_cfl_dt_noalloc(0, 4, None, None, None, None, None, None, ctypes.c_double(1.0),
                                ctypes.c_double(1.0), ctypes.byref(out), None)
    assert rc == -1
    assert "null pointer" in L.salec_gpu_last_error().decode() or "empty" in L.salec_gpu_last_error().decode()
