"""ctypes binding of the CPU oracle (the reference compiled by oracle/Makefile).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
legs, never by the product. All arrays are returned in the reference's own layout: one
row-major (y, x, component) block per field, i.e. its AoS ``field_var.data`` with the
x index fastest (src/mpi_vec/mpi_vec.h:372-376).

The reference keeps global state, so one process hosts one oracle run at a time; use
``run_isolated`` to run oracle work in a fresh process started with ``spawn``.
"""
from __future__ import annotations

import ctypes
import multiprocessing as mp
import os
from typing import Callable, Dict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libsalec_ref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle library missing: build it with `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        c_d, c_i, c_s = ctypes.c_double, ctypes.c_int, ctypes.c_char_p
        pd = ctypes.POINTER(c_d)
        pi = ctypes.POINTER(c_i)
        sig = {
            "ref_init": ([c_s, c_s, c_s], c_i), "ref_init_begin": ([c_s, c_s, c_s], c_i),
            "ref_init_material": ([], c_i), "ref_init_finish": ([], c_i),
            "ref_phase": ([c_i], c_i), "ref_phases": ([c_i, c_i], c_i), "ref_step": ([], c_i),
            "ref_run": ([c_i], c_i), "ref_write_output": ([], c_i),
            "ref_field_dims": ([c_s, pi], c_i), "ref_get_field": ([c_s, pd], c_i),
            "ref_set_field": ([c_s, pd], c_i), "ref_get_scalar": ([c_s, pd], c_i),
            "ref_set_scalar": ([c_s, c_d], c_i), "ref_get_material": ([c_i, c_s, pd], c_i),
            "ref_get_material_str": ([c_i, c_s, c_s, c_i], c_i), "ref_eos_type": ([c_i], c_i),
            "ref_get_tillotson": ([c_i, pd, pd, pd, pi], c_i),
            "ref_get_table": ([c_i, pi, pi, pd, pd, pd], c_i),
            "ref_eos_state": ([c_i, c_d, c_d, c_d, c_d, pd], c_i),
            "ref_tracer_count": ([], c_i), "ref_get_tracers": ([pd], c_i),
            "ref_ghost_fill": ([c_s], c_i), "ref_restrict": ([c_s], c_i),
            "ref_init_adopt": ([c_d], c_i),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _pd(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError("oracle call %s failed with %d" % (what, rc))


def init(deck: str, eosdir: str, workdir: str, material: bool = True) -> None:
    L = lib()
    _check(L.ref_init_begin(deck.encode(), eosdir.encode(), workdir.encode()), "init_begin")
    if material:
        _check(L.ref_init_material(), "init_material")
        _check(L.ref_init_finish(), "init_finish")


def init_adopt(damp_time: float) -> None:
    """After init(..., material=False) and set() of every field: make the adopted state steppable."""
    _check(lib().ref_init_adopt(float(damp_time)), "init_adopt")


def init_material() -> None:
    _check(lib().ref_init_material(), "init_material")


def init_finish() -> None:
    _check(lib().ref_init_finish(), "init_finish")


def phase(p: int) -> None:
    _check(lib().ref_phase(p), "phase %d" % p)


def phases(first: int, last: int) -> None:
    _check(lib().ref_phases(first, last), "phases")


def step(n: int = 1) -> None:
    _check(lib().ref_run(n), "run")


def dims(name: str):
    d = (ctypes.c_int * 3)()
    _check(lib().ref_field_dims(name.encode(), d), "dims " + name)
    return int(d[0]), int(d[1]), int(d[2])


def get(name: str) -> np.ndarray:
    """Field as an array of shape (ny, nx, ncomp)."""
    nx, ny, nc = dims(name)
    out = np.empty((ny, nx, nc), dtype=np.float64)
    _check(lib().ref_get_field(name.encode(), _pd(out)), "get " + name)
    return out


def set(name: str, arr: np.ndarray) -> None:  # noqa: A001 - mirrors the driver's name
    nx, ny, nc = dims(name)
    a = np.ascontiguousarray(arr, dtype=np.float64).reshape(ny, nx, nc)
    _check(lib().ref_set_field(name.encode(), _pd(a)), "set " + name)


def scalar(name: str) -> float:
    v = ctypes.c_double()
    _check(lib().ref_get_scalar(name.encode(), ctypes.byref(v)), "scalar " + name)
    return float(v.value)


def set_scalar(name: str, value: float) -> None:
    _check(lib().ref_set_scalar(name.encode(), float(value)), "set_scalar " + name)


def material(matid: int, name: str) -> float:
    v = ctypes.c_double()
    _check(lib().ref_get_material(matid, name.encode(), ctypes.byref(v)), "material " + name)
    return float(v.value)


def material_str(matid: int, name: str) -> str:
    buf = ctypes.create_string_buffer(128)
    _check(lib().ref_get_material_str(matid, name.encode(), buf, 128), "material_str " + name)
    return buf.value.decode()


def eos_type(matid: int) -> int:
    return int(lib().ref_eos_type(matid))


def tillotson(matid: int):
    n = ctypes.c_int()
    _check(lib().ref_get_tillotson(matid, None, None, None, ctypes.byref(n)), "tillotson n")
    p = np.zeros(13)
    x = np.zeros(n.value)
    y = np.zeros(n.value)
    _check(lib().ref_get_tillotson(matid, _pd(p), _pd(x), _pd(y), ctypes.byref(n)), "tillotson")
    return p, x, y


def table(matid: int):
    nt, nd = ctypes.c_int(), ctypes.c_int()
    _check(lib().ref_get_table(matid, ctypes.byref(nt), ctypes.byref(nd), None, None, None), "table n")
    xt, yd = np.zeros(nt.value), np.zeros(nd.value)
    data = np.zeros((nt.value, nd.value, 3))
    _check(lib().ref_get_table(matid, ctypes.byref(nt), ctypes.byref(nd), _pd(xt), _pd(yd), _pd(data)), "table")
    return xt, yd, data


def eos_state(matid: int, den: float, eng: float, plim: float, pty: float = 1.0):
    out = np.zeros(3)
    _check(lib().ref_eos_state(matid, den, eng, plim, pty, _pd(out)), "eos_state")
    return out


def tracers() -> np.ndarray:
    n = lib().ref_tracer_count()
    out = np.zeros((max(n, 1), 12))
    m = lib().ref_get_tracers(_pd(out))
    return out[:m]


def ghost_fill(name: str) -> None:
    _check(lib().ref_ghost_fill(name.encode()), "ghost_fill " + name)


def restrict(name: str) -> None:
    _check(lib().ref_restrict(name.encode()), "restrict " + name)


def write_output() -> None:
    _check(lib().ref_write_output(), "write_output")


def _child(fn, args, q):
    try:
        q.put(("ok", fn(*args)))
    except BaseException as e:  # report any failure to the parent
        import traceback
        q.put(("err", "%s\n%s" % (e, traceback.format_exc())))


def run_isolated(fn: Callable, *args, timeout: float = 3600.0):
    """Run ``fn(*args)`` (a module-level function) in a fresh spawned process; return its result."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(fn, args, q))
    p.start()
    try:
        status, val = q.get(timeout=timeout)
    finally:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    if status != "ok":
        raise RuntimeError("isolated oracle run failed: " + val)
    return val
