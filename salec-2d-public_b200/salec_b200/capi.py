"""ctypes mirror of include/salec_gpu.h: the host-side interface of the B200 mesh update.

``Simulation`` owns one device handle. Fields cross the boundary in the reference's own
layout and are exposed here as numpy arrays of shape (points_y, points_x, components), the
shape of the reference's ``field_var.data`` viewed row by row.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Optional, Sequence

import numpy as np

from . import build as _build

c_d, c_i, c_ll = ctypes.c_double, ctypes.c_int, ctypes.c_longlong
P_D = ctypes.POINTER(c_d)

SALEC_OK = 0
OUT_WAIT = 1          # salec_gpu_write_output flags
OUT_TRACER_TXT = 2
STATUS = {0: "SALEC_OK", -1: "SALEC_ERR_ARG", -2: "SALEC_ERR_CUDA", -3: "SALEC_ERR_ALLOC",
          -4: "SALEC_ERR_STATE", -5: "SALEC_ERR_UNSUPPORTED", -6: "SALEC_ERR_NUMERIC"}
EOS_ANEOS, EOS_TILLOTSON, EOS_SIEDEN = 0, 1, 2
DAMP = {"pml": 0, "pml2": 1, "pml3": 2, "sbc": 3, "ctlg": 4, "none": 5}
NPHASE = 16


class RunDesc(ctypes.Structure):
    _fields_ = [("nx", c_i), ("ny", c_i), ("nmat", c_i), ("damp_type", c_i), ("go", c_i * 4),
                ("partpres", c_i), ("porosity_model", c_i), ("acoustic_fluid", c_i), ("tensile_failure", c_i),
                ("tracer_lubrication", c_i), ("tracer_lub_gy0", c_i), ("tracer_lub_gy1", c_i),
                ("avis1", c_d), ("avis2", c_d), ("anc", c_d),
                ("density_cutoff", c_d), ("velocity_max", c_d), ("velocity_min", c_d), ("acceleration_min", c_d),
                ("alpha_damp_x", c_d), ("alpha_damp_y", c_d), ("damp_time", c_d),
                ("threshold_z", c_d), ("flow_resistance", c_d), ("flow_friction", c_d),
                ("tracer_lub_y0", c_d), ("tracer_lub_frac", c_d),
                ("max_dt", c_d), ("dt", c_d), ("time", c_d), ("i_step", c_i), ("precision", c_i)]

class AdjointResult(ctypes.Structure):
    _fields_ = [("misfit", c_d), ("d_params", c_d * 4), ("d_velocity_scale", c_d)]


PRECISION_FP64 = 0    # salec_precision: plain FP64 (bit-parity form)
PRECISION_MIXED = 1   # FP32 storage of the relaxed fields, FP32 arithmetic of stress, strength and viscosity


MAT_DOUBLES = ["VaporDen", "MeltDen", "GaCoef", "Yint0", "Yfricint", "Ylimint", "Ydam0", "Yfricdam", "Ylimdam",
               "Yten0", "IvanA", "IvanB", "IvanC", "Pbd", "Pbp", "minPint", "minPdam", "JCA", "JCB", "JCN", "JCC",
               "JCM", "JCTREF", "JCMaxPlastic", "Asimon", "Csimon", "Tmelt0", "Tfrac", "Tdelta"]
MAT_DOUBLES2 = ["Tlidc1", "Tlidc2", "Tlidc3", "Tsolc1", "Tsolc2", "Tsolc3", "Toff", "Cvib", "VibMax", "Tdamp",
                "Pvlim", "Acvis", "alpha0", "alphax", "epse0", "chi", "kappa", "avel", "epsec", "epsex",
                "alphamax", "alphamax2", "alphae", "gamfrac", "melt_viscosity"]


class MaterialDesc(ctypes.Structure):
    _fields_ = ([("eos_type", c_i), ("yfunc", c_i), ("tfunc", c_i), ("dsdf", c_i), ("porfunc", c_i)]
                + [(n, c_d) for n in MAT_DOUBLES]
                + [("PolyLiq", c_i), ("PolySol", c_i)]
                + [(n, c_d) for n in MAT_DOUBLES2]
                + [("till", c_d * 13), ("cold_n", c_i), ("cold_xden", P_D), ("cold_yeng", P_D),
                   ("ntem", c_i), ("nden", c_i), ("xtem", P_D), ("yden", P_D), ("data", P_D)])


_lib = None


def lib() -> ctypes.CDLL:
    """Load the in-tree library (building it first if it is missing or stale)."""
    global _lib
    if _lib is None:
        path = _build.LIB
        if not os.path.exists(path) or _build._stale():
            try:
                _build.build()
            except Exception as e:  # no nvcc on this machine: only a prebuilt library can be used
                if not os.path.exists(path):
                    raise RuntimeError("libsalec_b200.so is missing and cannot be built: %s" % e)
                # the prebuilt library is older than the sources: say so, it may not match them
                import warnings
                warnings.warn("libsalec_b200.so is older than its sources and the rebuild failed; "
                              "using the prebuilt library: %s" % str(e)[-400:], RuntimeWarning)
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        sig = {
            "salec_gpu_create": ([ctypes.POINTER(RunDesc), ctypes.POINTER(MaterialDesc), ctypes.POINTER(vp)], c_i),
            "salec_gpu_destroy": ([vp], c_i),
            "salec_gpu_field_index": ([ctypes.c_char_p], c_i),
            "salec_gpu_field_shape": ([vp, c_i, ctypes.POINTER(c_i), ctypes.POINTER(c_i), ctypes.POINTER(c_i)], c_i),
            "salec_gpu_set_field": ([vp, c_i, P_D, c_ll], c_i),
            "salec_gpu_get_field": ([vp, c_i, P_D, c_ll], c_i),
            "salec_gpu_step": ([vp, c_i], c_i),
            "salec_gpu_step_many": ([ctypes.POINTER(vp), c_i, c_i, c_i], c_i),
            "salec_gpu_step_report": ([vp, c_i, P_D, P_D, P_D, c_ll], c_i),
            "salec_gpu_step_report_async": ([vp, c_i, P_D, c_ll, c_i], c_i),
            "salec_gpu_report_wait": ([vp, c_i, P_D, P_D], c_i),
            "salec_gpu_autotune": ([vp, c_i, ctypes.POINTER(c_i)], c_i),
            "salec_gpu_set_block_shapes": ([vp, ctypes.POINTER(c_i), c_i], c_i),
            "salec_gpu_phases": ([vp, c_i, c_i], c_i),
            "salec_gpu_sync": ([vp], c_i),
            "salec_gpu_get_scalar": ([vp, ctypes.c_char_p, P_D], c_i),
            "salec_gpu_set_scalar": ([vp, ctypes.c_char_p, c_d], c_i),
            "salec_gpu_set_tracers": ([vp, c_i, P_D], c_i),
            "salec_gpu_get_tracers": ([vp, P_D, ctypes.POINTER(c_i)], c_i),
            "salec_gpu_check": ([vp, ctypes.POINTER(c_ll)], c_i),
            "salec_gpu_conservation": ([vp, P_D, c_i], c_i),
            "salec_gpu_set_dt_schedule": ([vp, P_D, c_i], c_i),
            "salec_gpu_adjoint_reset": ([vp], c_i),
            "salec_gpu_adjoint_set_field": ([vp, c_i, P_D, c_ll], c_i),
            "salec_gpu_adjoint_get_field": ([vp, c_i, P_D, c_ll], c_i),
            "salec_gpu_adjoint_phase": ([vp, c_i], c_i),
            "salec_gpu_adjoint_params": ([vp, P_D], c_i),
            "salec_gpu_adjoint_window": ([vp, c_i, c_i, P_D, P_D, c_i, P_D, c_ll, ctypes.POINTER(AdjointResult)], c_i),
            "salec_gpu_write_output": ([vp, ctypes.c_char_p, ctypes.c_char_p, c_i, c_i, c_i], c_i),
            "salec_gpu_output_wait": ([vp], c_i),
            "salec_gpu_func_index": ([ctypes.c_char_p], c_i),
            "salec_gpu_create_from_deck": ([ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(vp)], c_i),
            "salec_gpu_create_from_deck_ex": ([ctypes.c_char_p, ctypes.c_char_p, c_i, ctypes.POINTER(vp)], c_i),
            "salec_gpu_get_run": ([vp, ctypes.POINTER(RunDesc)], c_i),
            "salec_gpu_stream": ([vp, ctypes.POINTER(vp)], c_i),
            "salec_gpu_profile": ([vp, c_i], c_i),
            "salec_gpu_phase_times": ([vp, P_D, ctypes.POINTER(c_ll)], c_i),
            "salec_cfl_dt_noalloc": ([c_i, c_i, vp, vp, vp, vp, vp, vp, c_d, c_d, vp, vp], c_i),
            "salec_boundary_map": ([c_i, c_i, c_i, c_i, c_i, ctypes.POINTER(c_i), ctypes.POINTER(c_i),
                                    ctypes.POINTER(c_i), ctypes.POINTER(c_i), ctypes.POINTER(ctypes.c_uint)], c_i),
            "salec_gpu_last_error": ([], ctypes.c_char_p),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def step_many(sims, nsteps: int, chunk: int = 16) -> None:
    """Advance an ensemble of Simulations by nsteps cycles each, their kernels overlapping on
    the device (salec_gpu_step_many); returns once queued, sync() waits."""
    arr = (ctypes.c_void_p * len(sims))(*[s.h.value for s in sims])
    _check(lib().salec_gpu_step_many(arr, len(sims), int(nsteps), int(chunk)), "salec_gpu_step_many")


class SalecError(RuntimeError):
    def __init__(self, code: int, what: str):
        msg = lib().salec_gpu_last_error().decode(errors="replace")
        super().__init__("%s failed: %s (%s)" % (what, STATUS.get(code, code), msg))
        self.code = code


def _check(code: int, what: str) -> None:
    if code != SALEC_OK:
        raise SalecError(code, what)


def func_index(name: str) -> int:
    k = lib().salec_gpu_func_index(name.encode())
    if k < 0:
        raise ValueError("unknown strength/damage/porosity function %r" % name)
    return k


def field_index(name: str) -> int:
    k = lib().salec_gpu_field_index(name.encode())
    if k < 0:
        raise KeyError(name)
    return k


def boundary_map(kind: int, pattern: int, nx: int, ny: int, ncomp: int, go: Sequence[int]):
    """Gather map of a ghost (kind 0) or restriction (kind 1) table: arrays dst, src, ops."""
    g = (c_i * 4)(*go)
    n = c_i(0)
    _check(lib().salec_boundary_map(kind, pattern, nx, ny, ncomp, g, ctypes.byref(n), None, None, None),
           "boundary_map")
    dst = np.zeros(max(n.value, 1), np.int32)
    src = np.zeros(max(n.value, 1), np.int32)
    ops = np.zeros(max(n.value, 1), np.uint32)
    ip = ctypes.POINTER(c_i)
    _check(lib().salec_boundary_map(kind, pattern, nx, ny, ncomp, g, ctypes.byref(n), dst.ctypes.data_as(ip),
                                    src.ctypes.data_as(ip), ops.ctypes.data_as(ctypes.POINTER(ctypes.c_uint))),
           "boundary_map")
    return dst[: n.value], src[: n.value], ops[: n.value]


def cfl_dt_noalloc(nx: int, ny: int, vel_r: int, vel_z: int, csd: int, scale_r: int, scale_z: int,
                   vof_vacuum: int, dt_prev: float, max_dt: float, dt_out: int, stream: int = 0) -> None:
    """Enqueue the allocation-free CFL reduction; every pointer argument is a device address."""
    _check(lib().salec_cfl_dt_noalloc(nx, ny, vel_r, vel_z, csd, scale_r, scale_z, vof_vacuum, float(dt_prev),
                                      float(max_dt), dt_out, stream or None), "salec_cfl_dt_noalloc")


def apply_boundary_map(field: np.ndarray, dst, src, ops) -> np.ndarray:
    """Apply a gather map to a (ny, nx, ncomp) array on the host (numpy restatement of k_gather)."""
    f = field.reshape(-1, field.shape[-1])
    out = f.copy()
    nc = f.shape[1]
    for c in range(nc):
        op = (ops >> (3 * c)) & 7
        v = f[src, c]
        r = np.where(op == 0, v, np.where(op == 1, -1.0 * v, np.where(op == 2, np.abs(v),
                     np.where(op == 3, -np.abs(v), np.where(op == 4, 0.0, -0.0)))))
        out[dst, c] = r
    return out.reshape(field.shape)


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(P_D)


class Simulation:
    """One device-resident simulation (a salec_gpu handle)."""

    @classmethod
    def from_deck(cls, deck: str, eos_dir: str, precision: int = PRECISION_FP64) -> "Simulation":
        """Create a simulation from a reference input deck and its EOS folder (no reference code)."""
        self = cls.__new__(cls)
        self._keep = []
        h = ctypes.c_void_p()
        _check(lib().salec_gpu_create_from_deck_ex(deck.encode(), eos_dir.encode(), int(precision), ctypes.byref(h)),
               "salec_gpu_create_from_deck")
        self.h = h
        self.run = self.get_run()
        return self

    def get_run(self) -> RunDesc:
        r = RunDesc()
        _check(lib().salec_gpu_get_run(self.h, ctypes.byref(r)), "get_run")
        return r

    def stream(self) -> int:
        p = ctypes.c_void_p()
        _check(lib().salec_gpu_stream(self.h, ctypes.byref(p)), "stream")
        return int(p.value or 0)

    def profile(self, enable: bool) -> None:
        _check(lib().salec_gpu_profile(self.h, 1 if enable else 0), "profile")

    def phase_times(self):
        ms = (c_d * 16)()
        cnt = (c_ll * 16)()
        _check(lib().salec_gpu_phase_times(self.h, ms, cnt), "phase_times")
        return list(ms), list(cnt)

    def __init__(self, run: RunDesc, materials: Sequence[Dict]):
        """``materials``: one dict per material index (entry 0, vacuum, may be empty) with the
        MaterialDesc scalar fields plus ``till`` (13 values), ``cold_yeng`` (array) or
        ``xtem``/``yden``/``data`` arrays for tabulated kinds."""
        n = run.nmat
        arr = (MaterialDesc * n)()
        self._keep = []
        for m in range(1, n):
            spec = materials[m]
            md = arr[m]
            for k, v in spec.items():
                if k in ("till",):
                    for q in range(13):
                        md.till[q] = float(v[q])
                elif k in ("cold_yeng", "cold_xden", "xtem", "yden", "data"):
                    a = np.ascontiguousarray(v, dtype=np.float64).ravel()
                    self._keep.append(a)
                    setattr(md, k, _ptr(a))
                    if k == "cold_yeng":
                        md.cold_n = a.size
                else:
                    setattr(md, k, v)
        h = ctypes.c_void_p()
        _check(lib().salec_gpu_create(ctypes.byref(run), arr, ctypes.byref(h)), "salec_gpu_create")
        self.h = h
        self.run = run

    def close(self) -> None:
        if getattr(self, "h", None) is not None and self.h.value:
            lib().salec_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, name: str):
        nx, ny, nc = c_i(), c_i(), c_i()
        _check(lib().salec_gpu_field_shape(self.h, field_index(name), ctypes.byref(nx), ctypes.byref(ny),
                                           ctypes.byref(nc)), "field_shape")
        return ny.value, nx.value, nc.value

    def set_field(self, name: str, a: np.ndarray) -> None:
        shp = self.shape(name)
        b = np.ascontiguousarray(a, dtype=np.float64).reshape(shp)
        _check(lib().salec_gpu_set_field(self.h, field_index(name), _ptr(b), b.size), "set_field " + name)

    def get_field(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Download a field; `out`, when given, must be a C-contiguous float64 array of the
        field's shape (pinned host memory makes the copy a direct DMA)."""
        shp = self.shape(name)
        if out is None:
            out = np.empty(shp, dtype=np.float64)
        elif out.dtype != np.float64 or tuple(out.shape) != tuple(shp) or not out.flags.c_contiguous:
            raise ValueError(f"get_field {name}: out must be C-contiguous float64 of shape {shp}")
        _check(lib().salec_gpu_get_field(self.h, field_index(name), _ptr(out), out.size), "get_field " + name)
        return out

    def step(self, n: int = 1) -> None:
        _check(lib().salec_gpu_step(self.h, n), "step")

    def step_report(self, n: int = 1, profile: np.ndarray | None = None):
        """step(n), then (dt, time), and the surface profile into `profile` when given (a
        C-contiguous float64 array of y_profile's shape), with one synchronisation."""
        dt, t = c_d(), c_d()
        pp, pn = None, 0
        if profile is not None:
            shp = self.shape("y_profile")
            if profile.dtype != np.float64 or tuple(profile.shape) != tuple(shp) or not profile.flags.c_contiguous:
                raise ValueError("step_report: profile must be C-contiguous float64 of shape %s" % (shp,))
            pp, pn = _ptr(profile), profile.size
        _check(lib().salec_gpu_step_report(self.h, int(n), ctypes.byref(dt), ctypes.byref(t), pp, pn),
               "step_report")
        return dt.value, t.value

    def step_report_async(self, n: int, profile: np.ndarray | None, slot: int) -> None:
        """Queue step(n) and the read-back of dt, time and the surface profile into report slot
        `slot` without waiting (salec_gpu_step_report_async); `profile` should be page-locked."""
        pp, pn = None, 0
        if profile is not None:
            shp = self.shape("y_profile")
            if profile.dtype != np.float64 or tuple(profile.shape) != tuple(shp) or not profile.flags.c_contiguous:
                raise ValueError("step_report_async: profile must be C-contiguous float64 of shape %s" % (shp,))
            pp, pn = _ptr(profile), profile.size
        _check(lib().salec_gpu_step_report_async(self.h, int(n), pp, pn, int(slot)), "step_report_async")

    def report_wait(self, slot: int):
        """Wait for report slot `slot`; returns (dt, time) of its cycles."""
        dt, t = c_d(), c_d()
        _check(lib().salec_gpu_report_wait(self.h, int(slot), ctypes.byref(dt), ctypes.byref(t)), "report_wait")
        return dt.value, t.value

    def phases(self, first: int, last: int) -> None:
        _check(lib().salec_gpu_phases(self.h, first, last), "phases")

    def sync(self) -> None:
        _check(lib().salec_gpu_sync(self.h), "sync")

    def scalar(self, name: str) -> float:
        v = c_d()
        _check(lib().salec_gpu_get_scalar(self.h, name.encode(), ctypes.byref(v)), "get_scalar " + name)
        return v.value

    def set_scalar(self, name: str, value: float) -> None:
        _check(lib().salec_gpu_set_scalar(self.h, name.encode(), float(value)), "set_scalar " + name)

    def write_output(self, folder: str, prefix: str, out_step: int, rank: int = 0, wait: bool = True,
                     tracer_txt: bool = False) -> None:
        """Write the reference's .vts/.vtp (and optional tracer .txt) files of the current state
        under folder/vts, folder/vtp, folder/txt. Without wait the files are written by host
        threads while the device continues; output_wait() joins them."""
        flags = (OUT_WAIT if wait else 0) | (OUT_TRACER_TXT if tracer_txt else 0)
        _check(lib().salec_gpu_write_output(self.h, folder.encode(), prefix.encode(), rank, out_step, flags),
               "salec_gpu_write_output")

    def output_wait(self) -> None:
        _check(lib().salec_gpu_output_wait(self.h), "salec_gpu_output_wait")

    def autotune(self, cycles: int = 4) -> dict:
        """Pick the fastest block shape of every 2-D sweep for this mesh (state left unchanged);
        returns {phase: (block x, block y)}."""
        out = (c_i * 30)()
        _check(lib().salec_gpu_autotune(self.h, int(cycles), out), "salec_gpu_autotune")
        return {out[3 * k]: (out[3 * k + 1], out[3 * k + 2]) for k in range(10)}

    def set_block_shapes(self, shapes: dict) -> None:
        """Set block shapes {phase: (block x, block y)} of tunable sweeps (as autotune returns)."""
        items = sorted(shapes.items())
        arr = (c_i * (3 * max(len(items), 1)))()
        for k, (p, (bx, by)) in enumerate(items):
            arr[3 * k], arr[3 * k + 1], arr[3 * k + 2] = int(p), int(bx), int(by)
        _check(lib().salec_gpu_set_block_shapes(self.h, arr, len(items)), "salec_gpu_set_block_shapes")

    def check(self) -> int:
        n = c_ll()
        code = lib().salec_gpu_check(self.h, ctypes.byref(n))
        if code not in (SALEC_OK, -6):
            _check(code, "check")
        return n.value

    def conservation(self) -> Dict[str, object]:
        """Compensated FP64 conservation sums of the current state (salec_gpu_conservation):
        total mass, r and z momentum, internal and kinetic energy, mass per material."""
        nmat = self.get_run().nmat
        out = np.zeros(4 + nmat)
        _check(lib().salec_gpu_conservation(self.h, _ptr(out), len(out)), "salec_gpu_conservation")
        return {"mass": float(out[0]), "momentum_r": float(out[1]), "momentum_z": float(out[2]),
                "internal_energy": float(out[3]), "kinetic_energy": float(out[4]),
                "mass_by_material": [float(x) for x in out[5:]]}

    def set_dt_schedule(self, dts) -> None:
        """Prescribed time steps for the next len(dts) cycles (salec_gpu_set_dt_schedule)."""
        a = np.ascontiguousarray(dts, dtype=np.float64)
        _check(lib().salec_gpu_set_dt_schedule(self.h, _ptr(a) if a.size else None, int(a.size)),
               "salec_gpu_set_dt_schedule")

    # ---- adjoint (salec_gpu_adjoint_*)
    def adjoint_reset(self) -> None:
        _check(lib().salec_gpu_adjoint_reset(self.h), "salec_gpu_adjoint_reset")

    def adjoint_set(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _check(lib().salec_gpu_adjoint_set_field(self.h, field_index(name), _ptr(a), a.size), "adjoint_set " + name)

    def adjoint_get(self, name: str) -> np.ndarray:
        out = np.empty(self.shape(name), dtype=np.float64)
        _check(lib().salec_gpu_adjoint_get_field(self.h, field_index(name), _ptr(out), out.size), "adjoint_get " + name)
        return out

    def adjoint_phase(self, phase: int) -> None:
        _check(lib().salec_gpu_adjoint_phase(self.h, int(phase)), "salec_gpu_adjoint_phase")

    def adjoint_params(self) -> np.ndarray:
        out = np.zeros(4)
        _check(lib().salec_gpu_adjoint_params(self.h, _ptr(out)), "salec_gpu_adjoint_params")
        return out

    def adjoint_window(self, nsteps: int, every: int, target, weight=None, density: bool = True):
        """Adjoint of the next nsteps cycles (checkpoint every `every`) for the surface-height misfit
        against target; returns (misfit, d_params[4], d_velocity_scale, grad_density or None)."""
        t = np.ascontiguousarray(target, dtype=np.float64)
        w = None if weight is None else np.ascontiguousarray(weight, dtype=np.float64)
        res = AdjointResult()
        g = np.zeros(self.shape("e_den")[:2]) if density else None
        _check(lib().salec_gpu_adjoint_window(self.h, int(nsteps), int(every), _ptr(t), None if w is None else _ptr(w),
                                              t.size, None if g is None else _ptr(g), 0 if g is None else g.size,
                                              ctypes.byref(res)), "salec_gpu_adjoint_window")
        return res.misfit, np.array(res.d_params[:]), res.d_velocity_scale, g

    def set_tracers(self, rows: np.ndarray) -> None:
        r = np.ascontiguousarray(rows, dtype=np.float64).reshape(-1, 12)
        _check(lib().salec_gpu_set_tracers(self.h, r.shape[0], _ptr(r)), "set_tracers")

    def get_tracers(self) -> np.ndarray:
        n = c_i(0)
        _check(lib().salec_gpu_get_tracers(self.h, None, ctypes.byref(n)), "count tracers")
        out = np.zeros((max(n.value, 1), 12))
        _check(lib().salec_gpu_get_tracers(self.h, _ptr(out), ctypes.byref(n)), "get_tracers")
        return out[: n.value]
