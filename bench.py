#!/usr/bin/env python
"""Benchmark of the B200 per-timestep mesh update (cell-updates per second).

Workload: 2048 x 2048 cells, granite target on a seeded tabulated (density x specific
energy) EOS, ice Tillotson projectile at CPPR 40 and 15 km/s, rock strength with damage,
30-layer PML, FP64 plain form. One step = one full cycle of the reference's time loop
(src/salec2d.c:115-272) over the whole mesh, state resident in HBM.

Arms:
  default          the GPU library through its C ABI (include/salec_gpu.h)
  --impl reference the reference's own CPU step loop (the compiled reference in
                   oracle/_ref, one single-threaded reference process per host core, each on
                   its own bounded copy of the same workload, aggregate over a common window)

The default line also carries the mixed form (speed, and its accuracy against the FP64 form
after the timed cycles and after the configured 5000 cycles, with the transient crater depth),
the roofline of the dominant kernel, the end-to-end figure through host buffers and the CPU
baseline. --layered and --ensemble N run the layered-target and ensemble workloads instead.

Multi-GPU (torchrun): independent replicas, one simulation per GPU, no collective on the
data path; the reported value is the total over all ranks with the max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "salec-2d-public_b200"))
sys.path.insert(0, ROOT)

from salec_b200 import capi, decks, fields  # noqa: E402

METRIC = "cell-updates/s"
def workload(n: int) -> str:
    return "impact %dx%d cells, SieDen granite + Tillotson ice, CPPR 40, 15 km/s, PML 30, FP64" % (n, n)

# ---------------------------------------------------------------- algorithmic bytes model
# Bytes that each step kernel must move: every field its sweep reads, once, and every field
# it writes, once, at each point where the reference's algorithm touches that field (FP64,
# 8 bytes a value). Point classes, counted on the device state of the timed window:
#   C  interior cells                 V  active vertices (update + internal sections)
#   Cf cells holding no vacuum (vof0 <= 1e-6): the only cells whose stress and energy change
#   Cn cells that are not pure vacuum (vof0 < 1 - 1e-6)
#   L  damping-layer cells (sigma_x or sigma_y > 0) while t < damp_time
#   Cp all cells including the two-cell pad (surface profile sweep)
# Data-dependent extras are NOT counted, so the figures are lower bounds of what a launch
# needs: the upwind state members of a face record (read and written only on faces that
# carry flow), the cut-line reconstruction inputs of mixed cells, the void-vertex fills and
# the boundary gathers. Geometry that the reference stores per point (e_grad, v_vol, v_suf,
# v_subvol, v_laplace, e_pos, e_vol) is counted, since it is read from HBM, not recomputed.
def kernel_doubles(ph: int, k: dict, m: int, pml2: bool, damping: bool, porous: bool, acoustic: bool,
                   ntracers: int) -> float:
    C, V, Cf, Cn, L, Cp = k["C"], k["V"], k["Cf"], k["Cn"], k["L"], k["Cp"]
    if ph == 0:    # trace_profile: vof0, centre y
        return 2 * Cp
    if ph == 1:    # update_v_vof: m_vof (m) -> v_vof (m), and in the same sweep update_v_vel_inc:
        return m * C + m * V + 7 * C + 7 * V + k["T_v_vol"]   # e_wpt 4, e_den, e_dvel 2 | v_vel rw,
        #                                                        v_mass r1 w2 | v_vol table
    if ph == 3:    # update_e_vel: e_den, e_wpt 4, e_vel w2 | v_mass 2, v_vel 2
        return 7 * C + 4 * V
    if ph == 4:    # check_v_vel: e_den, e_wpt 4 (fills of void vertices are data-dependent)
        return 5 * C
    if ph == 5:    # gradvel + q + CFL: e_pos 3, vof0, csd, pre, den, e_vel 2 | v_vel 2; writes e_grad_vel 5,
        return 16 * C + 2 * V + k["T_e_grad"] + k["T_e_vol"]   # e_div_vel, e_q | e_grad, e_vol tables
    if ph == 7:    # stress: vof0, dam everywhere; vacuum cells write 7 zeros; full cells read ste 4, ste2s,
        d = 2 * C + 7 * (C - Cf) + (8 + m + 9 + 9) * Cf   # sta2s, tps, strength, m-1 vof, den, grad_vel 5,
        #                                                   mu, pre, tem, csd and write 9
        return d + (4 * Cf if acoustic else 0)
    if ph == 8:    # acceleration: v_subvol 4, v_suf 8, v_vol 4, v_vel 2, v_mass, v_bf 2, v_acc w2 | e_pre,
        #            e_q, e_ste 4, e_den; the Laplacian weights (9) only where one is non-zero (Vl), plus
        #            one mask bit per vertex
        return (7 * V + 9 * k["Vl"] + V / 64.0 + 7 * C + ((4 * V + 3 * C) if pml2 else 0)
                + k["T_v_subvol"] + k["T_v_suf"] + k["T_v_vol"])
    if ph == 9:    # v_dis: v_vel rw, v_acc | v_dis w
        return 8 * V
    if ph == 10:   # energy: vof0, den everywhere; full cells pre, q, div, grad_vel 5, ste 4, vof/den (m-1),
        d = 2 * C + (14 + 4 * (m - 1)) * Cf    # m_eng rw (m-1), e_cvs rw
        return d + ((2 * (m - 1) + 5) * Cf if porous else 0)
    if ph == 11:   # tracers: 12 members rw + 4 vertex displacements (2 each)
        return 32 * ntracers
    if ph == 12:   # flux: v_pos 2, v_dis 2 | m_vof m, e_vol; writes e_wpt 4 and m face volumes on 2 faces
        return (3 * m + 5) * C + 4 * V
    if ph == 14:   # remap: 2m face volumes, state 3m+9 in, 3m+11 out; EOS writes pre, csd, tem, mu;
        d = (8 * m + 24) * C   # damping reads sigma 2, dampref 2 on non-vacuum cells, 14 more in the layers
        if porous:
            d += 3 * (m + 1) * C
        if damping:
            d += 4 * Cn + (14 if pml2 else 10) * L
        return d
    return 0.0


def manifest_doubles(m: int, damp_type: int, porous: bool) -> float:
    """Whole-step lower bound per cell-update: every persistent field read once and written once
    (1 write for e_strength), read-only fields once, transient inter-phase arrays and separable
    geometry excluded. Cell rw: m_vof, m_den, m_eng (3m), e_ste 4, e_dvel 2, 12 scalars, e_wpt 4,
    e_vel 2, e_alpha 2 (pml, pml2, pml3); vertex rw: v_vel, v_acc, v_dis, v_mass (8), v_alpha 2
    (pml2, pml3); read-only: e_sigma 2, e_dampref 3, m_pty m, v_bf 2."""
    e_alpha = 2 if damp_type in (0, 1, 2) else 0
    v_alpha = 2 if damp_type in (1, 2) else 0
    rw = 3 * m + 4 + 2 + 12 + 4 + 2 + e_alpha + 8 + v_alpha
    ro = 2 + 3 + m + 2
    d = 2 * rw + 1 + ro
    if porous:
        d += 2 * (m - 1) + 2
    return d


PHASE_KERNELS = {0: "k_trace_profile", 1: "k_vertex_vof_momentum", 2: "-", 3: "k_cell_velocity",
                 4: "k_void_vertices", 5: "k_gradient_viscosity_cfl", 6: "k_finalize_dt", 7: "k_stress",
                 8: "k_vertex_acceleration", 9: "k_vertex_displacement", 10: "k_energy", 11: "k_tracers",
                 12: "k_flux", 13: "-", 14: "k_remap_damp_state", 15: "k_cycle"}


# ---------------------------------------------------------------- helpers
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel: str, cells: int):
    """DRAM bytes (read + write) of one launch of a kernel on the full workload, scaled from the
    committed ncu capture (profiles/ncu_summary.json: bytes per interior cell of the captured
    case, whose traffic grows in proportion to the cells), or None without a capture."""
    p = os.path.join(ROOT, "profiles", "ncu_summary.json")
    if not os.path.exists(p):
        return None
    try:
        with open(p) as f:
            d = json.load(f)
        per_cell = d["dram_bytes_per_cell"].get(kernel)
        return None if per_cell is None else per_cell * cells
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


def dense_top(e_den: np.ndarray, e_pos: np.ndarray, rho: float) -> np.ndarray:
    """Per interior column, the height where the density falls through rho above the highest
    cell at least that dense, interpolated linearly between that cell's centre and the next one
    up (NaN where no cell is that dense). Arrays in the reference layout (rows, columns,
    components)."""
    den = e_den[2:-2, 2:-2, 0]
    y = e_pos[2:-2, 2:-2, 1]
    rows = np.arange(den.shape[0])[:, None]
    k = np.where(den >= rho, rows, -1).max(axis=0)            # highest dense row per column
    cols = np.arange(den.shape[1])
    ok = k >= 0
    kk = np.clip(k, 0, den.shape[0] - 1)
    k1 = np.clip(kk + 1, 0, den.shape[0] - 1)
    d0, d1 = den[kk, cols], den[k1, cols]
    y0, y1 = y[kk, cols], y[k1, cols]
    frac = np.where((k1 > kk) & (d0 > d1), (d0 - rho) / np.where(d0 > d1, d0 - d1, 1.0), 0.0)
    return np.where(ok, y0 + frac * (y1 - y0), np.nan)


def crater_depth(e_den: np.ndarray, e_pos: np.ndarray, rho: float, surface: float) -> float:
    """Transient crater depth on the symmetry axis: the pre-impact surface height minus the top
    of the dense target (density >= rho, half the target's) in the column next to the axis. The
    vaporised plume above the floor is far less dense, so it does not count as surface."""
    return float(surface - dense_top(e_den, e_pos, rho)[0])


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_deck(n: int, folder: str) -> str:
    return decks.write_deck(decks.config2_deck(n=n), folder)


# ---------------------------------------------------------------- CPU reference leg
def _cpu_reference_worker(deck: str, eos_dir: str, steps: int, warmup: int, barrier, results) -> None:
    """One reference process of cpu_reference_cores: its own oracle instance (the reference
    keeps global state), started by the reference's own initialisation of the deck
    (src/salec2d.c:45-105: deck, EOS tables, geometry, hydrostatic target profile, materials),
    then timed between a common barrier and its own end. Nothing of this library runs here."""
    from oracle import ref
    run_dir = tempfile.mkdtemp(prefix="salec_cpu_run_")
    t0 = time.perf_counter()
    ref.init(deck, eos_dir, run_dir)
    init_s = time.perf_counter() - t0
    ref.step(warmup)
    barrier.wait()
    t0 = time.perf_counter()
    ref.step(steps)
    results.put((time.perf_counter() - t0, init_s))


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_reference_cores(n: int, steps: int, warmup: int, folder: str, procs: int):
    """The reference on every host core: the reference is an MPI code, single-threaded per rank,
    and the one-rank shim cannot split a domain, so each core runs its own reference process on
    its own n x n copy of the workload (the throughput an MPI run of procs ranks could reach at
    best, with no halo exchange). Each process starts from the reference's own initialisation of
    the same deck, steps `warmup` cycles, meets the others at a barrier and steps `steps` cycles;
    the rate is procs x n^2 x steps over the slowest process's time. Returns the rate, the
    slowest timed window and the slowest initialisation."""
    import multiprocessing as mp
    deck = make_deck(n, folder)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    results = ctx.Queue()
    workers = [ctx.Process(target=_cpu_reference_worker, args=(deck, folder, steps, warmup, barrier, results))
               for _ in range(procs)]
    for w in workers:
        w.start()
    got = [results.get(timeout=3600) for _ in workers]
    for w in workers:
        w.join()
    secs = max(g[0] for g in got)
    init_s = max(g[1] for g in got)
    return procs * n * n * steps / secs, secs, init_s


SAMPLE_WHY = ("the reference's own start-up of the 2048x2048 deck (its hydrostatic target profile and "
              "material placement) takes about 10 minutes and 7.3 GB per process, so each process starts "
              "and steps its own n x n copy of the same deck")


def run_reference_arm(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    n = args.cpu_n
    procs = host_cores()
    with tempfile.TemporaryDirectory() as tmp:
        rate, secs, init_s = cpu_reference_cores(n, args.steps, args.warmup, tmp, procs)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(args.n), "sample": "%dx%d cells of the same deck" % (n, n),
                       "same_config": n == args.n, "sample_why": SAMPLE_WHY.replace("n x n", "%dx%d" % (n, n)),
                       "start": "the reference's own initialisation in every process (%.0f s)" % init_s,
                       "parallelism": "%d reference processes, one per host core, each on its own copy "
                                      "(single-threaded per rank, no halo exchange)" % procs},
            "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
                             "sample": "%d steps of a %dx%d-cell copy of the workload on each of %d processes"
                                       % (args.steps, n, n, procs)},
            "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
class Ranks:
    """Replica plumbing for N ranks (one process per GPU): a barrier and the MAX over ranks of a
    timing. No collective touches the simulation data. backend "nccl" on GPUs; "gloo" lets the
    same code run on CPU ranks."""

    def __init__(self, backend: str = "nccl", timeout_s: int = 300):
        import torch
        self.world, self.rank, self.local = dist_setup()
        self.dist = None
        self.device = "cuda" if backend == "nccl" else "cpu"
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
        self.torch = torch

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def all_max(self, x: float) -> float:
        if self.dist is None:
            return x
        t = self.torch.tensor([x], device=self.device, dtype=self.torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def snapshot(sim, torch):
    """Pinned host copy of a simulation's state: every step field, the tracers and the scalars."""
    st = {}
    for name in fields.STEP_FIELDS:
        a = sim.get_field(name)
        buf = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape)
        buf[...] = a
        st[name] = buf
    return {"fields": st, "tracers": sim.get_tracers(),
            "scalars": {k: sim.scalar(k) for k in ("dt", "time", "i_step")}}


def restore(sim, snap, perturb=None):
    """Upload a snapshot (optionally with m_den and m_eng scaled by 1 + perturb)."""
    for name, a in snap["fields"].items():
        sim.set_field(name, a * (1.0 + perturb) if perturb and name in ("m_den", "m_eng") else a)
    sim.set_tracers(snap["tracers"])
    for k, v in snap["scalars"].items():
        sim.set_scalar(k, v)


def kernel_report(sim, run, n, prof_steps, step_ms):
    """Per-kernel device times over prof_steps cycles (CUDA events around every phase on the
    library's stream), the algorithmic bytes of each kernel on the state reached, the dominant
    kernel's roofline and the step-level rooflines."""
    cells = n * n
    nmat = run.nmat
    pml2 = run.damp_type in (1, 2)
    sim.profile(True)
    sim.step(prof_steps)
    sim.sync()
    phase_ms, phase_cnt = sim.phase_times()
    sim.profile(False)
    # point classes of this state, for the algorithmic bytes of each kernel
    vof0 = sim.get_field("m_vof")[..., 0][2:-2, 2:-2]
    sig = sim.get_field("e_sigma")[2:-2, 2:-2]
    damping = run.damp_type != 5 and run.damp_time > sim.scalar("time")
    lap = sim.get_field("v_laplace")
    # geometry read through tables of distinct rows: each table counts once per launch
    tables = {}
    for gname in ("v_vol", "v_subvol", "v_suf", "e_grad", "e_vol"):
        a = sim.get_field(gname)
        rows = {a[j].tobytes() for j in range(a.shape[0])}
        nrow = len(rows) if len(rows) <= 512 and len(rows) < a.shape[0] else a.shape[0]
        tables["T_" + gname] = float(nrow * a.shape[1] * a.shape[2])
    counts = {"C": cells, "V": (n + 3) * (n + 3), "Cp": (n + 4) * (n + 4),
              "Vl": int(np.count_nonzero(np.any(lap != 0.0, axis=-1))), **tables,
              "Cf": int(np.count_nonzero(vof0 <= 1e-6)), "Cn": int(np.count_nonzero(vof0 < 1.0 - 1e-6)),
              "L": int(np.count_nonzero(((sig[..., 0] > 0) | (sig[..., 1] > 0)) & (vof0 < 1.0 - 1e-6)))}
    ntr = len(sim.get_tracers())
    kd = {p: kernel_doubles(p, counts, nmat, pml2, damping, bool(run.porosity_model), bool(run.acoustic_fluid),
                            ntr) for p in range(16)}
    hbm, peak_kind = load_peaks()
    dom = max(range(16), key=lambda p: phase_ms[p])
    dom_ms = phase_ms[dom] / max(phase_cnt[dom], 1)
    dom_bytes = 8.0 * kd[dom]
    achieved = dom_bytes / (dom_ms / 1000.0) / 1e9
    kernel_bytes_step = 8.0 * sum(kd.values())
    manifest_bytes = 8.0 * manifest_doubles(nmat, run.damp_type, bool(run.porosity_model)) * cells
    per_kernel = {PHASE_KERNELS[p]: {"ms": round(phase_ms[p] / phase_cnt[p], 4),
                                     "bytes": 8.0 * kd[p],
                                     "GBps": round(8.0 * kd[p] / (phase_ms[p] / phase_cnt[p] / 1000.0) / 1e9, 1),
                                     "frac": round(8.0 * kd[p] / (phase_ms[p] / phase_cnt[p] / 1000.0) / 1e9 / hbm, 3)}
                  for p in range(16) if phase_cnt[p] and kd[p] > 0}
    return {
        "cycle": int(sim.scalar("i_step")),
        "kernels": per_kernel,
        "kernel_ms": {PHASE_KERNELS[p]: round(phase_ms[p] / max(phase_cnt[p], 1), 4) for p in range(16)
                      if phase_cnt[p]},
        "roofline": {"bound": "hbm", "kernel": PHASE_KERNELS[dom], "achieved": achieved, "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": profile_traffic(PHASE_KERNELS[dom], cells), "bytes_per_launch": dom_bytes,
                     "launch_ms": dom_ms},
        "step_roofline": {"manifest_bytes_per_cell_update": manifest_bytes / cells,
                          "manifest_GBps": manifest_bytes / (step_ms / 1000.0) / 1e9,
                          "manifest_frac": manifest_bytes / (step_ms / 1000.0) / 1e9 / hbm,
                          "kernel_bytes_per_cell_update": kernel_bytes_step / cells,
                          "kernel_GBps": kernel_bytes_step / (step_ms / 1000.0) / 1e9,
                          "kernel_frac": kernel_bytes_step / (step_ms / 1000.0) / 1e9 / hbm},
        "point_classes": counts, "tracers": ntr,
    }


def crater_metrics(e_den: np.ndarray, e_pos: np.ndarray, rho: float, surface: float, dx: float) -> dict:
    """Transient-crater depth and radius from the top of the dense target (density >= rho, half the
    target's) per column: depth = the pre-impact surface minus that height in the column next to
    the axis; radius = the centre r of the first column, going out from the axis, where that
    height is back at the pre-impact surface (within a tenth of a cell)."""
    top = dense_top(e_den, e_pos, rho)
    r = e_pos[2:-2, 2:-2, 0][0]
    depth = float(surface - top[0])
    back = np.nonzero(np.nan_to_num(top, nan=-np.inf) >= surface - 0.1 * dx)[0]
    radius = float(r[back[0]]) if len(back) else None
    return {"depth_m": depth, "radius_m": radius}


def run_profile(sim, cycles: int, chunk: int, stream, torch, rho: float, surface: float, dx: float, e_pos):
    """Step `cycles` cycles in chunks; the device time of every chunk from CUDA events recorded
    around it on the library's stream (the sampling between chunks is outside them), and the
    crater depth and radius and the compensated conservation sums (salec_gpu_conservation) after
    every chunk. Returns the chunk times and the history, which starts with the sums before the
    first chunk."""
    per_chunk, hist = [], []
    hist.append({"cycle": int(sim.scalar("i_step")), "time_s": sim.scalar("time"), "conservation": sim.conservation()})
    for k in range(cycles // chunk):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(chunk)
        b.record(stream)
        b.synchronize()
        per_chunk.append(a.elapsed_time(b))
        cm = crater_metrics(sim.get_field("e_den"), e_pos, rho, surface, dx)
        cm.update({"cycle": int(sim.scalar("i_step")), "time_s": sim.scalar("time"), "conservation": sim.conservation()})
        hist.append(cm)
    return per_chunk, hist


def transient(hist):
    """The sample of largest depth: the transient crater (its cycle, time, depth and radius)."""
    hist = [h for h in hist if "depth_m" in h]
    k = max(range(len(hist)), key=lambda q: hist[q]["depth_m"])
    return {kk: v for kk, v in hist[k].items() if kk != "conservation"}


def conservation_report(hist):
    """Sums at the run's start and end and their relative change (total energy = internal +
    kinetic); the per-chunk series stays in the history."""
    a, b = hist[0]["conservation"], hist[-1]["conservation"]

    def rel(x, y):
        return (y - x) / abs(x) if x else None

    ea, eb = a["internal_energy"] + a["kinetic_energy"], b["internal_energy"] + b["kinetic_energy"]
    return {"start": a, "end": b, "summation": "Neumaier-compensated FP64 over the interior cells",
            "every": "chunk of cycles (see history)",
            "rel_change": {"mass": rel(a["mass"], b["mass"]), "total_energy": rel(ea, eb),
                           "momentum_z": rel(a["momentum_z"], b["momentum_z"])}}


def run_gpu_arm(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    ranks = Ranks("nccl")
    barrier, all_max = ranks.barrier, ranks.all_max

    n = args.n
    tmp = tempfile.mkdtemp(prefix="salec_bench_%d_" % rank)
    deck = make_deck(n, tmp)
    t0 = time.perf_counter()
    sim = capi.Simulation.from_deck(deck, tmp)
    init_s = time.perf_counter() - t0
    run = sim.get_run()
    nmat = run.nmat
    cells = n * n
    dx = float(decks.config2_deck(n=n).dx)
    snap0 = snapshot(sim, torch)          # the initial state (pinned host memory)
    e_pos = snap0["fields"]["e_pos"]
    den0 = snap0["fields"]["e_den"]
    rho_half = 0.5 * float(np.median(den0[den0 > 0.0]))    # half the target's density
    surface = float(np.nanmedian(dense_top(den0, e_pos, rho_half)))
    stream = torch.cuda.ExternalStream(sim.stream())

    # the timed window starts at cycle --start-cycle of the run (untimed cycles before it)
    if args.start_cycle > 0:
        sim.step(args.start_cycle)
    if args.block_shapes:   # shapes given (e.g. those a plain run tuned, for a profiler capture)
        shapes = {int(p): tuple(v) for p, v in json.loads(args.block_shapes).items()}
        sim.set_block_shapes(shapes)
    else:
        shapes = sim.autotune(cycles=4)   # untimed; block shapes of the 2-D sweeps for this state
    snap_start = snapshot(sim, torch) if args.start_cycle > 0 else snap0
    sim.step(args.warmup)
    sim.sync()
    sampler = ClockSampler(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    # timed region: K steps, nothing else on the stream (no per-phase events)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    launches0 = sim.scalar("launches")
    e0.record(stream)
    torch.cuda.nvtx.range_push("timed_cycles")   # lets a profiler select exactly these launches
    sim.step(args.steps)
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = int(sim.scalar("launches") - launches0)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier()
    ms_max = all_max(ms)
    value = world * cells * args.steps / (ms_max / 1000.0)
    step_ms = ms_max / args.steps

    # per-kernel times: a separate profiled pass right after the timed region
    rep = kernel_report(sim, run, n, min(args.steps, 50), step_ms)

    # end to end through the C ABI with host buffers: upload the window's start state from pinned
    # host memory, K steps each reading back dt, time and the surface profile, then download the
    # output field set
    out_fields = fields.OUTPUT_FIELDS
    h2d = sum(a.nbytes for a in snap_start["fields"].values()) + snap_start["tracers"].nbytes
    d2h_step = 80 + 8 * (n + 4)   # the 80-byte scalar block (dt, time, ...) and the surface profile
    d2h_out = sum(8 * np.prod(sim.shape(f)) for f in out_fields)
    out_bufs = {f: torch.empty(int(np.prod(sim.shape(f))), dtype=torch.float64, pin_memory=True).numpy()
                .reshape(sim.shape(f)) for f in out_fields}
    prof_bufs = [torch.empty(int(np.prod(sim.shape("y_profile"))), dtype=torch.float64,
                             pin_memory=True).numpy().reshape(sim.shape("y_profile")) for _ in range(2)]
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    restore(sim, snap_start)
    t_up = time.perf_counter()
    # every cycle's dt, time and surface profile are read back; cycle k+1 is queued before the
    # host waits for cycle k's results (salec_gpu_step_report_async, two report slots)
    sim.step_report_async(1, prof_bufs[0], 0)
    for k in range(1, args.steps):
        sim.step_report_async(1, prof_bufs[k % 2], k % 2)
        sim.report_wait((k - 1) % 2)
    sim.report_wait((args.steps - 1) % 2)
    t_loop = time.perf_counter()
    outs = [sim.get_field(f, out=out_bufs[f]) for f in out_fields]
    sim.sync()
    e2e_s = time.perf_counter() - t0
    e2e_parts = {"upload_s": t_up - t0, "cycles_s": t_loop - t_up, "download_s": e2e_s - (t_loop - t0)}
    e2e_s = all_max(e2e_s)
    e2e = world * cells * args.steps / e2e_s
    nbad = sim.check()

    # the whole configured run in the FP64 form: device time of every chunk of cycles, the crater
    # history, and the per-kernel table of the developed state at its end
    whole = None
    long64 = None
    fields_cmp = ("e_den", "e_pre", "m_eng", "m_vof", "v_vel", "e_ste", "e_dam")
    if args.long_cycles > 0:
        restore(sim, snap0)
        chunks, hist64 = run_profile(sim, args.long_cycles, args.chunk, stream, torch, rho_half, surface, dx, e_pos)
        total_ms = sum(chunks)
        long64 = {f: sim.get_field(f) for f in fields_cmp}
        late_k0 = min(len(chunks) - 1, 4000 // args.chunk)
        late = {"cycles": [late_k0 * args.chunk, (late_k0 + 1) * args.chunk],
                "ms_per_cycle": chunks[late_k0] / args.chunk,
                "value": cells / (chunks[late_k0] / args.chunk / 1000.0)}
        dev = kernel_report(sim, run, n, 50, chunks[-1] / args.chunk)
        whole = {"cycles": args.long_cycles, "chunk": args.chunk,
                 "mean_ms_per_cycle": total_ms / args.long_cycles,
                 "value": world * cells * args.long_cycles / (all_max(total_ms) / 1000.0),
                 "ms_per_cycle_by_chunk": [round(c / args.chunk, 4) for c in chunks],
                 "late_window": late, "developed_state": dev,
                 "crater_fp64": {"transient": transient(hist64), "final": transient(hist64[-1:])},
                 "conservation_fp64": conservation_report(hist64),
                 "nonfinite": sim.check()}

    # mixed form (FP32 storage of the relaxed fields): same deck, same window, then its state
    # against the plain FP64 form after the same number of cycles from the start
    mixed = None
    if not args.no_mixed:
        mix = capi.Simulation.from_deck(deck, tmp, precision=capi.PRECISION_MIXED)
        if args.start_cycle > 0:
            mix.step(args.start_cycle)
        mshapes = mix.autotune(cycles=4)
        mix.step(args.warmup)
        mix.sync()
        mstream = torch.cuda.ExternalStream(mix.stream())
        barrier()
        torch.cuda.synchronize()
        e0.record(mstream)
        mix.step(args.steps)
        e1.record(mstream)
        e1.synchronize()
        mms = all_max(e0.elapsed_time(e1))
        mvalue = world * cells * args.steps / (mms / 1000.0)
        total = args.start_cycle + args.warmup + args.steps
        restore(sim, snap0)
        sim.step(total)
        ref_state = {f: sim.get_field(f) for f in fields_cmp}
        errs = {f: rel_l2(mix.get_field(f), ref_state[f]) for f in fields_cmp}
        # sensitivity of the FP64 form itself: the same run with m_den and m_eng perturbed by 1e-7
        # relative at the start (the size of one FP32 rounding)
        restore(sim, snap0, perturb=1e-7)
        sim.step(total)
        sens = {f: rel_l2(sim.get_field(f), ref_state[f]) for f in fields_cmp}
        c64 = crater_metrics(ref_state["e_den"], e_pos, rho_half, surface, dx)
        c32 = crater_metrics(mix.get_field("e_den"), e_pos, rho_half, surface, dx)
        mixed = {"value": mvalue, "unit": "cell-updates/s", "ms_per_step": mms / args.steps,
                 "speedup_vs_fp64": mvalue / value,
                 "storage": "FP32 relaxed fields, FP64 m_vof/m_den/m_eng/m_pty/e_cvs/positions/volumes/face records",
                 "arithmetic": "f32 in the stress update, strength, damage, artificial viscosity, stress "
                               "divergence and EOS table interpolation; f64 in the Tillotson EOS (mu = rho/rho0 - 1 "
                               "cancels), remap, fluxes, volume fractions and energies",
                 "rel_l2_vs_fp64": errs, "cycles_compared": total,
                 "fp64_sensitivity_rel_l2": sens,
                 "crater": {"fp64": c64, "mixed": c32,
                            "measure": "top of density >= %.0f kg/m3 per column against the pre-impact surface"
                                       % rho_half},
                 "nonfinite": mix.check()}
        # the configured run length: the mixed form from its window to --long-cycles with the same
        # chunked sampling, against the FP64 whole run above
        if long64 is not None and args.long_cycles > total:
            mix.close()
            mix = capi.Simulation.from_deck(deck, tmp, precision=capi.PRECISION_MIXED)
            mix.set_block_shapes(mshapes)
            mstream = torch.cuda.ExternalStream(mix.stream())
            mchunks, hist32 = run_profile(mix, args.long_cycles, args.chunk, mstream, torch, rho_half, surface, dx,
                                          e_pos)
            long_mix = {f: rel_l2(mix.get_field(f), long64[f]) for f in fields_cmp}
            restore(sim, snap0, perturb=1e-7)
            pchunks, histp = run_profile(sim, args.long_cycles, args.chunk, stream, torch, rho_half, surface, dx,
                                         e_pos)
            t64, t32, tp = transient(hist64), transient(hist32), transient(histp)

            def rel(a, b):
                return None if a is None or b is None or b == 0 else abs(a - b) / abs(b)

            mixed["long_run"] = {
                "cycles": args.long_cycles, "time_s": hist64[-1]["time_s"],
                "mean_ms_per_cycle": sum(mchunks) / args.long_cycles,
                "speedup_vs_fp64_whole_run": sum(chunks) / sum(mchunks),
                "rel_l2_vs_fp64": long_mix,
                "fp64_sensitivity_rel_l2": {f: rel_l2(sim.get_field(f), long64[f]) for f in fields_cmp},
                "transient_crater": {"fp64": t64, "mixed": t32, "fp64_perturbed": tp,
                                     "depth_rel_err": rel(t32["depth_m"], t64["depth_m"]),
                                     "radius_rel_err": rel(t32["radius_m"], t64["radius_m"]),
                                     "fp64_sensitivity_depth": rel(tp["depth_m"], t64["depth_m"]),
                                     "fp64_sensitivity_radius": rel(tp["radius_m"], t64["radius_m"])},
                "final_crater": {"fp64": transient(hist64[-1:]), "mixed": transient(hist32[-1:]),
                                 "fp64_perturbed": transient(histp[-1:])},
                "conservation": {"fp64": conservation_report(hist64), "mixed": conservation_report(hist32)},
                "crater_history_fp64": hist64, "crater_history_mixed": hist32,
                "nonfinite": mix.check() + sim.check()}
        mix.close()

    cpu = None
    if rank == 0 and not args.no_cpu:
        procs = host_cores()
        with tempfile.TemporaryDirectory() as ctmp:
            rate, secs, cinit = cpu_reference_cores(args.cpu_n, args.cpu_steps, 2, ctmp, procs)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": procs, "kind": "reference",
               "sample": "%d steps of a %dx%d-cell copy of the workload on each of %d reference processes, "
                         "one per host core, each started by the reference's own initialisation (%.0f s); "
                         "timed window %.1f s" % (args.cpu_steps, args.cpu_n, args.cpu_n, procs, cinit, secs)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload(n), "cells": cells, "materials": nmat, "form": "plain FP64",
                       "window": "cycles %d-%d of the run (the timed K cycles after %d untimed cycles from the "
                                 "deck's initial state and W warm-up cycles)"
                                 % (args.start_cycle + args.warmup, args.start_cycle + args.warmup + args.steps,
                                    args.start_cycle),
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "state %.1f GB, each step moves >= %.1f GB > 126 MB L2 (no flush needed)"
                             % (h2d / 1e9, rep["step_roofline"]["kernel_bytes_per_cell_update"] * cells / 1e9),
                       "init_s": round(init_s, 2), "point_classes": rep["point_classes"], "tracers": rep["tracers"],
                       "block_shapes": {PHASE_KERNELS[p]: list(v) for p, v in shapes.items()},
                       "block_shapes_by_phase": {str(p): list(v) for p, v in shapes.items()},
                       "block_shapes_source": "given" if args.block_shapes else "autotuned"},
            "roofline": rep["roofline"],
            "step_roofline": rep["step_roofline"],
            "kernels": rep["kernels"],
            "kernel_ms": rep["kernel_ms"],
            "whole_run": whole,
            "e2e": {"value": e2e, "unit": "cell-updates/s", "parts": e2e_parts,
                    "h2d_bytes_per_step": int(h2d / args.steps),
                    "d2h_bytes_per_step": int(d2h_step + d2h_out / args.steps)},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "nonfinite": nbad,
            "mixed": mixed,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    ranks.close()


# ---------------------------------------------------------------- layered-target mode
def run_layered(args):
    """--layered: the layered three-material target (decks.config3_deck, n x n cells, porous
    regolith over basalt over dunite, seeded +-1% density noise) in the plain FP64 and the mixed
    form, each autotuned, warmed up and timed over --steps cycles with CUDA events; then the
    mixed form's relative L2 error against the FP64 form after the same cycles."""
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    ranks = Ranks("nccl")
    n = args.layered_n
    tmp = tempfile.mkdtemp(prefix="salec_layered_%d_" % rank)
    deck = decks.write_deck(decks.config3_deck(n=n), tmp)
    out, sims = {}, {}
    for form, prec in (("fp64", capi.PRECISION_FP64), ("mixed", capi.PRECISION_MIXED)):
        t0 = time.perf_counter()
        sim = capi.Simulation.from_deck(deck, tmp, precision=prec)
        init_s = time.perf_counter() - t0
        md, ed = decks.density_noise(sim.get_field("m_den"), sim.get_field("e_den"), seed=3 + rank)
        sim.set_field("m_den", md)
        sim.set_field("e_den", ed)
        shapes = sim.autotune(cycles=2)
        sim.step(args.warmup)
        sim.sync()
        stream = torch.cuda.ExternalStream(sim.stream())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ranks.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        sim.step(args.steps)
        e1.record(stream)
        e1.synchronize()
        ms = ranks.all_max(e0.elapsed_time(e1))
        sim.profile(True)
        sim.step(20)
        sim.sync()
        pms, pcnt = sim.phase_times()
        sim.profile(False)
        out[form] = {"value": world * n * n * args.steps / (ms / 1000.0), "ms_per_step": ms / args.steps,
                     "init_s": round(init_s, 2), "nonfinite": sim.check(),
                     "block_shapes": {PHASE_KERNELS[p]: list(v) for p, v in shapes.items()},
                     "kernel_ms": {PHASE_KERNELS[p]: round(pms[p] / pcnt[p], 4) for p in range(16) if pcnt[p]}}
        sims[form] = sim
    err = {}
    for f in ("e_den", "e_pre", "m_eng", "m_vof", "v_vel", "m_pty"):
        a, b = sims["mixed"].get_field(f), sims["fp64"].get_field(f)
        nb = float(np.linalg.norm(b))
        err[f] = float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": out["fp64"]["value"], "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["fp64"]["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "layered target %dx%d cells: porous regolith 500 m (25%%), basalt 3 km, dunite "
                                   "half-space; basalt projectile CPPR 30 at 10 km/s; PML 50 side / 30 base layers; "
                                   "+-1%% seeded density noise" % (n, n),
                       "materials": 4, "parallelism": "single GPU" if world == 1 else "replicas"},
            "forms": out, "mixed_speedup": out["mixed"]["value"] / out["fp64"]["value"],
            "mixed_rel_l2_vs_fp64": err, "cycles_compared": args.warmup + args.steps + 20}), flush=True)
    for s_ in sims.values():
        s_.close()
    ranks.close()


# ---------------------------------------------------------------- ensemble mode
def run_ensemble(args):
    """--ensemble N: N seeded impacts of uneven size (decks.ensemble_decks), each initialised from
    its deck by the library (host threads in parallel) and stepped --ens-steps cycles, all members
    together through salec_gpu_step_many. Reports simulations per hour, whole job (deck
    initialisation included) and device stepping alone."""
    import concurrent.futures as cf
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    ranks = Ranks("nccl")
    members = decks.ensemble_decks(args.ensemble, seed=args.ens_seed + rank)
    tmp = tempfile.mkdtemp(prefix="salec_ens_%d_" % rank)
    paths = []
    for k, d in enumerate(members):
        folder = os.path.join(tmp, "m%04d" % k)
        paths.append((decks.write_deck(d, folder), folder))
    prec = capi.PRECISION_MIXED if args.ens_precision == "mixed" else capi.PRECISION_FP64
    ranks.barrier()
    t0 = time.perf_counter()

    def make(pf):
        torch.cuda.set_device(local)
        return capi.Simulation.from_deck(pf[0], pf[1], precision=prec)

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        sims = list(ex.map(make, paths))
    if args.ens_autotune:
        # block shapes tuned once, on the largest member, and shared: part of the timed
        # initialisation
        big = max(sims, key=lambda s: s.run.nx * s.run.ny)
        tuned = big.autotune(cycles=2)
        for s in sims:
            if s is not big:
                s.set_block_shapes(tuned)
    torch.cuda.synchronize()
    init_s = ranks.all_max(time.perf_counter() - t0)
    cells = [s.run.nx * s.run.ny for s in sims]
    ranks.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    capi.step_many(sims, args.ens_steps, chunk=args.ens_chunk)
    for s in sims:
        s.sync()
    e1.record()   # after every member's stream has drained
    e1.synchronize()
    run_s = ranks.all_max(e0.elapsed_time(e1) / 1000.0)
    nbad = sum(s.check() for s in sims)
    for s in sims:
        s.close()
    ranks.close()
    if rank == 0:
        n = len(sims) * world
        line = {"metric": "ensemble sims/h", "value": n / (init_s + run_s) * 3600.0, "unit": "simulations/h",
                "n_gpus": world, "steps": args.ens_steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if prec == capi.PRECISION_FP64 else "f32 storage / f64 arithmetic",
                "data": "synthetic",
                "config": {"workload": "ensemble of %d seeded basalt impacts, grids U[128,1024]^2, 5-20 km/s, CPPR "
                                       "10-40, cohesion 1-100 MPa, friction 0.6-1.4, PML" % args.ensemble,
                           "members": len(sims), "cells_total": int(sum(cells)), "cycles_each": args.ens_steps,
                           "chunk": args.ens_chunk, "seed": args.ens_seed},
                "init_s": init_s, "run_s": run_s,
                "device_sims_per_h": n / run_s * 3600.0,
                "cell_updates_per_s": world * sum(cells) * args.ens_steps / run_s,
                "timing": "stepping: CUDA events bracketing all members' streams, max over ranks; "
                          "initialisation: host wall clock, max over ranks",
                "nonfinite": int(nbad)}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- adjoint mode
def column_heights(sim) -> np.ndarray:
    vof, pos = sim.get_field("m_vof"), sim.get_field("e_pos")
    return ((1.0 - vof[2:-2, 2:-2, 0]) * pos[2:-2, 2:-2, 3]).sum(axis=0)


def run_adjoint(args):
    """--adjoint: the adjoint of a window of --adj-steps cycles (checkpoint every --adj-every) on the
    basalt deck of decks.config5_deck (n x n cells, CPPR 20, 8 km/s, Drucker-Prager as RockStrengthT
    cohesion/friction, no damping layers), for the misfit of the final surface-height profile against
    a seeded target. Times the forward window and the adjoint window with CUDA events on the
    library's stream, and checks the cohesion, friction, impactor-speed and density gradients
    against FP64 central finite differences (relative step 1e-6; 1e-8 along a smooth density
    direction; frozen time steps)."""
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    ranks = Ranks("nccl")
    n = args.adj_n
    base = dict(n=n, cohesion=1.0e7, friction=1.2, velocity=8000.0, cppr=20.0)
    tmp = tempfile.mkdtemp(prefix="salec_adj_%d_" % rank)
    deck = decks.write_deck(decks.config5_deck(**base), tmp)
    sim = capi.Simulation.from_deck(deck, tmp)
    stream = torch.cuda.ExternalStream(sim.stream())
    h0 = column_heights(sim)
    target = decks.target_profile(h0, 50.0)
    v0, md0, ed0 = sim.get_field("v_vel"), sim.get_field("m_den"), sim.get_field("e_den")
    init_state = snapshot(sim, torch)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    # forward window (warm-up first), recording the time steps
    sim.step(args.warmup)
    restore(sim, init_state)
    sim.sync()
    dts = []
    ranks.barrier()
    ev[0].record(stream)
    for _ in range(args.adj_steps):
        sim.step(1)
    ev[1].record(stream)
    ev[1].synchronize()
    fwd_ms = ev[0].elapsed_time(ev[1])
    restore(sim, init_state)
    for _ in range(args.adj_steps):
        sim.step(1)
        dts.append(sim.scalar("dt"))
    r = column_heights(sim) - target
    J_fwd = 0.5 * float(np.sum(r * r))
    # adjoint window (its own forward pass, replays and reverse sweeps), once untimed
    restore(sim, init_state)
    sim.adjoint_window(args.adj_steps, args.adj_every, target, density=False)
    restore(sim, init_state)
    sim.sync()
    ranks.barrier()
    ev[2].record(stream)
    J, dp, dvs, gden = sim.adjoint_window(args.adj_steps, args.adj_every, target)
    ev[3].record(stream)
    ev[3].synchronize()
    adj_ms = ev[2].elapsed_time(ev[3])
    # the same window as one segment: every cycle's undo log is written during the forward pass
    # and nothing is replayed (the logs of the whole window fit in HBM at this size)
    restore(sim, init_state)
    sim.adjoint_window(args.adj_steps, args.adj_steps, target, density=False)
    restore(sim, init_state)
    sim.sync()
    ranks.barrier()
    ev[2].record(stream)
    J1, dp1, dvs1, _ = sim.adjoint_window(args.adj_steps, args.adj_steps, target, density=False)
    ev[3].record(stream)
    ev[3].synchronize()
    adj1_ms = ev[2].elapsed_time(ev[3])
    same = bool(J1 == J and abs(dvs1 - dvs) <= 1e-9 * abs(dvs))
    adj_ms_max, fwd_ms_max, adj1_ms_max = ranks.all_max(adj_ms), ranks.all_max(fwd_ms), ranks.all_max(adj1_ms)
    sim.close()

    def fd_run(kw, edit=None):
        d = decks.write_deck(decks.config5_deck(**{**base, **kw}), os.path.join(tmp, "fd"))
        s_ = capi.Simulation.from_deck(d, os.path.join(tmp, "fd"))
        if edit:
            edit(s_)
        s_.set_dt_schedule(dts)
        s_.step(len(dts))
        rr = column_heights(s_) - target
        s_.close()
        return 0.5 * float(np.sum(rr * rr))

    eps = 1e-6
    fd = {}
    c, f = base["cohesion"], base["friction"]
    fd["cohesion"] = (fd_run({"cohesion": c * (1 + eps)}) - fd_run({"cohesion": c * (1 - eps)})) / (2 * eps * c)
    fd["friction"] = (fd_run({"friction": f * (1 + eps)}) - fd_run({"friction": f * (1 - eps)})) / (2 * eps * f)
    fd["speed"] = (fd_run({}, lambda s_: s_.set_field("v_vel", v0 * (1 + eps))) -
                   fd_run({}, lambda s_: s_.set_field("v_vel", v0 * (1 - eps)))) / (2 * eps * base["velocity"])
    # the density direction: smooth random cosine modes up to order 2, relative step 1e-8 (the
    # misfit jumps where cells cross the TOLRHO/TOLQPRE thresholds, which a larger step reaches)
    eps_rho = 1e-8
    rng = np.random.default_rng(11)
    ny, nx = ed0.shape[:2]
    yy, xx = np.meshgrid(np.linspace(0.0, 1.0, ny), np.linspace(0.0, 1.0, nx), indexing="ij")
    ds = np.zeros((ny, nx))
    for a in range(3):
        for b in range(3):
            ds += rng.uniform(-1.0, 1.0) * np.cos(np.pi * a * xx) * np.cos(np.pi * b * yy)
    ds /= np.abs(ds).max()

    def rho_edit(sg):
        def e(s_):
            fac = 1.0 + sg * eps_rho * ds
            md = md0.copy()
            md[..., 1:] *= fac[..., None]
            s_.set_field("m_den", md)
            s_.set_field("e_den", ed0 * fac[..., None])
        return e

    fd["density_direction"] = (fd_run({}, rho_edit(1.0)) - fd_run({}, rho_edit(-1.0))) / (2 * eps_rho)
    adj = {"cohesion": float(dp[0] + dp[2]), "friction": float(dp[1] + dp[3]),
           "speed": float(dvs / base["velocity"]), "density_direction": float(np.sum(gden * ed0[..., 0] * ds))}
    rel = {k: abs(adj[k] - fd[k]) / max(abs(fd[k]), 1e-300) for k in adj}
    ranks.close()
    if rank == 0:
        cells = n * n
        print(json.dumps({
            "metric": "adjoint/forward cost", "value": adj_ms_max / fwd_ms_max, "unit": "ratio", "n_gpus": world,
            "steps": args.adj_steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "adjoint of %d cycles, %dx%d basalt, CPPR 20 at 8 km/s, Drucker-Prager as "
                                   "RockStrengthT (cohesion 10 MPa, friction 1.2), no damping layers" % (args.adj_steps, n, n),
                       "checkpoint_every": args.adj_every,
                       "functional": "0.5 sum_i (h_i - target_i)^2, h_i the material column height of interior "
                                     "column i at the window's end, seeded target (decks.target_profile)",
                       "timing": "CUDA events on the library's stream: forward window of --adj-steps cycles vs "
                                 "salec_gpu_adjoint_window (its forward pass, checkpoints, replays and reverse sweeps)"},
            "forward_ms": fwd_ms_max, "adjoint_ms": adj_ms_max,
            "single_segment": {"adjoint_ms": adj1_ms_max, "ratio": adj1_ms_max / fwd_ms_max,
                               "same_gradients": same},
            "forward_cell_updates_per_s": world * cells * args.adj_steps / (fwd_ms_max / 1000.0),
            "misfit": J, "misfit_forward": J_fwd,
            "gradients": {"adjoint": adj, "finite_difference": fd, "rel_err": rel,
                          "fd_step": "1e-6 relative (cohesion, friction, speed), 1e-8 relative along a smooth "
                                     "density direction; central, frozen time steps",
                          "d_params_raw": [float(x) for x in dp]},
            "nonfinite_grad_density": int(np.count_nonzero(~np.isfinite(gden)))}), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=2048, help="cells per side of the GPU workload")
    ap.add_argument("--cpu-n", type=int, default=256, help="cells per side of the CPU sample")
    ap.add_argument("--cpu-steps", type=int, default=200)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision form")
    ap.add_argument("--long-cycles", type=int, default=5000,
                    help="cycles of the whole-run timing and of the mixed-vs-FP64 accuracy run at the configured "
                         "length (0: skip)")
    ap.add_argument("--chunk", type=int, default=250, help="cycles per timed chunk of the whole run")
    ap.add_argument("--start-cycle", type=int, default=2500,
                    help="untimed cycles from the deck's initial state before the warm-up and timed window")
    ap.add_argument("--ensemble", type=int, default=0, help="run the ensemble mode with this many members")
    ap.add_argument("--ens-steps", type=int, default=2000)
    ap.add_argument("--ens-chunk", type=int, default=32)
    ap.add_argument("--ens-seed", type=int, default=2024)
    ap.add_argument("--ens-precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--ens-autotune", action="store_true",
                    help="tune the block shapes on the largest member and set them on every member")
    ap.add_argument("--layered", action="store_true",
                    help="run the layered three-material target (plain and mixed forms) instead")
    ap.add_argument("--layered-n", type=int, default=4096, help="cells per side of the layered target")
    ap.add_argument("--adjoint", action="store_true", help="run the adjoint window (configuration 5) instead")
    ap.add_argument("--adj-n", type=int, default=512, help="cells per side of the adjoint deck")
    ap.add_argument("--adj-steps", type=int, default=200)
    ap.add_argument("--adj-every", type=int, default=20)
    ap.add_argument("--block-shapes", default="",
                    help='JSON {phase: [x, y]} of block shapes to set instead of autotuning, '
                         'e.g. the "block_shapes_by_phase" of an earlier run')
    args = ap.parse_args()
    if args.warmup < 1:
        args.warmup = 1
    if args.adjoint and args.impl == "ours":
        run_adjoint(args)
    elif args.ensemble > 0 and args.impl == "ours":
        run_ensemble(args)
    elif args.layered and args.impl == "ours":
        run_layered(args)
    elif args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
