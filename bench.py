#!/usr/bin/env python
"""Benchmark of the B200 per-timestep mesh update (cell-updates per second).

Workload: 2048 x 2048 cells, granite target on a seeded tabulated (density x specific
energy) EOS, ice Tillotson projectile at CPPR 40 and 15 km/s, rock strength with damage,
30-layer PML, FP64 plain form. One step = one full cycle of the reference's time loop
(src/salec2d.c:115-272) over the whole mesh, state resident in HBM.

Arms:
  default          the GPU library through its C ABI (include/salec_gpu.h)
  --impl reference the reference's own CPU step loop (the compiled reference in
                   oracle/_ref, single-threaded as the reference is), timed on a bounded
                   sample of the same workload

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
WORKLOAD = "impact 2048x2048 cells, SieDen granite + Tillotson ice, CPPR 40, 15 km/s, PML 30, FP64"

# ---------------------------------------------------------------- algorithmic bytes model
# Doubles that each step kernel must read and write once per point of its domain (fields
# touched x components, read and write counted separately). "c" = interior cells, "C" = all
# cells, "v" = active vertices; m = materials (with vacuum), phi = face record length.
def phase_doubles(m: int, phi: int, pml2: bool):
    return {
        0: [("C", 1 + 1 + 2)],                                   # vof0, y, e_ejt rw
        1: [("C", m), ("v", m)],                                 # m_vof -> v_vof
        2: [("C", 4 + 1 + 2), ("v", 4 + 2 * 2 + 2 * 2)],         # wpt, den, dvel | v_vol, v_vel rw, v_mass rw
        3: [("c", 1 + 4 + 2), ("v", 2 + 2)],                     # den, wpt, e_vel w | v_mass, v_vel
        4: [("C", 1 + 4), ("v", 2 * 2)],                         # den, wpt | v_vel rw
        5: [("c", 12 + 1 + 1 + 1 + 1 + 3 + 1 + 2 + 5 + 1 + 1), ("v", 2)],
        6: [],
        7: [("c", m + 1 + 2 * 4 + 2 * 3 + 1 + 1 + 5 + 1 + 1 + 1 + 1)],
        8: [("v", 4 + 8 + 4 + 9 + 2 + 2 + 1 + 2 + (4 if pml2 else 0)), ("C", 7 + (3 if pml2 else 0))],
        9: [("v", 2 * 2 + 2 + 2)],
        10: [("c", m + 1 + 1 + 1 + 1 + 5 + 4 + m + 2 * m + 2)],
        11: [],
        12: [("v", 2 + 2 + m), ("C", 8 + m + 1 + 2 + 2 * m + 2 + 4 + 4 + 4), ("f", phi)],
        13: [],
        14: [("f", 2 * phi), ("C", 2 * (3 * m) + 1 + 2 * 1 + 2 * 4 + 2 * 4 + 2 + 2 + 3 + 2 * 2 + 3 + 2 + 1 + 4)],
        15: [],
    }


def phase_bytes(ph: int, nx: int, ny: int, m: int, phi: int, pml2: bool) -> float:
    npts = {"c": nx * ny, "C": (nx + 4) * (ny + 4), "v": (nx + 3) * (ny + 3), "f": (nx + 4) * (ny + 4)}
    return 8.0 * sum(npts[d] * k for d, k in phase_doubles(m, phi, pml2)[ph])


PHASE_KERNELS = {0: "k_trace_profile", 1: "k_vertex_vof", 2: "k_vertex_momentum", 3: "k_cell_velocity",
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


def profile_traffic(kernel: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "ncu_summary.json")
    if not os.path.exists(p):
        return None
    try:
        with open(p) as f:
            d = json.load(f)
        return d.get("dram_bytes_per_launch_full_workload", {}).get(kernel)
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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
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


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_deck(n: int, folder: str) -> str:
    return decks.write_deck(decks.config2_deck(n=n), folder)


# ---------------------------------------------------------------- CPU reference leg
def cpu_reference(n: int, steps: int, warmup: int, folder: str, gpu_state=None):
    """Time the reference's own step loop (oracle/_ref) on an n x n sample of the workload.

    The reference starts from the state the GPU arm starts from: its geometry comes from its
    own init_mesh_pos, every field is then set from the deck initialiser's state (the
    reference's own target-profile search over the 512 x 512 table would take minutes).
    """
    from oracle import ref
    cwd = os.getcwd()
    deck = make_deck(n, folder)
    sim = capi.Simulation.from_deck(deck, folder) if gpu_state is None else None
    ref.init(deck, folder, os.path.join(folder, "run"), material=False)
    for name in fields.STEP_FIELDS:
        ref.set(name, sim.get_field(name) if sim is not None else gpu_state[name])
    damp = sim.get_run().damp_time if sim is not None else gpu_state["damp_time"]
    if sim is not None:
        sim.close()
    ref.init_adopt(damp)
    ref.step(warmup)
    t0 = time.perf_counter()
    ref.step(steps)
    dt = time.perf_counter() - t0
    os.chdir(cwd)   # the oracle works in its own folder
    return n * n * steps / dt, dt


def run_reference_arm(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    n = args.cpu_n
    with tempfile.TemporaryDirectory() as tmp:
        rate, secs = cpu_reference(n, args.steps, args.warmup, tmp)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": "%dx%d cells of the same deck" % (n, n),
                       "parallelism": "single host thread (the reference is single-threaded per rank)"},
            "cpu_baseline": {"value": rate, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
                             "sample": "%d steps of a %dx%d-cell copy of the workload" % (args.steps, n, n)},
            "e2e": {"value": rate, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU arm
def run_gpu_arm(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier()

    def all_max(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.n
    tmp = tempfile.mkdtemp(prefix="salec_bench_%d_" % rank)
    deck = make_deck(n, tmp)
    t0 = time.perf_counter()
    sim = capi.Simulation.from_deck(deck, tmp)
    init_s = time.perf_counter() - t0
    run = sim.get_run()
    nmat = run.nmat
    phi = 3 * nmat + 10 + (nmat + 1 if run.porosity_model else 0)
    pml2 = run.damp_type in (1, 2)
    cells = n * n

    # keep a host copy of the initial state for the end-to-end run (pinned host buffers)
    init_state = {}
    for name in fields.STEP_FIELDS:
        a = sim.get_field(name)
        buf = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy().reshape(a.shape)
        buf[...] = a
        init_state[name] = buf
    init_tracers = sim.get_tracers()

    sim.step(args.warmup)
    sim.sync()
    stream = torch.cuda.ExternalStream(sim.stream())
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    sampler.start()
    sim.profile(True)
    launches0 = sim.scalar("launches")
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    phase_ms, phase_cnt = sim.phase_times()
    launches = int(sim.scalar("launches") - launches0)
    sim.profile(False)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier()
    ms_max = all_max(ms)
    value = world * cells * args.steps / (ms_max / 1000.0)

    # dominant kernel and its roofline
    hbm, peak_kind = load_peaks()
    dom = max(range(16), key=lambda p: phase_ms[p])
    dom_ms = phase_ms[dom] / max(phase_cnt[dom], 1)
    dom_bytes = phase_bytes(dom, n, n, nmat, phi, pml2)
    achieved = dom_bytes / (dom_ms / 1000.0) / 1e9
    step_bytes = sum(phase_bytes(p, n, n, nmat, phi, pml2) for p in range(16))
    step_ms = ms / args.steps
    breakdown = {PHASE_KERNELS[p]: round(phase_ms[p] / max(phase_cnt[p], 1), 4) for p in range(16) if phase_cnt[p]}

    # end to end through the C ABI with host buffers: upload the initial state from pinned
    # host memory, K steps each reading back dt, time and the surface profile, then download
    # the output field set
    sim.set_scalar("time", 0.0)
    out_fields = fields.OUTPUT_FIELDS
    h2d = sum(a.nbytes for a in init_state.values()) + init_tracers.nbytes
    d2h_step = 8 * 2 + 8 * (n + 4)
    d2h_out = sum(8 * np.prod(sim.shape(f)) for f in out_fields)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for name, a in init_state.items():
        sim.set_field(name, a)
    sim.set_tracers(init_tracers)
    sim.set_scalar("dt", run.dt)
    for _ in range(args.steps):
        sim.step(1)
        sim.scalar("dt")
        sim.scalar("time")
        sim.get_field("y_profile")
    outs = [sim.get_field(f) for f in out_fields]
    sim.sync()
    e2e_s = time.perf_counter() - t0
    e2e_s = all_max(e2e_s)
    e2e = world * cells * args.steps / e2e_s
    nbad = sim.check()

    cpu = None
    if rank == 0 and not args.no_cpu:
        with tempfile.TemporaryDirectory() as ctmp:
            rate, secs = cpu_reference(args.cpu_n, args.cpu_steps, 2, ctmp)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": 1, "kind": "reference",
               "sample": "%d steps of a %dx%d-cell copy of the workload (%.1f s)" % (args.cpu_steps, args.cpu_n,
                                                                                   args.cpu_n, secs)}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": cells, "materials": nmat, "form": "plain FP64",
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "working set %.1f GB > 126 MB L2 (no flush needed)" % (step_bytes / 1e9),
                       "init_s": round(init_s, 2)},
            "roofline": {"bound": "hbm", "kernel": PHASE_KERNELS[dom], "achieved": achieved, "peak": hbm,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": profile_traffic(PHASE_KERNELS[dom]), "bytes_per_launch": dom_bytes,
                         "launch_ms": dom_ms},
            "step_roofline": {"algorithmic_bytes_per_cell_update": step_bytes / cells,
                              "achieved_GBps": step_bytes / (step_ms / 1000.0) / 1e9,
                              "frac": step_bytes / (step_ms / 1000.0) / 1e9 / hbm},
            "kernel_ms": breakdown,
            "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": int(h2d / args.steps),
                    "d2h_bytes_per_step": int(d2h_step + d2h_out / args.steps)},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
            "nonfinite": nbad,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=2048, help="cells per side of the GPU workload")
    ap.add_argument("--cpu-n", type=int, default=256, help="cells per side of the CPU sample")
    ap.add_argument("--cpu-steps", type=int, default=60)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 1:
        args.warmup = 1
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_gpu_arm(args)


if __name__ == "__main__":
    main()
