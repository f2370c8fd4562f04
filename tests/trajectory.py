"""Oracle trajectories for the GPU parity tests (test infrastructure).

``oracle_trajectory`` runs in a fresh spawned process (the reference keeps global state):
it writes a small synthetic deck, runs the reference's own initialisation, and records
the initial upload set plus the evolved fields after every step. The parent process then
drives the GPU library from the same initial state and compares.
"""
from __future__ import annotations

import concurrent.futures as cf
import multiprocessing as mp
import os
from typing import Dict, List

import numpy as np

import bridge
from bridge import ref

RUN_FIELDS = [n for n, _ in bridge.capi.RunDesc._fields_]


def oracle_trajectory(kind: str, nsteps: int, folder: str, phase_steps: int = 0) -> Dict:
    deck, folder = bridge.write_small_deck(kind, folder)
    ref.init(deck, folder, os.path.join(folder, "run"))
    run = bridge.run_desc_from_oracle()
    out = {
        "kind": kind,
        "run": {n: (list(getattr(run, n)) if n == "go" else getattr(run, n)) for n in RUN_FIELDS},
        "mats": bridge.materials_from_oracle(run.nmat),
        "init": {n: ref.get(n) for n in bridge.UPLOAD_FIELDS},
        "tracers0": ref.tracers(),
        "phases": [],
        "steps": [],
    }
    # optional phase-by-phase record of the first steps
    for s in range(phase_steps):
        for p in range(16):
            ref.phase(p)
            out["phases"].append({n: ref.get(n) for n in bridge.STATE_FIELDS})
    for s in range(phase_steps, nsteps):
        ref.step()
        rec = {n: ref.get(n) for n in bridge.STATE_FIELDS}
        rec["dt"] = ref.scalar("dt")
        rec["time"] = ref.scalar("time")
        rec["tracers"] = ref.tracers()
        out["steps"].append(rec)
    return out


def trajectories(kinds: List[str], nsteps: int, root: str, phase_steps: int = 0) -> Dict[str, Dict]:
    """Run several oracle trajectories in parallel spawned processes."""
    ctx = mp.get_context("spawn")
    workers = max(1, min(len(kinds), os.cpu_count() or 1))
    with cf.ProcessPoolExecutor(max_workers=workers, mp_context=ctx) as ex:
        futs = {k: ex.submit(oracle_trajectory, k, nsteps, os.path.join(root, k), phase_steps) for k in kinds}
        return {k: f.result() for k, f in futs.items()}


def simulation_from_record(rec: Dict, precision: int = 0):
    run = bridge.capi.RunDesc()
    for n, v in rec["run"].items():
        if n == "go":
            for k in range(4):
                run.go[k] = int(v[k])
        else:
            setattr(run, n, v)
    run.precision = precision
    sim = bridge.capi.Simulation(run, rec["mats"])
    for n, a in rec["init"].items():
        sim.set_field(n, a)
    sim.set_tracers(rec["tracers0"])
    return sim


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


def oracle_output_case(kind: str, nsteps: int, folder: str) -> Dict:
    """The reference's own output files of a mid-cycle state: nsteps cycles, then phases 0-13
    (the point where src/salec2d.c writes its VTK files), then sale2d_write_vtk/_vtp. Returns
    the state at that point (to load into the GPU library) and the bytes of every written file."""
    deck, folder = bridge.write_small_deck(kind, folder)
    run_dir = os.path.join(folder, "run")
    ref.init(deck, folder, run_dir)
    ref.step(nsteps)
    ref.phases(0, 13)
    run = bridge.run_desc_from_oracle()
    out = {
        "run": {n: (list(getattr(run, n)) if n == "go" else getattr(run, n)) for n in RUN_FIELDS},
        "mats": bridge.materials_from_oracle(run.nmat),
        "init": {n: ref.get(n) for n in bridge.UPLOAD_FIELDS},
        "tracers0": ref.tracers(),
        "files": {},
    }
    for sub in ("vts", "vtp", "txt"):
        d = os.path.join(run_dir, sub)
        for f in os.listdir(d):
            os.unlink(os.path.join(d, f))
    ref.write_output()
    for sub in ("vts", "vtp", "txt"):
        d = os.path.join(run_dir, sub)
        for f in sorted(os.listdir(d)):
            with open(os.path.join(d, f), "rb") as fh:
                out["files"][sub + "/" + f] = fh.read()
    return out


def oracle_output_cases(kinds: List[str], nsteps: int, root: str) -> Dict[str, Dict]:
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=max(1, min(len(kinds), os.cpu_count() or 1)), mp_context=ctx) as ex:
        futs = {k: ex.submit(oracle_output_case, k, nsteps, os.path.join(root, k)) for k in kinds}
        return {k: f.result() for k, f in futs.items()}


CONFIG1_FIELDS = ["e_den", "e_pre", "m_eng", "m_vof", "v_vel", "e_ste", "e_dam", "y_profile"]


def oracle_config_run(deck_fn: str, checkpoints: List[int], folder: str, deck_kwargs: Dict = None) -> Dict:
    """The reference's own initialisation and time loop on a named deck
    (decks.<deck_fn>(**deck_kwargs)), recording CONFIG1_FIELDS, dt and time at each checkpoint
    cycle."""
    d = getattr(bridge.decks, deck_fn)(**(deck_kwargs or {}))
    deck = bridge.decks.write_deck(d, folder)
    ref.init(deck, folder, os.path.join(folder, "run"))
    out = {"deck": deck, "folder": folder, "at": {}}
    done = 0
    for k in checkpoints:
        ref.step(k - done)
        done = k
        rec = {n: ref.get(n) for n in CONFIG1_FIELDS}
        rec["dt"] = ref.scalar("dt")
        rec["time"] = ref.scalar("time")
        out["at"][k] = rec
    return out


def oracle_noisy_deck_run(deck_kwargs: Dict, checkpoints: List[int], folder: str, seed: int,
                          fields: List[str]) -> Dict:
    """The reference's own initialisation of decks.config3_deck(**deck_kwargs), the seeded density
    noise of decks.density_noise applied to its state, then its own time loop, recording
    ``fields``, dt and time at each checkpoint cycle."""
    d = bridge.decks.config3_deck(**deck_kwargs)
    deck = bridge.decks.write_deck(d, folder)
    ref.init(deck, folder, os.path.join(folder, "run"))
    md, ed = bridge.decks.density_noise(ref.get("m_den"), ref.get("e_den"), seed=seed)
    ref.set("m_den", md)
    ref.set("e_den", ed)
    out = {"deck": deck, "folder": folder, "at": {}}
    done = 0
    for k in checkpoints:
        ref.step(k - done)
        done = k
        rec = {n: ref.get(n) for n in fields}
        rec["dt"] = ref.scalar("dt")
        rec["time"] = ref.scalar("time")
        out["at"][k] = rec
    return out


def oracle_noisy_deck_run_isolated(deck_kwargs: Dict, checkpoints: List[int], folder: str, seed: int,
                                   fields: List[str]) -> Dict:
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=1, mp_context=ctx) as ex:
        return ex.submit(oracle_noisy_deck_run, deck_kwargs, checkpoints, folder, seed, fields).result()


def oracle_config_run_isolated(deck_fn: str, checkpoints: List[int], folder: str, deck_kwargs: Dict = None) -> Dict:
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=1, mp_context=ctx) as ex:
        return ex.submit(oracle_config_run, deck_fn, checkpoints, folder, deck_kwargs).result()


def _interior_nonvacuum_cells(m_vof: np.ndarray) -> List:
    """Interior cells that are not pure vacuum, in the reference's traversal order of
    calculate_dt (src/sale2d.c:1965-1978: rows j outer, columns i inner)."""
    ny, nx = m_vof.shape[:2]
    return [(i, j) for j in range(2, ny - 2) for i in range(2, nx - 2) if not m_vof[j, i, 0] > 1.0 - 1e-6]


def oracle_nan_dt(kind: str, folder: str) -> Dict:
    """The reference's own CFL phase (calculate_dt and the MIN, phases 5-6) on a mid-cycle state
    of a small deck, with the sound speed of one cell set to NaN: the first, a middle and the
    last cell of its traversal, and no cell. Returns the state before phase 5 (to load into the
    GPU library) and the dt of each case."""
    deck, folder = bridge.write_small_deck(kind, folder)
    ref.init(deck, folder, os.path.join(folder, "run"))
    ref.step(3)
    ref.phases(0, 4)
    run = bridge.run_desc_from_oracle()
    out = {
        "run": {n: (list(getattr(run, n)) if n == "go" else getattr(run, n)) for n in RUN_FIELDS},
        "mats": bridge.materials_from_oracle(run.nmat),
        "init": {n: ref.get(n) for n in bridge.UPLOAD_FIELDS},
        "tracers0": ref.tracers(),
        "cells": {}, "dt": {},
    }
    order = _interior_nonvacuum_cells(out["init"]["m_vof"])
    dt_prev = ref.scalar("dt")
    csd = out["init"]["e_csd"]
    for case, cell in (("none", None), ("first", order[0]), ("middle", order[len(order) // 2]), ("last", order[-1])):
        c = csd.copy()
        if cell is not None:
            c[cell[1], cell[0], 0] = np.nan
        ref.set("e_csd", c)
        ref.set_scalar("dt", dt_prev)
        ref.phases(5, 6)
        out["cells"][case] = cell
        out["dt"][case] = ref.scalar("dt")
    return out


def oracle_nan_dt_isolated(kind: str, folder: str) -> Dict:
    ctx = mp.get_context("spawn")
    with cf.ProcessPoolExecutor(max_workers=1, mp_context=ctx) as ex:
        return ex.submit(oracle_nan_dt, kind, folder).result()
