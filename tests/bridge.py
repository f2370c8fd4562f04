"""Test bridge: initialise a deck with the oracle (the reference compiled from its sources),
hand its initialised state to the GPU library through the C ABI, and compare the two.

This mirrors the reference-side integration a host driver performs: run-wide parameters
from sale2d_var / mesh2d_info / cycle_control, per-material state_reference values and EOS
tables, then every field's bytes as they lie in field_var.data.
"""
from __future__ import annotations

import os
import sys
from typing import Dict, List, Optional, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (ROOT, os.path.join(ROOT, "salec-2d-public_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import ref  # noqa: E402
from salec_b200 import capi, decks  # noqa: E402

# every field the GPU path holds, in upload order
UPLOAD_FIELDS = [
    "v_vel", "v_bf", "v_acc", "v_dis", "v_pos", "v_vof", "v_mass", "v_vol", "v_subvol", "v_laplace", "v_suf",
    "v_alpha", "e_vel", "e_div_vel", "e_grad_vel", "e_ste", "e_mu", "e_dvel", "e_pre", "e_tem", "e_den", "e_csd",
    "e_dam", "e_cvs", "m_vof", "m_den", "m_eng", "m_pty", "e_wpt", "e_pos", "e_vol", "e_grad", "e_q",
    "e_strength", "e_cnd", "e_tps", "e_ste2s", "e_sta2s", "e_alpha", "e_beta", "e_sigma", "e_dampref", "e_vib",
    "e_ejt", "bx_phi", "by_phi", "bx_normal", "by_normal", "y_profile",
]

# fields the step evolves (compared after every phase)
STATE_FIELDS = [
    "v_vel", "v_acc", "v_dis", "v_vof", "v_mass", "v_alpha", "e_vel", "e_div_vel", "e_grad_vel", "e_ste", "e_mu",
    "e_dvel", "e_pre", "e_tem", "e_den", "e_csd", "e_dam", "e_cvs", "m_vof", "m_den", "m_eng", "m_pty", "e_wpt",
    "e_q", "e_strength", "e_tps", "e_ste2s", "e_sta2s", "e_alpha", "e_beta", "e_vib", "e_ejt", "e_cnd", "y_profile",
]

DAMP_IDS = {0: "pml", 1: "pml2", 2: "pml3", 3: "sbc", 4: "ctlg", 5: "none"}


def run_desc_from_oracle() -> capi.RunDesc:
    s = ref.scalar
    r = capi.RunDesc()
    r.nx, r.ny, r.nmat = int(s("nx")), int(s("ny")), int(s("nmat"))
    r.damp_type = int(s("damp_type"))
    for k, side in enumerate(("go_left", "go_right", "go_bottom", "go_top")):
        r.go[k] = int(s(side))
    for name in ("partpres", "porosity_model", "acoustic_fluid", "tensile_failure", "tracer_lubrication",
                 "tracer_lub_gy0", "tracer_lub_gy1"):
        setattr(r, name, int(s(name)))
    for name in ("avis1", "avis2", "anc", "density_cutoff", "velocity_max", "velocity_min", "acceleration_min",
                 "alpha_damp_x", "alpha_damp_y", "damp_time", "threshold_z", "flow_resistance", "flow_friction",
                 "tracer_lub_y0", "tracer_lub_frac", "max_dt", "dt"):
        setattr(r, name, s(name))
    r.time = s("time")
    r.i_step = int(s("i_step"))
    return r


def materials_from_oracle(nmat: int) -> List[Dict]:
    mats: List[Dict] = [{}]
    for m in range(1, nmat):
        d: Dict = {}
        for name in capi.MAT_DOUBLES + capi.MAT_DOUBLES2:
            d[name] = ref.material(m, name)
        d["PolyLiq"] = int(ref.material(m, "PolyLiq"))
        d["PolySol"] = int(ref.material(m, "PolySol"))
        d["yfunc"] = capi.func_index(ref.material_str(m, "yfunc"))
        d["tfunc"] = capi.func_index(ref.material_str(m, "tfunc"))
        d["dsdf"] = capi.func_index(ref.material_str(m, "dSDf"))
        d["porfunc"] = capi.func_index(ref.material_str(m, "porosityfunc"))
        et = ref.eos_type(m)
        d["eos_type"] = et
        if et == capi.EOS_TILLOTSON:
            p, x, y = ref.tillotson(m)
            d["till"] = p
            d["cold_yeng"] = y
        else:
            xt, yd, data = ref.table(m)
            d["ntem"], d["nden"] = len(xt), len(yd)
            d["xtem"], d["yden"], d["data"] = xt, yd, data
        mats.append(d)
    return mats


def gpu_from_oracle() -> capi.Simulation:
    run = run_desc_from_oracle()
    sim = capi.Simulation(run, materials_from_oracle(run.nmat))
    for name in UPLOAD_FIELDS:
        sim.set_field(name, ref.get(name))
    sim.set_tracers(ref.tracers())
    return sim


def compare(a: np.ndarray, b: np.ndarray, floor: float) -> Tuple[float, Tuple]:
    """Largest |a-b| / max(|b|, floor) over the array (NaN counts as equal to NaN)."""
    both_nan = np.isnan(a) & np.isnan(b)
    d = np.abs(a - b)
    d[both_nan] = 0.0
    rel = d / np.maximum(np.abs(b), floor)
    rel[both_nan] = 0.0
    rel = np.where(np.isnan(rel), np.inf, rel)
    k = int(np.argmax(rel))
    return float(rel.flat[k]), np.unravel_index(k, rel.shape)


# absolute floors (SI units) under which differences are judged against the floor
FLOORS = {"v_vel": 1e-6, "v_acc": 1e-4, "v_dis": 1e-9, "e_vel": 1e-6, "e_dvel": 1e-6, "e_pre": 1.0, "e_ste": 1.0,
          "e_q": 1.0, "e_strength": 1.0, "e_ste2s": 1.0, "m_eng": 1.0, "e_alpha": 1e-9, "v_alpha": 1e-6,
          "e_grad_vel": 1e-9, "e_div_vel": 1e-9, "e_sta2s": 1e-9, "e_tem": 1e-6, "e_mu": 1.0, "v_mass": 1e-6}


def compare_state(sim: capi.Simulation, names=STATE_FIELDS) -> Dict[str, Tuple[float, Tuple]]:
    out = {}
    for n in names:
        out[n] = compare(sim.get_field(n), ref.get(n), FLOORS.get(n, 1e-12))
    return out


def small_deck(kind: str = "base") -> decks.Deck:
    """Small decks covering the reference's branches (CPU oracle init in ~20 s each)."""
    if kind == "base":
        return decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4)
    if kind == "tiny":
        return decks.Deck(npx=12, npy=16, radius_cells=3, maxstep=40, damp_x=3, damp_y=3)
    if kind == "pml2_acfl":
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damping="pml2", damp_x=4, damp_y=4)
        d.materials = [decks.Material("basalt_", toff=16.0, block_size=200.0)]
        return d
    if kind == "two_mat":
        d = decks.Deck(npx=28, npy=36, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, projectile="dunite_",
                       velocity=-8000.0)
        d.materials = [decks.Material("basalt_"), decks.Material("dunite_")]
        return d
    if kind == "sieden_projectile":
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, projectile="granit_",
                       velocity=-9000.0)
        d.materials = [decks.Material("basalt_"), decks.Material("granit_", eos="aneos.sd")]
        return d
    if kind == "sbc_tensile":
        return decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damping="sbc", damp_x=4, damp_y=4,
                          lambda_x=0.3, lambda_y=0.3, tensile_failure=1, right="outflow", bottom="freeslip")
    if kind == "pml3":
        return decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damping="pml3", damp_x=4, damp_y=4)
    if kind == "lubrication":
        return decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, velocity=-9000.0,
                          extra={"tracer": {"lubrication": "3", "lub_y0": "0.0", "lub_frac": "0.5"}})
    if kind == "porous":
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, damping="pml2")
        d.materials = [decks.Material("basalt_", porosity="Wunnemann", alpha0=1.0 / 0.75, alphax=1.1,
                                      epse0=-1.0e-5, kappa=0.98, chi=0.5)]
        return d
    if kind == "ejecta_drag":
        # ejecta_flow (src/ejecta.c:65-133) with both the drag and the friction branch on
        # (the threshold at half the projectile radius marks the projectile's upper cells as ejecta)
        return decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, velocity=-8000.0,
                          ejecta_threshold=0.5, ejecta_resistance=40.0, ejecta_friction=0.5)
    if kind == "aneos_td":
        # target on a tabulated temperature-density EOS (eos_type ANEOS, src/eos/eos_state.c:793-841)
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, projectile="dunite_",
                       velocity=-8000.0)
        d.materials = [decks.Material("basalt_", eos="aneos.td"), decks.Material("dunite_")]
        return d
    if kind == "jc_vm":
        # JohnsonCook1 with Collins damage, and VonMises1 (src/strength.c:470-570)
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, projectile="dunite_",
                       velocity=-7000.0)
        d.materials = [decks.Material("basalt_", yshear="JohnsonCook1", damage="Collins",
                                      jc={"JcA": 2.0e8, "JcB": 4.0e8, "JcTref": 250.0}),
                       decks.Material("dunite_", yshear="VonMises1", yint0=5.0e8, ydam0=1.0e8)]
        return d
    if kind == "jc2_vm2":
        # JohnsonCook2 (thermal softening through the Simon melt curve) and VonMises2 with Collins
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, projectile="dunite_",
                       velocity=-9000.0)
        d.materials = [decks.Material("basalt_", yshear="JohnsonCook2",
                                      jc={"JcA": 2.0e8, "JcB": 4.0e8, "JcTref": 250.0, "JcC": 0.05}),
                       decks.Material("dunite_", yshear="VonMises2", damage="Collins", yint0=5.0e8, ydam0=1.0e8)]
        return d
    if kind == "ice":
        # IceStrength (piecewise ice melting curve, src/strength.c:725-754); the 100 K melting shift
        # keeps the ice below its softened melting point, so the strength is not zero
        d = decks.Deck(npx=24, npy=32, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, projectile="ice____",
                       velocity=-6000.0)
        d.materials = [decks.Material("ice____", poisson=0.33, yshear="IceStrength", yint0=1.0e6, yintfri=0.8,
                                      yintlim=1.0e9, ydam0=1.0e4, ydamfri=0.6, ydamlim=1.0e9, simon_t0=273.0,
                                      tdelta=100.0)]
        d.target_materials = ["ice____"]
        return d
    raise KeyError(kind)


def write_small_deck(kind: str, root: str) -> Tuple[str, str]:
    folder = os.path.join(root, kind)
    deck = decks.write_deck(small_deck(kind), folder)
    return deck, folder
