"""Mixed form (FP32 storage of the relaxed fields, FP64 arithmetic and FP64 conserved fields)
against the reference's FP64 run.

Tolerances, stated here: relative L2 error of density and pressure at most 1e-4 after every
cycle of a 40-cycle run on each feature deck, against the oracle (the reference compiled from
its own sources); on a 192x192 impact run for 300 cycles, the same bound against the plain FP64
form (which itself matches the reference to 1e-9), and the transient crater depth read from the
surface profile within 1 % of the FP64 form's.
"""
import numpy as np
import pytest

import trajectory as tj
from salec_b200 import capi, decks

KINDS = ["base", "pml2_acfl", "two_mat", "sieden_projectile", "sbc_tensile", "porous"]
NSTEPS = 40
TOL_DEN_PRE = 1e-4


@pytest.fixture(scope="module")
def records(tmp_path_factory):
    return tj.trajectories(KINDS, NSTEPS, str(tmp_path_factory.mktemp("mixed")))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_mixed_form_tracks_reference(cuda_device, records, kind):
    rec = records[kind]
    sim = tj.simulation_from_record(rec, precision=capi.PRECISION_MIXED)
    worst = {}
    for s, want in enumerate(rec["steps"], start=1):
        sim.step(1)
        for n in ("e_den", "e_pre", "m_eng", "m_vof", "v_vel"):
            worst[n] = max(worst.get(n, 0.0), tj.rel_l2(sim.get_field(n), want[n]))
        assert worst["e_den"] <= TOL_DEN_PRE and worst["e_pre"] <= TOL_DEN_PRE, (kind, s, worst)
    assert sim.check() == 0
    sim.close()
    print(kind, {k: "%.2e" % v for k, v in worst.items()})


def crater_depth(profile: np.ndarray, surface: float, ncols: int = 4) -> float:
    """Depth of the transient crater from the surface profile: the lowest surface height over
    the columns next to the symmetry axis, below the pre-impact surface."""
    return float(surface - np.min(profile[2:2 + ncols]))


@pytest.mark.gpu
def test_mixed_form_on_a_developed_impact(cuda_device, tmp_path):
    d = decks.Deck(npx=192, npy=192, radius_cells=12, maxstep=400, damp_x=16, damp_y=16, velocity=-8000.0)
    deck = decks.write_deck(d, str(tmp_path))
    ref = capi.Simulation.from_deck(deck, str(tmp_path))
    mix = capi.Simulation.from_deck(deck, str(tmp_path), precision=capi.PRECISION_MIXED)
    depth_ref, depth_mix = 0.0, 0.0
    for k in range(30):
        ref.step(10)
        mix.step(10)
        prof = ref.get_field("y_profile").reshape(-1)
        surface = float(np.median(prof[2:-2]))   # most columns are still at the pre-impact surface
        depth_ref = max(depth_ref, crater_depth(prof, surface))
        depth_mix = max(depth_mix, crater_depth(mix.get_field("y_profile").reshape(-1), surface))
    errs = {n: tj.rel_l2(mix.get_field(n), ref.get_field(n)) for n in ("e_den", "e_pre", "m_eng", "m_vof", "v_vel")}
    print("192x192, 300 cycles:", {k: "%.2e" % v for k, v in errs.items()}, "depth", depth_ref, depth_mix)
    assert errs["e_den"] <= TOL_DEN_PRE and errs["e_pre"] <= TOL_DEN_PRE, errs
    assert depth_ref > 0.0
    assert abs(depth_mix - depth_ref) <= 0.01 * depth_ref, (depth_mix, depth_ref)
    ref.close()
    mix.close()
