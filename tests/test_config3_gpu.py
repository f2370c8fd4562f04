"""The layered three-material target: porous regolith (Wunnemann compaction, 25% porosity) over
basalt over a dunite half-space, basalt projectile at 10 km/s, separate side and base PML layer
counts, seeded +-1% cell-by-cell density noise on the initial state.

1. Parity on a small copy (48 x 48 cells, the same layers and materials thinner): the reference
   initialises and runs the deck with its own code, the library from the same .inp deck with
   its own initialiser; both get the same seeded density noise. Tolerances, stated here:
   relative L2 at most 1e-9 for every recorded field at cycles 40 and 150, dt within 1e-12, the
   surface profile and the cell material flags exact.
2. The full 4096 x 4096 deck: the mixed form against the plain FP64 form after 100 cycles,
   relative L2 at most 1e-4 in density and pressure (measured: 1.4e-7 and 2.6e-5), no
   non-finite value in either.
"""
import numpy as np
import pytest

import trajectory as tj
from salec_b200 import capi, decks

SMALL = dict(n=48, maxstep=999, regolith=150.0, basalt=400.0, cppr=4.0, side_layers=6, base_layers=4)
FIELDS = ["e_den", "e_pre", "m_eng", "m_den", "m_vof", "m_pty", "v_vel", "e_ste", "e_dam", "y_profile"]
CHECKPOINTS = [40, 150]
TOL_L2 = 1e-9
TOL_DT = 1e-12
SEED = 3


def _noisy(sim, seed):
    md, ed = decks.density_noise(sim.get_field("m_den"), sim.get_field("e_den"), seed=seed)
    sim.set_field("m_den", md)
    sim.set_field("e_den", ed)


@pytest.mark.gpu
def test_layered_small_copy_matches_reference(cuda_device, oracle_lib, tmp_path):
    rec = tj.oracle_noisy_deck_run_isolated(SMALL, CHECKPOINTS, str(tmp_path), SEED, FIELDS)
    sim = capi.Simulation.from_deck(rec["deck"], rec["folder"])
    assert sim.get_run().nmat == 4 and sim.get_run().porosity_model
    _noisy(sim, SEED)
    done = 0
    for k in CHECKPOINTS:
        sim.step(k - done)
        done = k
        want = rec["at"][k]
        assert abs(sim.scalar("dt") - want["dt"]) <= TOL_DT * want["dt"], k
        for n in FIELDS:
            err = tj.rel_l2(sim.get_field(n), want[n])
            assert err <= TOL_L2, "cycle %d %s: relative L2 %.3e" % (k, n, err)
        assert np.array_equal(sim.get_field("y_profile"), want["y_profile"])
        assert np.array_equal(sim.get_field("m_vof") > 1e-6, want["m_vof"] > 1e-6)
    assert sim.check() == 0
    sim.close()


@pytest.mark.gpu
def test_layered_full_size_mixed_against_fp64(cuda_device, tmp_path):
    deck = decks.write_deck(decks.config3_deck(n=4096), str(tmp_path))
    sims = {}
    for form, prec in (("fp64", capi.PRECISION_FP64), ("mixed", capi.PRECISION_MIXED)):
        s = capi.Simulation.from_deck(deck, str(tmp_path), precision=prec)
        _noisy(s, SEED)
        s.step(100)
        sims[form] = s
    for n in ("e_den", "e_pre"):
        err = tj.rel_l2(sims["mixed"].get_field(n), sims["fp64"].get_field(n))
        assert err <= 1e-4, "%s: mixed vs FP64 relative L2 %.3e" % (n, err)
    for s in sims.values():
        assert s.check() == 0
        s.close()
