"""Parity of the benchmarked workload: the 15 km/s ice-on-granite impact (tabulated SieDen
granite target, Tillotson ice projectile at CPPR 40, rock strength with Ivanov damage, gravity,
30-layer PML) that bench.py times at 2048 x 2048 cells, here on a 256 x 256 copy of the same
deck over 400 cycles.

The reference initialises and runs the deck with its own code (the oracle, compiled from its
sources); the library starts from the same .inp deck with its own initialiser. Tolerances,
stated here: relative L2 at most 1e-9 for every recorded field at every checkpoint, the
surface profile and the cell material flags exact, dt within 1e-12. The reference run itself,
with every material density moved by one ulp at the start, stays within 5e-12 of the
unperturbed run over these 400 cycles, so the bound leaves room only for ulp-level differences
of the math library, not for a wrong branch.
"""
import numpy as np
import pytest

import trajectory as tj
from salec_b200 import capi

CHECKPOINTS = [1, 25, 100, 200, 400]
TOL_L2 = 1e-9
TOL_DT = 1e-12


@pytest.mark.gpu
def test_config2_copy_matches_reference(cuda_device, oracle_lib, tmp_path):
    rec = tj.oracle_config_run_isolated("config2_deck", CHECKPOINTS, str(tmp_path), {"n": 256})
    sim = capi.Simulation.from_deck(rec["deck"], rec["folder"])
    done = 0
    worst = {}
    for k in CHECKPOINTS:
        sim.step(k - done)
        done = k
        want = rec["at"][k]
        assert abs(sim.scalar("dt") - want["dt"]) <= TOL_DT * want["dt"], k
        for n in tj.CONFIG1_FIELDS:
            err = tj.rel_l2(sim.get_field(n), want[n])
            worst[n] = max(worst.get(n, 0.0), err)
            assert err <= TOL_L2, "cycle %d %s: relative L2 %.3e" % (k, n, err)
        assert np.array_equal(sim.get_field("y_profile"), want["y_profile"]), k
        assert np.array_equal(sim.get_field("m_vof") > 1e-6, want["m_vof"] > 1e-6), k
    assert sim.check() == 0
    sim.close()
    print("config-2 copy, 256^2 x %d cycles: worst relative L2 %s" % (CHECKPOINTS[-1], worst))
