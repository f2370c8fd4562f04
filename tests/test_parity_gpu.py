"""FP64 parity of the GPU mesh update with the reference's own FP64 run (CUDA device).

Each small deck exercises a group of the reference's branches; the oracle (the reference
compiled from its sources) and the GPU library start from the same initialised state and
are stepped side by side.

Tolerance: CUDA's exp/pow/log/tanh differ from glibc's by an ulp now and then, so the FP64
states drift apart at the 1e-16..1e-13 level; per field the relative L2 difference must
stay below 1e-9 over 40 steps, dt must agree to 1e-12, and the integer-valued quantities
(void-corner counts, which materials occupy each cell, tracer count, cell index and
ejecta sign) must be identical.
"""
import numpy as np
import pytest

import bridge
import trajectory as tj

KINDS = ["base", "pml2_acfl", "two_mat", "sieden_projectile", "sbc_tensile", "porous", "pml3", "lubrication",
         "ejecta_drag", "aneos_td", "jc_vm", "jc2_vm2", "ice"]
NSTEPS = 40
TOL_L2 = 1e-9
TOL_DT = 1e-12
TOLVOF = 1e-6


@pytest.fixture(scope="module")
def records(tmp_path_factory, oracle_lib):
    root = str(tmp_path_factory.mktemp("decks"))
    recs = tj.trajectories(KINDS, NSTEPS, root, phase_steps=2)
    return recs


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_step_parity(records, cuda_device, kind):
    rec = records[kind]
    sim = tj.simulation_from_record(rec)
    # the first two steps were recorded phase by phase; replay them the same way
    k = 0
    for s in range(2):
        for p in range(16):
            sim.phases(p, p)
            want = rec["phases"][k]
            k += 1
            if p == 1:
                continue   # the reference runs half of the vertex-momentum sweep inside phase 1
            for n in bridge.STATE_FIELDS:
                err = tj.rel_l2(sim.get_field(n), want[n])
                assert err <= TOL_L2, "%s step %d phase %d field %s rel-L2 %.3e" % (kind, s, p, n, err)
    worst = {}
    for s, want in enumerate(rec["steps"], start=2):
        sim.step(1)
        dt = sim.scalar("dt")
        assert abs(dt - want["dt"]) <= TOL_DT * want["dt"], "%s step %d dt %r vs %r" % (kind, s, dt, want["dt"])
        got = {n: sim.get_field(n) for n in bridge.STATE_FIELDS}
        for n in bridge.STATE_FIELDS:
            err = tj.rel_l2(got[n], want[n])
            worst[n] = max(worst.get(n, 0.0), err)
            assert err <= TOL_L2, "%s step %d field %s rel-L2 %.3e" % (kind, s, n, err)
        # integer-valued quantities are bit-exact
        assert np.array_equal(got["v_mass"][..., 1], want["v_mass"][..., 1]), "void-corner counts differ"
        assert np.array_equal(got["m_vof"] > TOLVOF, want["m_vof"] > TOLVOF), "cell material flags differ"
        tg, tr = sim.get_tracers(), want["tracers"]
        assert tg.shape == tr.shape, "tracer count %d vs %d" % (len(tg), len(tr))
        assert np.array_equal(tg[:, 6:12], tr[:, 6:12]), "tracer ids, tags, matid or cells differ"
        assert tj.rel_l2(tg[:, 0:4], tr[:, 0:4]) <= TOL_L2
        assert tj.rel_l2(tg[:, 4:6], tr[:, 4:6]) <= 1e-6   # peak P/T are float32 in the reference
    assert sim.check() == 0
    sim.close()


INIT_KINDS = ["base", "two_mat", "sieden_projectile", "porous", "sbc_tensile", "pml3", "lubrication",
              "ejecta_drag", "aneos_td", "jc_vm", "jc2_vm2", "ice"]
# fields computed by the host initialiser with the reference's own arithmetic: bit-exact
INIT_EXACT = ["v_pos", "e_pos", "e_vol", "e_grad", "v_vol", "v_subvol", "v_suf", "e_sigma", "bx_normal",
              "by_normal", "v_bf", "m_vof", "m_pty", "e_wpt", "e_tem", "e_dam"]


@pytest.mark.gpu
@pytest.mark.parametrize("kind", INIT_KINDS)
def test_deck_initialiser_matches_reference_init(records, cuda_device, tmp_path, kind):
    """salec_gpu_create_from_deck (no reference code) against the reference's start-up."""
    from salec_b200 import capi
    rec = records[kind]
    deck, folder = bridge.write_small_deck(kind, str(tmp_path))
    sim = capi.Simulation.from_deck(deck, folder)
    run = sim.get_run()
    for name, v in rec["run"].items():
        if name == "go":
            assert list(run.go) == list(v)
        elif name not in ("dt", "time", "i_step"):
            assert getattr(run, name) == pytest.approx(v, rel=1e-12, abs=0.0), name
    for name in bridge.UPLOAD_FIELDS:
        got, want = sim.get_field(name), rec["init"][name]
        if name in INIT_EXACT:
            assert np.array_equal(got, want), "%s differs from the reference init" % name
        elif name == "v_laplace":
            # only evaluated inside the ANC taper band; zero (possibly -0.0) elsewhere in the reference
            assert np.array_equal(got == 0, want == 0) and tj.rel_l2(got, want) == 0.0, name
        else:
            assert tj.rel_l2(got, want) <= 1e-12, "%s rel-L2 %.3e" % (name, tj.rel_l2(got, want))
    tg, tr = sim.get_tracers(), rec["tracers0"]
    assert np.array_equal(tg[:, 6:12], tr[:, 6:12])
    assert tj.rel_l2(tg[:, :4], tr[:, :4]) <= 1e-12
    # the deck-initialised run then tracks the reference's own run
    # rec["steps"][0] is the state after three steps (two were recorded phase by phase)
    for s, want in enumerate(rec["steps"][:10], start=2):
        sim.step(3 if s == 2 else 1)
        for n in bridge.STATE_FIELDS:
            err = tj.rel_l2(sim.get_field(n), want[n])
            assert err <= TOL_L2, "%s step %d field %s rel-L2 %.3e" % (kind, s, n, err)
    sim.close()


@pytest.mark.gpu
def test_ejecta_drag_branch_is_exercised(records, cuda_device):
    """The ejecta deck's parity run only proves ejecta_flow if the drag and friction change the
    result: the same start with both switched off must end elsewhere."""
    rec = records["ejecta_drag"]
    assert rec["run"]["flow_resistance"] > 0.0 and rec["run"]["flow_friction"] > 0.0
    off = dict(rec)
    off["run"] = dict(rec["run"], flow_resistance=-1.0, flow_friction=0.0)
    a, b = tj.simulation_from_record(rec), tj.simulation_from_record(off)
    a.step(10)
    b.step(10)
    assert tj.rel_l2(a.get_field("e_dvel"), b.get_field("e_dvel")) > 1e-6
    a.close()
    b.close()
