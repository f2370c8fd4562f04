"""Golden vectors of the mesh update (tests/golden/tiny_impact.npz, made by make_golden.py from
the reference's own compiled time loop).

CPU: the oracle, re-run here from the same deck, reproduces the committed vectors bit for bit,
which pins the oracle to the reference run that made them.
GPU: the C ABI, loaded with the committed initial state, reproduces the committed steps 1, 2, 5
and 10 (relative L2 1e-9 per field, dt 1e-12, integer-valued flags exactly). This case needs
no reference tree and no oracle library at run time.
"""
import os
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

TOL_L2 = 1e-9
TOL_DT = 1e-12


@pytest.fixture(scope="module")
def golden():
    return make_golden.load()


def test_golden_file_is_well_formed(golden):
    rec, steps = golden
    assert sorted(steps) == list(make_golden.KEPT_STEPS)
    assert rec["run"]["nx"] == 12 and rec["run"]["ny"] == 16 and len(rec["mats"]) == rec["run"]["nmat"]
    for k, st in steps.items():
        assert st["dt"] > 0 and np.isfinite(st["dt"])
        for n, a in st.items():
            if isinstance(a, np.ndarray) and a.dtype.kind == "f":
                assert np.isfinite(a).all(), (k, n)
    times = [steps[k]["time"] for k in sorted(steps)]
    assert all(b > a for a, b in zip(times, times[1:]))


def test_oracle_reproduces_golden_vectors(oracle_lib, golden):
    import trajectory
    rec, steps = golden
    with tempfile.TemporaryDirectory() as tmp:
        now = trajectory.trajectories(["tiny"], max(steps), tmp)["tiny"]
    for n, a in rec["init"].items():
        assert np.array_equal(now["init"][n], a, equal_nan=True), "init " + n
    for k, want in steps.items():
        got = now["steps"][k - 1]
        for n, a in want.items():
            assert np.array_equal(np.asarray(got[n]), np.asarray(a), equal_nan=True), "step %d %s" % (k, n)


@pytest.mark.gpu
def test_gpu_reproduces_golden_vectors(cuda_device, golden):
    import trajectory
    rec, steps = golden
    sim = trajectory.simulation_from_record(rec)
    done = 0
    for k in sorted(steps):
        sim.step(k - done)
        done = k
        want = steps[k]
        assert abs(sim.scalar("dt") - want["dt"]) <= TOL_DT * want["dt"], "step %d dt" % k
        for n, a in want.items():
            if not isinstance(a, np.ndarray) or n == "tracers" or a.ndim < 3:
                continue
            err = trajectory.rel_l2(sim.get_field(n), a)
            assert err <= TOL_L2, "step %d %s: relative L2 %.3e" % (k, n, err)
        # integer-valued quantities: void-corner counts, cell material flags, tracer ids and cells
        assert np.array_equal(sim.get_field("v_mass")[..., 1], want["v_mass"][..., 1]), "step %d void corners" % k
        assert np.array_equal(sim.get_field("m_vof") > 1e-6, want["m_vof"] > 1e-6), "step %d material flags" % k
        tg, tr = sim.get_tracers(), want["tracers"]
        assert tg.shape == tr.shape, "step %d tracer count" % k
        assert np.array_equal(tg[:, 6:12], tr[:, 6:12]), "step %d tracer ids, tags, matid or cells" % k
        assert trajectory.rel_l2(tg[:, 0:4], tr[:, 0:4]) <= TOL_L2
        assert trajectory.rel_l2(tg[:, 4:6], tr[:, 4:6]) <= 1e-6   # peak P/T are float32 in the reference
    sim.close()
