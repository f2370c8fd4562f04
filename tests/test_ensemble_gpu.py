"""Ensemble stepping (salec_gpu_step_many): several independent impacts of different mesh
sizes advanced together, their kernels interleaved on the device through one stream per
member. Every member must end bit for bit where the same deck stepped alone ends, and the
members' seeded decks follow the ensemble distribution."""
import numpy as np
import pytest

from salec_b200 import capi, decks, fields


def test_ensemble_decks_are_seeded_and_in_range():
    a = decks.ensemble_decks(16, seed=5)
    b = decks.ensemble_decks(16, seed=5)
    assert [(d.npx, d.npy, d.velocity) for d in a] == [(d.npx, d.npy, d.velocity) for d in b]
    for d in a:
        assert 128 <= d.npx <= 1024 and 128 <= d.npy <= 1024
        assert -20000.0 <= d.velocity <= -5000.0
        assert 1e6 <= d.materials[0].yint0 <= 1e8 and 0.6 <= d.materials[0].yintfri <= 1.4


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.PRECISION_FP64, capi.PRECISION_MIXED])
def test_ensemble_matches_members_stepped_alone(cuda_device, tmp_path, precision):
    shapes = [(24, 32, -6000.0), (40, 28, -9000.0), (32, 48, -12000.0)]
    paths = []
    for k, (nx, ny, v) in enumerate(shapes):
        d = decks.Deck(npx=nx, npy=ny, radius_cells=4, maxstep=40, damp_x=4, damp_y=4, velocity=v)
        folder = tmp_path / ("m%d" % k)
        paths.append((decks.write_deck(d, str(folder)), str(folder)))
    ens = [capi.Simulation.from_deck(p, f, precision=precision) for p, f in paths]
    capi.step_many(ens, 25, chunk=4)
    for s in ens:
        s.sync()
    for (p, f), s in zip(paths, ens):
        alone = capi.Simulation.from_deck(p, f, precision=precision)
        alone.step(25)
        for n in fields.STATE_FIELDS:
            assert np.array_equal(s.get_field(n), alone.get_field(n), equal_nan=True), n
        assert s.scalar("dt") == alone.scalar("dt") and s.scalar("time") == alone.scalar("time")
        alone.close()
        s.close()
