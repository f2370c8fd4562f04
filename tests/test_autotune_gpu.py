"""Block-shape autotuning (salec_gpu_autotune): it leaves the simulation exactly where it was,
and a run with the tuned shapes ends bit for bit where a run with the default shapes ends."""
import numpy as np
import pytest

from salec_b200 import capi, decks, fields


@pytest.mark.gpu
def test_autotune_keeps_state_and_results(cuda_device, tmp_path):
    deck = decks.write_deck(decks.Deck(npx=64, npy=80, radius_cells=6, damp_x=6, damp_y=6, velocity=-9000.0),
                            str(tmp_path))
    a = capi.Simulation.from_deck(deck, str(tmp_path))
    b = capi.Simulation.from_deck(deck, str(tmp_path))
    a.step(5)
    b.step(5)
    before = {n: a.get_field(n) for n in fields.STATE_FIELDS}
    t_before, dt_before = a.scalar("time"), a.scalar("dt")
    shapes = a.autotune(cycles=2)
    assert sorted(shapes) == [1, 3, 4, 5, 7, 8, 9, 10, 12, 14]
    for ph, (bx, by) in shapes.items():
        assert bx % 32 == 0 and bx * by <= 256, (ph, bx, by)
    for n in fields.STATE_FIELDS:
        assert np.array_equal(a.get_field(n), before[n], equal_nan=True), n
    assert a.scalar("time") == t_before and a.scalar("dt") == dt_before
    a.step(20)
    b.step(20)
    for n in fields.STATE_FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n), equal_nan=True), n
    assert np.array_equal(a.get_tracers(), b.get_tracers())
    a.close()
    b.close()
