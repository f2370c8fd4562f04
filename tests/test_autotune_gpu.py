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


@pytest.mark.gpu
def test_set_block_shapes_reuses_a_tuning(cuda_device, tmp_path):
    """Shapes tuned on one handle, set on another of the same deck, change no result; invalid
    triples are rejected as argument errors."""
    deck = decks.write_deck(decks.Deck(npx=48, npy=64, radius_cells=5, damp_x=5, damp_y=5, velocity=-9000.0),
                            str(tmp_path))
    a = capi.Simulation.from_deck(deck, str(tmp_path))
    b = capi.Simulation.from_deck(deck, str(tmp_path))
    shapes = a.autotune(cycles=1)
    odd = {ph: ((64, 4) if (bx, by) != (64, 4) else (32, 1)) for ph, (bx, by) in shapes.items()}
    b.set_block_shapes(odd)
    for bad in ({2: (32, 4)}, {7: (16, 2)}, {7: (32, 16)}, {7: (48, 1)}, {12: (32, 0)}):
        with pytest.raises(capi.SalecError) as e:
            b.set_block_shapes(bad)
        assert e.value.code == -1
    a.step(12)
    b.step(12)
    for n in fields.STATE_FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n), equal_nan=True), n
    b.set_block_shapes(shapes)
    a.step(5)
    b.step(5)
    for n in fields.STATE_FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n), equal_nan=True), n
    a.close()
    b.close()
