"""Failure detection without a GPU fault (the reference calls exit(0) on these, which reports
success; the library returns an error code and a message instead).

CPU: a missing deck, a deck naming an EOS file that does not exist, an unknown EOS type, and
out-of-range run descriptions are rejected before any device work.
GPU: a non-finite value seeded into the state is counted by salec_gpu_check, and two runs of
the same deck end bit for bit in the same state (the device reductions are exact and ordered:
atomic MIN of ordered bits and atomic additions of small integers).
"""
import ctypes
import os

import numpy as np
import pytest

from salec_b200 import capi, decks, fields


def _from_deck(deck, folder):
    h = ctypes.c_void_p()
    rc = capi.lib().salec_gpu_create_from_deck(deck.encode(), folder.encode(), ctypes.byref(h))
    return rc, capi.lib().salec_gpu_last_error().decode()


def test_missing_deck_is_an_argument_error(tmp_path):
    rc, msg = _from_deck(str(tmp_path / "no_such.inp"), str(tmp_path))
    assert rc == -1 and "cannot open" in msg


def test_missing_eos_file_is_an_argument_error(tmp_path):
    deck = decks.write_deck(decks.Deck(npx=16, npy=16, radius_cells=3, damp_x=3, damp_y=3), str(tmp_path))
    for f in os.listdir(str(tmp_path)):
        if f.endswith(".tillotson"):
            os.unlink(os.path.join(str(tmp_path), f))
    rc, msg = _from_deck(deck, str(tmp_path))
    assert rc == -1 and "cannot open" in msg


def test_unknown_eos_type_is_an_argument_error(tmp_path):
    deck = decks.write_deck(decks.Deck(npx=16, npy=16, radius_cells=3, damp_x=3, damp_y=3), str(tmp_path))
    text = open(deck).read().replace("postfix = [null, tillotson]", "postfix = [null, unobtainium]")
    open(deck, "w").write(text)
    rc, msg = _from_deck(deck, str(tmp_path))
    assert rc == -1 and "unknown EOS type" in msg


@pytest.mark.parametrize("field, value", [("nx", 2), ("nmat", 1), ("nmat", 11), ("damp_type", 9), ("precision", 7)])
def test_bad_run_descriptions_are_rejected(field, value):
    run = capi.RunDesc()
    run.nx, run.ny, run.nmat = 16, 16, 2
    setattr(run, field, value)
    mats = (capi.MaterialDesc * 12)()
    h = ctypes.c_void_p()
    assert capi.lib().salec_gpu_create(ctypes.byref(run), mats, ctypes.byref(h)) == -1
    assert not h.value


@pytest.mark.gpu
def test_nonfinite_values_are_counted(cuda_device, tmp_path):
    deck = decks.write_deck(decks.Deck(npx=24, npy=32, radius_cells=4, damp_x=4, damp_y=4), str(tmp_path))
    sim = capi.Simulation.from_deck(deck, str(tmp_path))
    sim.step(2)
    assert sim.check() == 0
    den = sim.get_field("m_den")
    den[10, 10, 1] = np.nan
    den[12, 11, 1] = np.inf
    sim.set_field("m_den", den)
    assert sim.check() == 2
    sim.close()


@pytest.mark.gpu
def test_two_runs_are_bitwise_identical(cuda_device, tmp_path):
    deck = decks.write_deck(decks.Deck(npx=40, npy=48, radius_cells=5, damp_x=5, damp_y=5, velocity=-12000.0),
                            str(tmp_path))
    a = capi.Simulation.from_deck(deck, str(tmp_path))
    b = capi.Simulation.from_deck(deck, str(tmp_path))
    a.step(30)
    b.step(30)
    for n in fields.STATE_FIELDS:
        assert np.array_equal(a.get_field(n), b.get_field(n), equal_nan=True), n
    assert np.array_equal(a.get_tracers(), b.get_tracers())
    a.close()
    b.close()
