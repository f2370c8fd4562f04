"""Field uploads of large host arrays (tens of MiB, pageable and pinned): the set_field /
get_field round trip through the staging buffer and the layout conversion must be exact."""
import numpy as np
import pytest
import torch

from salec_b200 import capi, decks


@pytest.mark.gpu
def test_large_pageable_upload_round_trip(cuda_device, tmp_path):
    deck = decks.write_deck(decks.Deck(npx=1100, npy=1000, radius_cells=20, damp_x=10, damp_y=10), str(tmp_path))
    sim = capi.Simulation.from_deck(deck, str(tmp_path))
    rng = np.random.default_rng(5)
    for name in ("e_ste", "m_den", "v_vel", "e_pre"):
        shape = sim.shape(name)
        b = rng.standard_normal(shape)           # pageable numpy memory
        sim.set_field(name, b)
        assert np.array_equal(sim.get_field(name), b), name
    # the same from pinned host memory
    shape = sim.shape("e_ste")
    pinned = torch.empty(int(np.prod(shape)), dtype=torch.float64, pin_memory=True).numpy().reshape(shape)
    pinned[...] = rng.standard_normal(shape)
    sim.set_field("e_ste", pinned)
    assert np.array_equal(sim.get_field("e_ste"), pinned)
    sim.close()
