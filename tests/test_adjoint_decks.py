"""The adjoint's deck and target helpers (CPU): config5_deck writes the strength parameters
exactly (repr of the double), so that a finite-difference step of 1e-8 relative reaches the
solver, and target_profile is a seeded, deterministic bowl below the initial heights."""
import numpy as np

from salec_b200 import decks


def _deck_text(tmp_path, **kw):
    path = decks.write_deck(decks.config5_deck(**kw), str(tmp_path))
    with open(path) as fh:
        return fh.read()


def test_config5_deck_writes_parameters_exactly(tmp_path):
    c = 1.0e7 * (1.0 + 1e-8)
    f = 1.2 * (1.0 - 1e-8)
    text = _deck_text(tmp_path / "a", n=64, cohesion=c, friction=f, velocity=1000.0, cppr=6.0)
    assert repr(c) in text and repr(f) in text
    base = _deck_text(tmp_path / "b", n=64, velocity=1000.0, cppr=6.0)
    assert base != text


def test_target_profile_is_seeded_and_below_the_surface():
    h0 = np.full(256, 1.0e4)
    a = decks.target_profile(h0, 50.0)
    b = decks.target_profile(h0, 50.0)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, decks.target_profile(h0, 50.0, seed=6))
    bowl = h0 - a
    assert 199.0 <= bowl[0] <= 401.0            # the bowl's depth at the axis, plus roughness
    assert np.all(np.abs(bowl[-10:]) <= 1.0)    # far from the axis only the roughness remains
