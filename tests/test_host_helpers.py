"""Host-side helpers of the benchmark and the decks (CPU): the crater-depth measure, the seeded
density noise of the layered target and the layered deck itself."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from salec_b200 import decks  # noqa: E402


def _column_mesh(ny=24, nx=12):
    y = (np.arange(ny) - 14.0)[:, None] * np.ones((1, nx))
    e_pos = np.zeros((ny, nx, 4))
    e_pos[..., 1] = y
    return y, e_pos


def test_crater_depth_interpolates_the_dense_top():
    y, e_pos = _column_mesh()
    den = np.where(y <= 0.0, 2680.0, 0.0)[..., None]
    rho = 0.5 * float(np.median(den[den > 0]))
    surface = float(np.nanmedian(bench.dense_top(den, e_pos, rho)))
    assert surface == 0.5                         # halfway between the top dense cell and vacuum
    assert bench.crater_depth(den, e_pos, rho, surface) == 0.0
    cav = den.copy()
    cav[y[:, 2] > -5.0, 2, 0] = 30.0              # a low-density plume above y = -5 on the axis
    d = bench.crater_depth(cav, e_pos, rho, surface)
    assert abs(d - (0.5 - (-5.0 + (2680.0 - rho) / (2680.0 - 30.0)))) < 1e-12
    empty = den.copy()
    empty[:, 2, 0] = 0.0                          # no dense cell on the axis: no depth
    assert np.isnan(bench.crater_depth(empty, e_pos, rho, surface))


def test_density_noise_is_seeded_and_bounded():
    rng = np.random.default_rng(0)
    m_den = rng.uniform(1000.0, 3000.0, (20, 30, 4))
    e_den = rng.uniform(1000.0, 3000.0, (20, 30, 1))
    a1, b1 = decks.density_noise(m_den, e_den, seed=3)
    a2, b2 = decks.density_noise(m_den, e_den, seed=3)
    a3, _ = decks.density_noise(m_den, e_den, seed=4)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    assert not np.array_equal(a1, a3)
    assert np.array_equal(a1[..., 0], m_den[..., 0])            # vacuum density untouched
    f = b1[..., 0] / e_den[..., 0]
    assert f.min() >= 0.99 and f.max() <= 1.01
    for m in range(1, 4):                                       # one factor per cell
        assert np.allclose(a1[..., m] / m_den[..., m], f, rtol=0, atol=1e-14)


def test_layered_deck(tmp_path):
    d = decks.config3_deck(n=64, regolith=150.0, basalt=400.0, cppr=4.0, side_layers=6, base_layers=4)
    path = decks.write_deck(d, str(tmp_path))
    text = open(path).read()
    assert "material = [regolit, basalt_, dunite_]" in text
    assert "depth = [150, 400, 1e+07]" in text
    assert "Porosity = [, Wunnemann, None, None]" in text
    assert "DampX = 6" in text and "DampY = 4" in text
    assert "nm = 4" in text
    for name in ("regolit", "basalt_", "dunite_"):
        assert os.path.exists(os.path.join(str(tmp_path), name + ".tillotson"))
