"""Host helpers of bench.py (CPU): the crater measure on a synthetic bowl-shaped density field,
and the conservation report's relative changes."""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_crater_metrics_on_a_bowl():
    bench = _bench()
    nx, ny, dx = 64, 48, 10.0
    # reference layout: (rows y, columns x, components), two pad cells on each side
    e_pos = np.zeros((ny + 4, nx + 4, 4))
    xs = (np.arange(nx + 4) - 2 + 0.5) * dx
    ys = (np.arange(ny + 4) - 2 + 0.5) * dx
    e_pos[..., 0] = xs[None, :]
    e_pos[..., 1] = ys[:, None]
    surface = 300.0                                 # pre-impact surface height
    depth, radius = 120.0, 200.0                    # a parabolic bowl on the axis
    top = surface - depth * np.clip(1.0 - (xs / radius) ** 2, 0.0, None)
    e_den = np.where(ys[:, None] < top[None, :], 2700.0, 0.0)[..., None]
    m = bench.crater_metrics(e_den, e_pos, 1350.0, surface, dx)
    # cell-centre sampling: the top is known to within a cell
    assert abs(m["depth_m"] - depth) <= dx, m
    assert abs(m["radius_m"] - radius) <= dx, m


def test_conservation_report():
    bench = _bench()
    a = {"mass": 2.0, "momentum_r": 0.0, "momentum_z": -4.0, "internal_energy": 1.0, "kinetic_energy": 3.0,
         "mass_by_material": [0.0, 2.0]}
    b = dict(a, mass=2.0 * (1 - 1e-8), momentum_z=-3.0, internal_energy=2.5, kinetic_energy=1.0)
    r = bench.conservation_report([{"conservation": a}, {"depth_m": 1.0, "conservation": b}])
    assert abs(r["rel_change"]["mass"] + 1e-8) < 1e-15
    assert abs(r["rel_change"]["total_energy"] - (-0.125)) < 1e-15
    assert abs(r["rel_change"]["momentum_z"] - 0.25) < 1e-15
