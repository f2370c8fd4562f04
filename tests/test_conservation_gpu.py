"""Compensated conservation sums (salec_gpu_conservation) against exactly rounded sums.

The device sums every product in FP64 with Neumaier's compensated summation; here the same
products are formed with numpy from the fields read back, and math.fsum (exactly rounded)
sums them. The two must agree to a few ulps (relative 1e-14), in both storage forms, on a
developed impact (20 cycles, so that velocities, vertex masses and mixed cells are present).
"""
import math

import numpy as np
import pytest

from salec_b200 import capi, decks

TOL = 1e-14


def exact_sums(sim):
    run = sim.get_run()
    nx, ny, nmat = run.nx, run.ny, run.nmat
    vof, den, eng = sim.get_field("m_vof"), sim.get_field("m_den"), sim.get_field("m_eng")
    vol = sim.get_field("e_vol")[2:ny + 2, 2:nx + 2, 0]
    out = {"mass_by_material": []}
    total, ie = [], []
    for m in range(1, nmat):
        vf = vof[2:ny + 2, 2:nx + 2, m] * vol
        mass = vf * den[2:ny + 2, 2:nx + 2, m]
        total.append(mass.ravel())
        ie.append((vf * eng[2:ny + 2, 2:nx + 2, m]).ravel())
        out["mass_by_material"].append(math.fsum(mass.ravel()))
    out["mass"] = math.fsum(np.concatenate(total))
    out["internal_energy"] = math.fsum(np.concatenate(ie))
    vel, vm = sim.get_field("v_vel"), sim.get_field("v_mass")
    mv = vm[1:ny + 4, 1:nx + 4, 0]
    vx, vy = vel[1:ny + 4, 1:nx + 4, 0], vel[1:ny + 4, 1:nx + 4, 1]
    out["momentum_r"] = math.fsum((mv * vx).ravel())
    out["momentum_z"] = math.fsum((mv * vy).ravel())
    out["kinetic_energy"] = math.fsum((0.5 * mv * (vx * vx + vy * vy)).ravel())
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [capi.PRECISION_FP64, capi.PRECISION_MIXED])
def test_conservation_sums_are_exactly_rounded(cuda_device, tmp_path, precision):
    d = decks.Deck(npx=96, npy=128, radius_cells=8, maxstep=40, damp_x=6, damp_y=6, velocity=-9000.0)
    deck = decks.write_deck(d, str(tmp_path))
    sim = capi.Simulation.from_deck(deck, str(tmp_path), precision=precision)
    sim.step(20)
    got = sim.conservation()
    want = exact_sums(sim)
    for k in ("mass", "momentum_r", "momentum_z", "internal_energy", "kinetic_energy"):
        scale = max(abs(want[k]), 1e-300)
        assert abs(got[k] - want[k]) <= TOL * scale, "%s: %r vs exactly rounded %r" % (k, got[k], want[k])
    for g, w in zip(got["mass_by_material"], want["mass_by_material"]):
        assert abs(g - w) <= TOL * abs(w)
    assert got["kinetic_energy"] > 0.0 and got["mass"] > 0.0
    sim.close()
