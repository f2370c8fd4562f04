"""Adjoint of the mesh update against central finite differences (FP64, CUDA device).

Per phase (dot-product test): from a developed state of the adjoint's deck, the reverse of phase
p applied to random output adjoints ybar must satisfy <ybar, J dx_f> = <J^T ybar, dx_f> for a
random relative perturbation dx_f of each input field f in turn, with J dx_f from central
differences of the forward phase (relative step 1e-8). Tolerance: 1e-5 of the phase's largest
term (the central differences carry rounding of about 1e-16 / 1e-8 of each output).

Window: the adjoint of a checkpointed window against central differences (frozen time steps, as
the adjoint differentiates) of the surface-height misfit with respect to cohesion, friction and
the initial velocity scale (impactor speed), relative step 1e-6, and the initial density field
along a smooth random direction (cosine modes up to order 2), relative step 1e-8: the forward
model has thresholds (void vertices at TOLRHO, the viscosity cut at TOLQPRE) at which the misfit
jumps, and a density perturbation of 1e-6 already moves cells across them, while a per-cell
random direction crosses the viscosity kink of nearly uniformly moving cells at any step.
Tolerance: 1e-3 relative. The result must not depend on the checkpoint interval.
"""
import numpy as np
import pytest

from salec_b200 import capi, decks

# phase -> (input fields perturbed, output fields seeded)
PHASE_IO = {
    1: (["m_vof", "e_dvel", "e_den", "v_vel", "v_mass"], ["v_vof", "v_vel", "v_mass"]),
    3: (["v_vel", "v_mass"], ["e_vel"]),
    4: (["e_vel", "e_den"], ["v_vel"]),
    5: (["v_vel", "e_den", "e_csd"], ["e_grad_vel", "e_div_vel", "e_q"]),
    7: (["e_ste", "e_ste2s", "e_dam", "e_grad_vel", "e_mu", "e_pre", "e_tem", "m_vof"], ["e_ste", "e_ste2s", "e_dam"]),
    8: (["e_pre", "e_q", "e_ste", "e_den", "v_vel"], ["v_acc"]),
    9: (["v_vel", "v_acc"], ["v_dis", "v_vel"]),
    10: (["e_pre", "e_q", "e_div_vel", "e_grad_vel", "e_ste", "m_eng"], ["m_eng"]),
    12: (["v_dis", "m_vof", "v_vof", "m_den", "m_eng", "e_vel", "e_ste", "e_dam"], ["bx_phi", "by_phi"]),
    14: (["bx_phi", "by_phi", "m_vof", "m_den", "m_eng", "e_den", "e_ste", "e_dam"],
         ["m_vof", "m_den", "m_eng", "e_dvel", "e_ste", "e_dam", "e_den", "e_pre", "e_csd", "e_tem", "e_mu"]),
}
STATE = sorted({f for i, o in PHASE_IO.values() for f in i + o} | {"e_wpt", "v_acc", "v_dis"})
EPS_PHASE = 1e-8
TOL_PHASE = 1e-5
EPS_FD = 1e-6
EPS_FD_DENSITY = 1e-8
TOL_FD = 1e-3


def column_heights(sim):
    vof, pos = sim.get_field("m_vof"), sim.get_field("e_pos")
    return ((1.0 - vof[2:-2, 2:-2, 0]) * pos[2:-2, 2:-2, 3]).sum(axis=0)


def misfit(sim, target):
    r = column_heights(sim) - target
    return 0.5 * float(np.sum(r * r))


@pytest.fixture(scope="module")
def developed(tmp_path_factory):
    folder = str(tmp_path_factory.mktemp("adj"))
    # a 1 km/s impact: plastic flow and damage growth without vaporisation, so that few points sit
    # on a kink of the forward model (clamps, min/max switches), where central differences average
    # the two one-sided derivatives
    deck = decks.write_deck(decks.config5_deck(n=48, cppr=6.0, velocity=1000.0), folder)
    sim = capi.Simulation.from_deck(deck, folder)
    sim.step(12)
    state = {f: sim.get_field(f) for f in STATE}
    dt = sim.scalar("dt")
    return sim, state, dt


def _set(sim, state, dt, delta=None, eps=0.0):
    for f, a in state.items():
        sim.set_field(f, a + eps * delta[f] if delta is not None and f in delta else a)
    sim.set_scalar("dt", dt)


@pytest.mark.gpu
@pytest.mark.parametrize("phase", sorted(PHASE_IO))
def test_adjoint_phase_dot_product(cuda_device, developed, phase):
    """One input field at a time: <ybar, J_f dx_f> from central differences against <xbar_f, dx_f>."""
    sim, state, dt = developed
    ins, outs = PHASE_IO[phase]
    rng = np.random.default_rng(100 + phase)
    delta = {f: state[f] * rng.uniform(-1.0, 1.0, state[f].shape) for f in ins}
    if "v_mass" in delta:
        delta["v_mass"][..., 1] = 0.0   # the void-corner count is an integer, not differentiated
    ybar = {f: rng.uniform(-1.0, 1.0, state[f].shape) / max(float(np.sqrt(np.mean(state[f] ** 2))), 1e-30)
            for f in outs}
    if phase == 5:
        # the viscosity switches on where the velocity divergence turns negative; where the
        # divergence is smaller than the perturbation makes it (a body in nearly uniform motion)
        # the central differences straddle that kink and match neither one-sided derivative
        _set(sim, state, dt)
        sim.phases(5, 5)
        div = sim.get_field("e_div_vel")
        ybar["e_q"][np.abs(div) < 1e-6 * float(np.max(np.abs(div)))] = 0.0
    _set(sim, state, dt)
    sim.adjoint_reset()
    for f in outs:
        sim.adjoint_set(f, ybar[f])
    sim.adjoint_phase(phase)
    rhs = {f: float(np.sum(sim.adjoint_get(f) * delta[f])) for f in ins}
    lhs = {}
    for f in ins:
        res = {}
        for sgn in (1.0, -1.0):
            _set(sim, state, dt, {f: delta[f]}, sgn * EPS_PHASE)
            sim.phases(phase, phase)
            res[sgn] = {o: sim.get_field(o) for o in outs}
        lhs[f] = sum(float(np.sum(ybar[o] * (res[1.0][o] - res[-1.0][o]))) for o in outs) / (2.0 * EPS_PHASE)
    _set(sim, state, dt)
    scale = max(max(abs(v) for v in lhs.values()), max(abs(v) for v in rhs.values()), 1e-300)
    bad = {f: (lhs[f], rhs[f]) for f in ins if abs(lhs[f] - rhs[f]) > TOL_PHASE * scale}
    print("phase", phase, {f: "%.9e / %.9e" % (lhs[f], rhs[f]) for f in ins})
    assert not bad, "phase %d: finite differences vs adjoint per input field %s" % (phase, bad)


def _fd_run(deck_kw, folder, dts, target, init_edit=None):
    deck = decks.write_deck(decks.config5_deck(**deck_kw), folder)
    sim = capi.Simulation.from_deck(deck, folder)
    if init_edit:
        init_edit(sim)
    sim.set_dt_schedule(dts)
    sim.step(len(dts))
    J = misfit(sim, target)
    sim.close()
    return J


@pytest.mark.gpu
def test_adjoint_window_against_finite_differences(cuda_device, tmp_path):
    base = dict(n=64, cppr=6.0, cohesion=1.0e7, friction=1.2, velocity=1000.0)
    nsteps, every = 30, 10
    folder = str(tmp_path / "base")
    deck = decks.write_deck(decks.config5_deck(**base), folder)
    ref = capi.Simulation.from_deck(deck, folder)
    h0 = column_heights(ref)
    target = decks.target_profile(h0, 50.0)
    dts = []
    for _ in range(nsteps):
        ref.step(1)
        dts.append(ref.scalar("dt"))
    J_ref = misfit(ref, target)
    ref.close()
    sim = capi.Simulation.from_deck(deck, folder)
    v0 = sim.get_field("v_vel")
    md0, ed0 = sim.get_field("m_den"), sim.get_field("e_den")
    J, dp, dvs, gden = sim.adjoint_window(nsteps, every, target)
    assert abs(J - J_ref) <= 1e-12 * J_ref
    sim.close()
    # one cycle per segment replays nothing from undo logs: the same sensitivities up to the order
    # of the atomic sums
    sim = capi.Simulation.from_deck(deck, folder)
    J1, dp1, dvs1, gden1 = sim.adjoint_window(nsteps, 1, target)
    sim.close()
    assert J1 == J
    assert abs(dvs1 - dvs) <= 1e-9 * abs(dvs)
    assert np.allclose(dp1, dp, rtol=1e-9, atol=0.0)
    assert np.allclose(gden1, gden, rtol=1e-8, atol=1e-12 * float(np.max(np.abs(gden))))

    def fd(kw_plus, kw_minus, edit_plus=None, edit_minus=None):
        jp = _fd_run({**base, **kw_plus}, str(tmp_path / "p"), dts, target, edit_plus)
        jm = _fd_run({**base, **kw_minus}, str(tmp_path / "m"), dts, target, edit_minus)
        return jp - jm

    c = base["cohesion"]
    d_coh = fd({"cohesion": c * (1 + EPS_FD)}, {"cohesion": c * (1 - EPS_FD)}) / (2 * EPS_FD * c)
    f = base["friction"]
    d_fri = fd({"friction": f * (1 + EPS_FD)}, {"friction": f * (1 - EPS_FD)}) / (2 * EPS_FD * f)

    def scale_v(s):
        return lambda sim: sim.set_field("v_vel", v0 * s)

    d_vel = fd({}, {}, scale_v(1 + EPS_FD), scale_v(1 - EPS_FD)) / (2 * EPS_FD)
    rng = np.random.default_rng(11)
    ny, nx = ed0.shape[:2]
    yy, xx = np.meshgrid(np.linspace(0.0, 1.0, ny), np.linspace(0.0, 1.0, nx), indexing="ij")
    ds = np.zeros((ny, nx))
    for a in range(3):
        for b in range(3):
            ds += rng.uniform(-1.0, 1.0) * np.cos(np.pi * a * xx) * np.cos(np.pi * b * yy)
    ds /= np.abs(ds).max()

    def scale_rho(sg):
        def edit(sim):
            f_ = 1.0 + sg * EPS_FD_DENSITY * ds
            md = md0.copy()
            md[..., 1:] *= f_[..., None]
            sim.set_field("m_den", md)
            sim.set_field("e_den", ed0 * f_[..., None])
        return edit

    d_rho = fd({}, {}, scale_rho(1.0), scale_rho(-1.0)) / (2 * EPS_FD_DENSITY)
    adj = {"cohesion": dp[0] + dp[2], "friction": dp[1] + dp[3], "velocity": dvs,
           "density": float(np.sum(gden * ed0[..., 0] * ds))}
    fds = {"cohesion": d_coh, "friction": d_fri, "velocity": d_vel, "density": d_rho}
    print("adjoint", adj, "finite differences", fds)
    for k in adj:
        assert abs(adj[k] - fds[k]) <= TOL_FD * max(abs(fds[k]), 1e-300), (k, adj[k], fds[k])
