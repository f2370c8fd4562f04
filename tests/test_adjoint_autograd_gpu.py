"""The adjoint window as a torch.autograd.Function (test-side only; the product is the C ABI).

Inputs x (float64, 4): relative changes of cohesion and friction, of the initial velocity scale
(impactor speed) and the amplitude of a smooth relative density perturbation. The forward runs
salec_gpu_adjoint_window on a fresh simulation of the perturbed deck at the base run's time
steps (salec_gpu_set_dt_schedule) and returns the misfit; backward returns the gradients the
same call computed. torch.autograd.gradcheck compares them with its own central differences:
step 1e-6 for the first three inputs and 1e-8 for the density amplitude (the misfit has
threshold jumps that a larger density step reaches), relative tolerance 1e-3.
"""
import numpy as np
import pytest

from salec_b200 import capi, decks

torch = pytest.importorskip("torch")

BASE = dict(n=64, cppr=6.0, cohesion=1.0e7, friction=1.2, velocity=1000.0)
NSTEPS, EVERY = 30, 10


def column_heights(sim):
    vof, pos = sim.get_field("m_vof"), sim.get_field("e_pos")
    return ((1.0 - vof[2:-2, 2:-2, 0]) * pos[2:-2, 2:-2, 3]).sum(axis=0)


class Problem:
    def __init__(self, folder):
        self.folder = folder
        deck = decks.write_deck(decks.config5_deck(**BASE), folder)
        sim = capi.Simulation.from_deck(deck, folder)
        self.target = decks.target_profile(column_heights(sim), 50.0)
        self.v0, self.md0, self.ed0 = sim.get_field("v_vel"), sim.get_field("m_den"), sim.get_field("e_den")
        self.dts = []
        for _ in range(NSTEPS):
            sim.step(1)
            self.dts.append(sim.scalar("dt"))
        sim.close()
        rng = np.random.default_rng(11)
        ny, nx = self.ed0.shape[:2]
        yy, xx = np.meshgrid(np.linspace(0.0, 1.0, ny), np.linspace(0.0, 1.0, nx), indexing="ij")
        ds = np.zeros((ny, nx))
        for a in range(3):
            for b in range(3):
                ds += rng.uniform(-1.0, 1.0) * np.cos(np.pi * a * xx) * np.cos(np.pi * b * yy)
        self.ds = ds / np.abs(ds).max()

    def misfit_and_grad(self, x):
        kw = dict(BASE, cohesion=BASE["cohesion"] * (1.0 + x[0]), friction=BASE["friction"] * (1.0 + x[1]))
        folder = self.folder + "/eval"
        deck = decks.write_deck(decks.config5_deck(**kw), folder)
        sim = capi.Simulation.from_deck(deck, folder)
        sim.set_field("v_vel", self.v0 * (1.0 + x[2]))
        f = 1.0 + x[3] * self.ds
        md = self.md0.copy()
        md[..., 1] *= f
        sim.set_field("m_den", md)
        sim.set_field("e_den", self.ed0 * f[..., None])
        sim.set_dt_schedule(self.dts)
        J, dp, dvs, _ = sim.adjoint_window(NSTEPS, EVERY, self.target, density=False)
        bm, be = sim.adjoint_get("m_den"), sim.adjoint_get("e_den")
        sim.close()
        g = np.array([
            (dp[0] + dp[2]) * BASE["cohesion"],            # Yint0 = Ydam0 = cohesion
            (dp[1] + dp[3]) * BASE["friction"],            # Yfricint = Yfricdam = friction
            dvs / (1.0 + x[2]),                            # sum vbar . v0
            float(np.sum((bm[..., 1] * self.md0[..., 1] + be[..., 0] * self.ed0[..., 0]) * self.ds)),
        ])
        return J, g


class Window(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, problem):
        J, g = problem.misfit_and_grad(x.detach().cpu().numpy())
        ctx.save_for_backward(torch.tensor(g, dtype=torch.float64))
        return torch.tensor(J, dtype=torch.float64)

    @staticmethod
    def backward(ctx, gout):
        (g,) = ctx.saved_tensors
        return gout * g, None


@pytest.mark.gpu
def test_adjoint_window_as_autograd_function(cuda_device, tmp_path):
    problem = Problem(str(tmp_path))
    x = torch.zeros(4, dtype=torch.float64, requires_grad=True)
    J = Window.apply(x, problem)
    (2.0 * J).backward()                            # the chain rule through torch
    _, g = problem.misfit_and_grad(np.zeros(4))
    assert torch.allclose(x.grad, 2.0 * torch.tensor(g), rtol=1e-12, atol=0.0)

    def first3(x3):
        return Window.apply(torch.cat([x3, torch.zeros(1, dtype=torch.float64)]), problem)

    def density(x1):
        return Window.apply(torch.cat([torch.zeros(3, dtype=torch.float64), x1]), problem)

    x3 = torch.zeros(3, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(first3, (x3,), eps=1e-6, atol=0.0, rtol=1e-3)
    x1 = torch.zeros(1, dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(density, (x1,), eps=1e-8, atol=0.0, rtol=1e-3)
