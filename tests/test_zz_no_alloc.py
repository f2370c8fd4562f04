"""The allocation-free CFL entry point (salec_cfl_dt_noalloc) against the step's own CFL phase.

salec_cfl_dt_noalloc serves callers that cannot call cudaMalloc while their time loop runs:
a host code whose device memory is handed to its own pool allocator, or one that cannot
afford cudaMalloc's device-wide synchronisation inside a cycle. It keeps its reduction
scratch in a fixed array inside the library instead of allocating. This test hands it the
same cell fields the step's CFL phase reads, through the C ABI, and checks that two calls in
a row give the time step the step computed, bit for bit: both evaluate the same expression
without contraction and take an exact MIN of order-preserving bits. Two meshes: one whose
cells fit in one block's partial, and one of 300 x 500 cells (37 partials, a row length that
is no multiple of the block) for the multi-block path of both stages. The device buffers are
allocated here by the test, before the calls; the calls themselves allocate nothing. The
file is named so that pytest collects it last.
"""
import numpy as np
import pytest

from salec_b200 import capi, decks


def _bits(x: float) -> int:
    return int(np.array(x, dtype=np.float64).view(np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("npx,npy,radius", [(40, 48, 5), (300, 500, 12)])
def test_cfl_noalloc_matches_step_dt(cuda_device, tmp_path, npx, npy, radius):
    import torch

    d = decks.Deck(npx=npx, npy=npy, radius_cells=radius, maxstep=40, damp_x=5, damp_y=5)
    deck = decks.write_deck(d, str(tmp_path))
    sim = capi.Simulation.from_deck(deck, str(tmp_path))
    run = sim.get_run()
    sim.step(6)                       # a developed impact, not the initial state
    sim.phases(0, 4)                  # everything the CFL phase depends on
    dt_prev = sim.scalar("dt")
    e_vel, e_csd = sim.get_field("e_vel"), sim.get_field("e_csd")
    e_pos, m_vof = sim.get_field("e_pos"), sim.get_field("m_vof")
    sim.phases(5, 6)                  # the step's own CFL reduction
    dt_step = sim.scalar("dt")
    sim.close()
    ncell = run.nx * run.ny
    if npx == 300:
        assert (ncell + 4095) // 4096 >= 20, "the large case must span many partials"

    dev = torch.device("cuda", cuda_device)
    planes = [np.ascontiguousarray(a) for a in (e_vel[..., 0], e_vel[..., 1], e_csd[..., 0], e_pos[..., 2],
                                                  e_pos[..., 3], m_vof[..., 0])]
    bufs = [torch.from_numpy(p).to(dev) for p in planes]
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    for call in range(2):
        out.fill_(-1.0)
        capi.cfl_dt_noalloc(run.nx, run.ny, *[b.data_ptr() for b in bufs], dt_prev, run.max_dt, out.data_ptr(),
                            stream.cuda_stream)
        torch.cuda.synchronize(dev)
        got = float(out.item())
        assert _bits(got) == _bits(dt_step), "call %d: %r vs step dt %r" % (call, got, dt_step)

    # a mesh beyond the scratch limit is refused before anything is launched
    with pytest.raises(capi.SalecError) as err:
        capi.cfl_dt_noalloc(8192, 8192, *[b.data_ptr() for b in bufs], dt_prev, run.max_dt, out.data_ptr(),
                            stream.cuda_stream)
    assert err.value.code == -1 and "limit" in str(err.value)


@pytest.mark.gpu
def test_cfl_noalloc_nan_candidates_match_step(cuda_device, tmp_path):
    """NaN sound speeds in the middle and at the end of the traversal: the allocation-free
    entry point folds NaN candidates as the step does (the reference's sequential MIN), over
    many partials."""
    import torch

    d = decks.Deck(npx=300, npy=500, radius_cells=12, maxstep=40, damp_x=5, damp_y=5)
    deck = decks.write_deck(d, str(tmp_path))
    sim = capi.Simulation.from_deck(deck, str(tmp_path))
    run = sim.get_run()
    sim.step(6)
    sim.phases(0, 4)
    dt_prev = sim.scalar("dt")
    e_vel, e_csd = sim.get_field("e_vel"), sim.get_field("e_csd")
    e_pos, m_vof = sim.get_field("e_pos"), sim.get_field("m_vof")
    vac = m_vof[..., 0] > 1.0 - 1e-6
    order = [(i, j) for j in range(2, run.ny + 2) for i in range(2, run.nx + 2) if not vac[j, i]]
    dev = torch.device("cuda", cuda_device)
    stream = torch.cuda.current_stream(dev)
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    for cell in (order[len(order) // 3], order[-1]):
        csd = e_csd.copy()
        csd[cell[1], cell[0], 0] = np.nan
        sim.set_field("e_csd", csd)
        sim.set_scalar("dt", dt_prev)
        sim.phases(5, 6)
        dt_step = sim.scalar("dt")
        planes = [np.ascontiguousarray(a) for a in (e_vel[..., 0], e_vel[..., 1], csd[..., 0], e_pos[..., 2],
                                                      e_pos[..., 3], m_vof[..., 0])]
        bufs = [torch.from_numpy(p).to(dev) for p in planes]
        torch.cuda.synchronize(dev)
        capi.cfl_dt_noalloc(run.nx, run.ny, *[b.data_ptr() for b in bufs], dt_prev, run.max_dt, out.data_ptr(),
                            stream.cuda_stream)
        torch.cuda.synchronize(dev)
        got = float(out.item())
        if cell == order[-1]:
            assert np.isnan(got) and np.isnan(dt_step)
        else:
            assert not np.isnan(got) and _bits(got) == _bits(dt_step), (cell, got, dt_step)
    sim.close()
