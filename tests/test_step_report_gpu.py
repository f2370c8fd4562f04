"""salec_gpu_step_report: the cycles plus the per-cycle read-backs (dt, time, surface profile)
with one synchronisation. It must give exactly what salec_gpu_step followed by
salec_gpu_get_scalar and salec_gpu_get_field give, and reject a profile buffer of the wrong size.
The pipelined form (salec_gpu_step_report_async / salec_gpu_report_wait, two slots, cycle k+1
queued before cycle k's results are waited for) must give the same per-cycle results, and
refuse a slot that is still in flight or was never queued."""
import numpy as np
import pytest

from salec_b200 import capi, decks


@pytest.mark.gpu
def test_step_report_matches_separate_calls(cuda_device, tmp_path):
    deck = decks.write_deck(decks.Deck(npx=40, npy=48, radius_cells=5, damp_x=5, damp_y=5, velocity=-9000.0),
                            str(tmp_path))
    a = capi.Simulation.from_deck(deck, str(tmp_path))
    b = capi.Simulation.from_deck(deck, str(tmp_path))
    prof = np.empty(a.shape("y_profile"))
    for n in (1, 1, 3, 1):
        dt, t = a.step_report(n, prof)
        b.step(n)
        assert dt == b.scalar("dt") and t == b.scalar("time")
        assert np.array_equal(prof, b.get_field("y_profile"))
    dt, t = a.step_report(2)            # no profile requested
    b.step(2)
    assert dt == b.scalar("dt") and t == b.scalar("time")
    t_before = a.scalar("time")
    rc = capi.lib().salec_gpu_step_report(a.h, 1, None, None, capi._ptr(prof), prof.size + 1)
    assert rc == -1                      # argument error, checked before any cycle runs
    assert a.scalar("time") == t_before
    a.close()
    b.close()


@pytest.mark.gpu
def test_step_report_async_pipeline(cuda_device, tmp_path):
    torch = pytest.importorskip("torch")
    deck = decks.write_deck(decks.Deck(npx=40, npy=48, radius_cells=5, damp_x=5, damp_y=5, velocity=-9000.0),
                            str(tmp_path))
    a = capi.Simulation.from_deck(deck, str(tmp_path))
    b = capi.Simulation.from_deck(deck, str(tmp_path))
    shp = a.shape("y_profile")
    bufs = [torch.empty(int(np.prod(shp)), dtype=torch.float64, pin_memory=True).numpy().reshape(shp)
            for _ in range(2)]
    want = []
    for _ in range(6):
        want.append(b.step_report(1, np.empty(shp)) + (b.get_field("y_profile"),))
    got = []
    a.step_report_async(1, bufs[0], 0)
    for k in range(1, 6):
        a.step_report_async(1, bufs[k % 2], k % 2)
        dt, t = a.report_wait((k - 1) % 2)
        got.append((dt, t, bufs[(k - 1) % 2].copy()))
    dt, t = a.report_wait(1)
    got.append((dt, t, bufs[1].copy()))
    for (dw, tw, pw), (dg, tg, pg) in zip(want, got):
        assert dg == dw and tg == tw
        assert np.array_equal(pg, pw)
    a.step_report_async(1, None, 0)
    assert capi.lib().salec_gpu_step_report_async(a.h, 1, None, 0, 0) == -4   # slot 0 still in flight
    a.report_wait(0)
    assert capi.lib().salec_gpu_report_wait(a.h, 0, None, None) == -4         # nothing queued
    a.close()
    b.close()
