"""salec_gpu_step_report: the cycles plus the per-cycle read-backs (dt, time, surface profile)
with one synchronisation. It must give exactly what salec_gpu_step followed by
salec_gpu_get_scalar and salec_gpu_get_field give, and reject a profile buffer of the wrong size."""
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
