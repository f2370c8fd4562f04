"""NaN candidates in the time-step reduction, against the reference's own CFL phase.

The reference folds the CFL candidates in traversal order with MIN(a, b) = a < b ? a : b
(src/mpi_vec/mpi_vec_types.h:262), starting from 1.1 * dt_prev (src/sale2d.c:1959-2016): a NaN
candidate turns the running value into NaN and the next candidate replaces it, so the result
is the MIN of the candidates after the last NaN, and NaN when the NaN came last. The library's
parallel MIN reproduces that. Here one cell's sound speed is NaN on a mid-cycle state (the
first, a middle and the last cell of the traversal, and none); dt must equal the reference's
bit for bit (NaN for NaN).
"""
import numpy as np
import pytest

import trajectory as tj


def _same(a: float, b: float) -> bool:
    return (np.isnan(a) and np.isnan(b)) or np.array(a).view(np.uint64) == np.array(b).view(np.uint64)


@pytest.mark.gpu
def test_nan_candidates_follow_reference_min(cuda_device, oracle_lib, tmp_path):
    rec = tj.oracle_nan_dt_isolated("base", str(tmp_path))
    assert np.isnan(rec["dt"]["last"]) and not np.isnan(rec["dt"]["middle"])
    sim = tj.simulation_from_record(rec)
    dt_prev = rec["run"]["dt"]
    csd = rec["init"]["e_csd"]
    for case in ("none", "first", "middle", "last"):
        c = csd.copy()
        cell = rec["cells"][case]
        if cell is not None:
            c[cell[1], cell[0], 0] = np.nan
        sim.set_field("e_csd", c)
        sim.set_scalar("dt", dt_prev)
        sim.phases(5, 6)
        got = sim.scalar("dt")
        assert _same(got, rec["dt"][case]), "%s: dt %r vs the reference's %r" % (case, got, rec["dt"][case])
    sim.close()
