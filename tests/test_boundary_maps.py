"""Ghost-cell and vertex-restriction tables compiled to gather maps (CPU, no device).

For every field that carries a ghost or restriction table in the reference
(src/sale2d.c:2018-2079), random data is pushed through the reference's own sequential
table walk (flush_ght / sync_restrict_vertexes, run by the oracle) and through the gather
map of the library (salec_boundary_map, applied on the host). The results must agree bit
for bit, including the signs of zeros.
"""
import os

import numpy as np
import pytest

from oracle import ref
from salec_b200 import capi, decks

# field -> (ghost pattern, kind) as wired in init_sale2d_ghost (src/sale2d.c:2018-2079)
GHOST = {"m_vof": 0, "e_vel": 3, "e_dvel": 2, "e_den": 5, "e_pre": 0, "e_ste": 4, "e_q": 0, "m_den": 5,
         "m_eng": 5, "m_pty": 0, "e_cvs": 0, "e_vib": 0}
RESTRICT = ["v_dis", "v_acc", "v_vel"]

BOUNDARIES = [
    dict(left="freeslip", right="freeslip", bottom="fixed", top="outflow"),
    dict(left="outflow", right="outflow", bottom="freeslip", top="freeslip"),
    dict(left="freeslip", right="fixed", bottom="outflow", top="fixed"),
    dict(left="mystery", right="mystery", bottom="mystery", top="outflow"),
]


def _run_case(case_id: int, folder: str):
    b = BOUNDARIES[case_id]
    d = decks.Deck(npx=11, npy=9, radius_cells=2, maxstep=1, damp_x=2, damp_y=2, **b)
    d.materials = [decks.Material("basalt_"), decks.Material("dunite_")]
    deck = decks.write_deck(d, folder)
    ref.init(deck, folder, os.path.join(folder, "run"), material=False)
    go = [int(ref.scalar(k)) for k in ("go_left", "go_right", "go_bottom", "go_top")]
    rng = np.random.default_rng(1234 + case_id)
    failures = []
    for name, pat in list(GHOST.items()) + [(n, None) for n in RESTRICT]:
        nx, ny, nc = ref.dims(name)
        data = rng.standard_normal((ny, nx, nc))
        data[rng.random((ny, nx, nc)) < 0.1] = 0.0
        data[rng.random((ny, nx, nc)) < 0.05] = -0.0
        ref.set(name, data)
        if pat is None:
            ref.restrict(name)
            dst, src, ops = capi.boundary_map(1, 0, nx, ny, nc, go)
        else:
            ref.ghost_fill(name)
            dst, src, ops = capi.boundary_map(0, pat, nx, ny, nc, go)
        want = ref.get(name)
        if np.array_equal(want.view(np.int64), data.view(np.int64)) or len(dst) == 0:
            failures.append((name, "table changed nothing", 0))
        got = capi.apply_boundary_map(data, dst, src, ops)
        if not np.array_equal(want.view(np.int64), got.view(np.int64)):
            bad = np.argwhere(want.view(np.int64) != got.view(np.int64))
            failures.append((name, len(bad), bad[:3].tolist()))
    return go, failures


@pytest.mark.parametrize("case_id", range(len(BOUNDARIES)))
def test_boundary_maps_match_reference_tables(oracle_lib, tmp_path, case_id):
    go, failures = ref.run_isolated(_run_case, case_id, str(tmp_path))
    assert not failures, "go=%s mismatches: %s" % (go, failures)
