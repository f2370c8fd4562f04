"""Generate the committed golden vectors of the mesh update (test infrastructure).

Run where the oracle library oracle/_ref/libsalec_ref.so exists (it is compiled from the
reference's own C sources by oracle/Makefile):

    python tests/golden/make_golden.py

It writes ``tiny_impact.npz``: the reference's initialised state of a 12x16-cell impact deck
(Tillotson basalt projectile into a basalt target, RockStrengthT strength with Ivanov damage,
PML 3 layers, gravity), the run-wide scalars and material parameters a host driver hands to
the C ABI, the initial tracers, and the evolved state after steps 1, 2, 5 and 10 of the
reference's own time loop (src/salec2d.c:115-272), every value as FP64 bytes.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = os.path.dirname(HERE)
ROOT = os.path.dirname(TESTS)
for p in (ROOT, os.path.join(ROOT, "salec-2d-public_b200"), TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(HERE, "tiny_impact.npz")
KEPT_STEPS = (1, 2, 5, 10)


def generate(path: str = GOLDEN) -> str:
    import trajectory
    with tempfile.TemporaryDirectory() as tmp:
        rec = trajectory.trajectories(["tiny"], max(KEPT_STEPS), tmp)["tiny"]
    out = {}
    for n, v in rec["run"].items():
        out["run/" + n] = np.asarray(v)
    for m, mat in enumerate(rec["mats"]):
        for n, v in mat.items():
            out["mat%d/%s" % (m, n)] = np.asarray(v)
    out["nmat"] = np.asarray(len(rec["mats"]))
    for n, a in rec["init"].items():
        out["init/" + n] = a
    out["tracers0"] = rec["tracers0"]
    for k in KEPT_STEPS:
        st = rec["steps"][k - 1]
        for n, a in st.items():
            out["step%d/%s" % (k, n)] = np.asarray(a)
    np.savez_compressed(path, **out)
    return path


def load(path: str = GOLDEN):
    """Return (record, steps): ``record`` in the layout of trajectory.oracle_trajectory (run,
    mats, init, tracers0) and ``steps`` = {step number: {field or 'dt'/'time'/'tracers': array}}."""
    z = np.load(path)
    rec = {"run": {}, "mats": [], "init": {}, "tracers0": z["tracers0"]}
    nmat = int(z["nmat"])
    rec["mats"] = [{} for _ in range(nmat)]
    steps = {}
    for key in z.files:
        if "/" not in key:
            continue
        head, name = key.split("/", 1)
        v = z[key]
        if head == "run":
            rec["run"][name] = v.tolist() if v.ndim else v.item()
        elif head.startswith("mat"):
            rec["mats"][int(head[3:])][name] = v if v.ndim else v.item()
        elif head == "init":
            rec["init"][name] = v
        elif head.startswith("step"):
            steps.setdefault(int(head[4:]), {})[name] = v if v.ndim else v.item()
    return rec, steps


if __name__ == "__main__":
    p = generate()
    print(p, os.path.getsize(p), "bytes")
