"""The reference-side C driver (tests/c_driver.c) against the reference's own run.

The driver is a C program compiled against the reference's headers and sources (oracle/Makefile,
target salec_c_driver): it runs the reference's start-up on the reference's own structures,
fills salec_run_desc and salec_material_desc from sale2d_var, mesh2d_info, cycle_control and
state_reference in C, uploads every field and the tracer list, steps the reference's CPU-runnable
configuration (200 x 400 basalt impact) for 100 cycles with salec_gpu_step_report, and writes the
next cycle's output files with salec_gpu_write_output. The oracle runs the same deck with the
reference's own loop and writers.

Tolerances, stated here: dt within 1e-12, relative L2 at most 1e-9 per field; the output files
hold the same arrays, in the same order, with FP32 values within 1e-5 relative L2 (the FP64
states agree to about 1e-13, so a value sitting on an FP32 rounding boundary can differ in its
last bit, and a one-bit change alters the compressed bytes).
"""
import base64
import os
import re
import subprocess
import zlib

import numpy as np
import pytest

import trajectory as tj
from salec_b200 import decks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "salec_c_driver")
NSTEPS = 100
FIELDS = ["e_den", "e_pre", "m_eng", "m_vof", "v_vel", "e_ste", "e_dam"]


def decode_arrays(xml: bytes):
    """Name -> float32 array of every binary DataArray of a VTK XML file (four-int32 header, zlib)."""
    out = []
    for m in re.finditer(rb'<DataArray type="Float32" Name="([^"]+)" NumberOfComponents="(\d+)" format="binary">\n'
                         rb"(.*?)\n\s*</DataArray>", xml, re.S):
        payload = m.group(3).strip()
        raw = zlib.decompress(base64.b64decode(payload[24:]))
        out.append((m.group(1).decode(), np.frombuffer(raw, dtype=np.float32)))
    return out


def _oracle(deck, folder, nsteps):
    from oracle import ref
    run = os.path.join(folder, "ref")
    ref.init(deck, folder, run)
    ref.step(nsteps)
    res = {n: ref.get(n) for n in FIELDS}
    res["dt"], res["time"] = ref.scalar("dt"), ref.scalar("time")
    ref.phases(0, 13)
    ref.write_output()
    res["files"] = {}
    for sub in ("vts", "vtp"):
        for f in sorted(os.listdir(os.path.join(run, sub))):
            with open(os.path.join(run, sub, f), "rb") as fh:
                res["files"][sub + "/" + f] = fh.read()
    return res


@pytest.mark.gpu
def test_c_driver_matches_reference(cuda_device, oracle_lib, tmp_path):
    assert os.path.exists(DRIVER), "the C driver is built by oracle/Makefile (salec_c_driver) with the library"
    folder = str(tmp_path)
    deck = decks.write_deck(decks.config1_deck(), folder)
    want = oracle_lib.run_isolated(_oracle, deck, folder, NSTEPS)
    work = os.path.join(folder, "gpu")
    res = subprocess.run([DRIVER, deck, folder, work, str(NSTEPS)], capture_output=True, text=True, timeout=1200)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    with open(os.path.join(work, "gpu_fields.bin"), "rb") as fh:
        blob = np.frombuffer(fh.read(), dtype=np.float64)
    dt, t = blob[0], blob[1]
    assert abs(dt - want["dt"]) <= 1e-12 * want["dt"], (dt, want["dt"])
    assert abs(t - want["time"]) <= 1e-12 * want["time"]
    off = 2
    for n in FIELDS:
        w = want[n]
        got = blob[off:off + w.size].reshape(w.shape)
        off += w.size
        err = tj.rel_l2(got, w)
        assert err <= 1e-9, "%s: relative L2 %.3e" % (n, err)
    assert off == blob.size
    for name, ref_bytes in want["files"].items():
        path = os.path.join(work, name)
        assert os.path.exists(path), name
        with open(path, "rb") as fh:
            mine = fh.read()
        a, b = decode_arrays(mine), decode_arrays(ref_bytes)
        assert [x[0] for x in a] == [x[0] for x in b], name
        for (n, x), (_, y) in zip(a, b):
            assert x.shape == y.shape, (name, n)
            assert tj.rel_l2(x.astype(np.float64), y.astype(np.float64)) <= 1e-5, (name, n)
        head = lambda s: re.sub(rb">\n[A-Za-z0-9+/=]+\n", b">\n\n", s)
        assert head(mine) == head(ref_bytes), name
