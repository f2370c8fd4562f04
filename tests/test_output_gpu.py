"""Output files: the library's .vts/.vtp writer against the reference's own writer.

The oracle runs a deck for a few cycles, stops where the reference writes its VTK files (after
the flux, before the remap: src/salec2d.c:246-250), writes them with sale2d_write_vtk and
sale2d_write_vtp, and hands its state over. The GPU library, loaded with that state, must write
byte-identical files: the same FP32 conversion, zlib stream, base64 encoding, XML and extents.
"""
import os
import re

import pytest

import trajectory as tj

KINDS = ["base", "two_mat", "porous"]


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    return tj.oracle_output_cases(KINDS, 6, str(tmp_path_factory.mktemp("out_oracle")))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", KINDS)
def test_output_files_match_reference(cuda_device, cases, kind, tmp_path):
    rec = cases[kind]
    files = rec["files"]
    vts = [f for f in files if f.startswith("vts/")]
    vtp = [f for f in files if f.startswith("vtp/")]
    assert len(vts) == 1 and len(vtp) == 1, sorted(files)
    m = re.match(r"vts/(.+)\.proc(\d{4})\.(\d{4})\.vts$", vts[0])
    prefix, rank, step = m.group(1), int(m.group(2)), int(m.group(3))

    sim = tj.simulation_from_record(rec)
    sim.write_output(str(tmp_path), prefix, step, rank=rank, wait=True)
    for name, want in files.items():
        path = os.path.join(str(tmp_path), name)
        assert os.path.exists(path), "missing " + name
        with open(path, "rb") as fh:
            got = fh.read()
        if got != want:
            k = next(i for i in range(min(len(got), len(want))) if got[i] != want[i]) \
                if got[:len(want)] != want[:len(got)] else min(len(got), len(want))
            pytest.fail("%s differs from the reference at byte %d (sizes %d vs %d): %r vs %r"
                        % (name, k, len(got), len(want), got[max(0, k - 40):k + 40], want[max(0, k - 40):k + 40]))

    # asynchronous form: queued behind the stream, joined by output_wait
    sim.write_output(str(tmp_path / "async"), prefix, step, rank=rank, wait=False)
    sim.output_wait()
    for name, want in files.items():
        with open(os.path.join(str(tmp_path / "async"), name), "rb") as fh:
            assert fh.read() == want, name
    sim.close()
