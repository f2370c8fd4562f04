"""Output format, pinned on the CPU: a test-side restatement of the reference's VTK writers
(src/write_vtk.c:189-298 and 354-480 with the encoders of src/io/output.c:117-392) rebuilds,
from the oracle's mid-cycle state, the exact bytes of the .vts and .vtp files the reference
wrote. This pins every detail the GPU writer reproduces (array list and order, FP32
conversion, zlib stream fed in 16 KiB pieces, base64 with the four-int32 VTK header, XML,
OUTPUT_GHT extents of a single rank). The GPU writer is checked against the same files in
test_output_gpu.py.
"""
import base64
import struct
import zlib

import numpy as np
import pytest

import trajectory as tj

VTS_ARRAYS = [("v_vel", "v_vel", 0), ("v_acc", "v_acc", 0), ("v_gra", "v_bf", 0), ("v_vof", "v_vof", 0),
              ("e_den", "e_den", 1), ("e_pre", "e_pre", 1), ("e_wpt", "e_wpt", 1), ("e_vof", "m_vof", 1),
              ("e_csd", "e_csd", 1), ("e_dam", "e_dam", 1), ("e_tps", "e_tps", 1), ("e_q", "e_q", 1),
              ("e_tem", "e_tem", 1), ("e_eng", "m_eng", 1), ("m_den", "m_den", 1), ("e_ste2s", "e_ste2s", 1),
              ("e_sta2s", "e_sta2s", 1), ("e_ste", "e_ste", 1), ("e_strength", "e_strength", 1),
              ("e_vib", "e_vib", 1), ("e_ejt", "e_ejt", 1), ("e_cvs", "e_cvs", 1), ("m_pty", "m_pty", 1)]


def encode(values: np.ndarray) -> bytes:
    raw = np.ascontiguousarray(values, dtype=np.float32).tobytes()
    co = zlib.compressobj(zlib.Z_DEFAULT_COMPRESSION)
    z = b"".join(co.compress(raw[i:i + 16384]) for i in range(0, len(raw), 16384)) + co.flush(zlib.Z_FINISH)
    return base64.b64encode(struct.pack("<4i", 1, len(raw), len(raw), len(z))) + base64.b64encode(z)


def data_array(name: str, ncomp: int, values: np.ndarray) -> bytes:
    head = '        <DataArray type="Float32" Name="%s" NumberOfComponents="%d" format="binary">\n' % (name, ncomp)
    return head.encode() + encode(values) + b"\n        </DataArray>\n"


def rebuild_vts(state, nx, ny) -> bytes:
    out = [b'<?xml version="1.0"?>\n',
           b'<VTKFile type="StructuredGrid" version="0.1" compressor="vtkZLibDataCompressor" byte_order="LittleEndian">\n',
           ('  <StructuredGrid WholeExtent="0 %d 0 %d 0 0">\n' % (nx + 2, ny + 2)).encode(),
           ('    <Piece Extent="0 %d 0 %d 0 0">\n' % (nx + 4, ny + 4)).encode(),
           b"      <PointData>\n"]
    for sec in (0, 1):
        if sec == 1:
            out.append(b"      </PointData>\n      <CellData>\n")
        for name, field, s in VTS_ARRAYS:
            if s == sec:
                a = state[field]
                out.append(data_array(name, a.shape[-1], a.reshape(-1)))
    pos = state["v_pos"]
    xyz = np.zeros(pos.shape[:2] + (3,))
    xyz[..., :2] = pos
    out += [b"      </CellData>\n      <Points>\n", data_array("coordinate", 3, xyz.reshape(-1)),
            b"      </Points>\n    </Piece>\n  </StructuredGrid>\n</VTKFile>\n"]
    return b"".join(out)


def rebuild_vtp(state, tracers) -> bytes:
    n = len(tracers)
    cx, cy = tracers[:, 10].astype(int), tracers[:, 11].astype(int)
    f32 = lambda a: np.asarray(a, dtype=np.float64).astype(np.float32)
    cols = [("matid", 1, f32(tracers[:, 9])), ("tag", 1, f32(tracers[:, 8])), ("gx", 1, f32(tracers[:, 6])),
            ("gy", 1, f32(tracers[:, 7])), ("vel", 2, f32(tracers[:, 2:4]).reshape(-1)),
            ("den", 1, f32(state["e_den"][cy, cx, 0])), ("tem", 1, f32(state["e_tem"][cy, cx, 0])),
            ("pre", 1, f32(state["e_pre"][cy, cx, 0])), ("mpre", 1, f32(tracers[:, 4])),
            ("mtem", 1, f32(tracers[:, 5]))]
    out = [b'<?xml version="1.0"?>\n',
           b'<VTKFile type="PolyData" version="1.0" compressor="vtkZLibDataCompressor" byte_order="LittleEndian">\n',
           b"  <PolyData>\n",
           ('    <Piece NumberOfPoints="%d" NumberOfVerts="0" NumberOfLines="0" NumberOfStrips="0" '
            'NumberOfPolys="0">\n' % n).encode(),
           b"      <PointData>\n"]
    out += [data_array(name, k, v) for name, k, v in cols]
    pos = np.zeros((n, 3), dtype=np.float32)
    pos[:, 0], pos[:, 1] = f32(tracers[:, 0]), f32(tracers[:, 1])
    out += [b"      </PointData>\n      <Points>\n", data_array("coordinate", 3, pos.reshape(-1)),
            b"      </Points>\n    </Piece>\n  </PolyData>\n</VTKFile>\n"]
    return b"".join(out)


@pytest.fixture(scope="module")
def case(oracle_lib, tmp_path_factory):
    return tj.oracle_output_cases(["tiny"], 3, str(tmp_path_factory.mktemp("fmt")))["tiny"]


def test_vts_bytes_rebuilt_from_state(case):
    vts = [v for k, v in case["files"].items() if k.startswith("vts/")]
    assert len(vts) == 1
    got = rebuild_vts(case["init"], case["run"]["nx"], case["run"]["ny"])
    assert got == vts[0]


def test_vtp_bytes_rebuilt_from_state(case):
    vtp = [v for k, v in case["files"].items() if k.startswith("vtp/")]
    assert len(vtp) == 1
    assert len(case["tracers0"]) > 0
    assert rebuild_vtp(case["init"], case["tracers0"]) == vtp[0]
