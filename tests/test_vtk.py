"""VTK output (.vtu): geometry, sub-cells and point data read back."""
from __future__ import annotations

import base64
import struct
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import bfam_b200 as bf
from bfam_b200 import vtk


def _read(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    arrays = {}
    for da in root.iter("DataArray"):
        t = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}[da.get("type")]
        if da.get("format") == "binary":
            raw = base64.b64decode(da.text)
            n = struct.unpack("<Q", raw[:8])[0]
            arrays[da.get("Name")] = np.frombuffer(raw[8:8 + n], dtype=t)
        else:
            arrays[da.get("Name")] = np.array(da.text.split(), dtype=t)
    return piece, arrays


@pytest.mark.parametrize("dim,N,n", [(3, 3, (2, 2, 2)), (2, 4, (3, 2))])
@pytest.mark.parametrize("binary", [True, False])
def test_vtu_round_trip(tmp_path, dim, N, n, binary):
    m = bf.Mesh(dim, N, n, refine_prob=0.5, seed=2)
    rng = np.random.default_rng(0)
    q = rng.standard_normal((m.nfields, m.K * m.Np))
    p = vtk.write_vtu(tmp_path / "state.vtu", m, q, time=0.25, binary=binary)
    piece, a = _read(p)
    nsub = (N ** dim)
    assert int(piece.get("NumberOfPoints")) == m.K * m.Np
    assert int(piece.get("NumberOfCells")) == m.K * nsub
    names = bf.FIELDS_3D if dim == 3 else bf.FIELDS_2D
    for f, nm in enumerate(names):
        assert np.array_equal(a[nm], q[f])
    assert a["TIME"][0] == 0.25
    pts = a["Points"].reshape(-1, 3)
    x, y, z = m.node_coordinates(bf.lgl_operators(N)[0])
    assert np.array_equal(pts[:, 0], x) and np.array_equal(pts[:, 1], y)
    conn = a["connectivity"].reshape(m.K * nsub, -1)
    assert conn.shape[1] == (8 if dim == 3 else 4)
    assert conn.min() == 0 and conn.max() == m.K * m.Np - 1
    # every sub-cell has positive volume (vertex order as VTK expects)
    c0 = pts[conn[:, 0]]
    e1 = pts[conn[:, 1]] - c0
    e3 = pts[conn[:, 3]] - c0
    if dim == 3:
        e4 = pts[conn[:, 4]] - c0
        assert np.all(np.einsum("ij,ij->i", np.cross(e1, e3), e4) > 0)
    else:
        assert np.all(e1[:, 0] * e3[:, 1] - e1[:, 1] * e3[:, 0] > 0)


@pytest.mark.gpu
def test_domain_writes_its_device_state(tmp_path):
    m = bf.Mesh(3, 3, (2, 2, 2), refine_prob=0.5, seed=2)
    rho, lam, mu = bf.material_random(m.K, 1)
    q0 = m.gaussian_pulse(bf.lgl_operators(3)[0], (0.5, 0.5, 0.5), 0.2)
    d = bf.GpuDomain(m, rho, lam, mu)
    d.set_fields(q0)
    bf.LSRK(d).step(1e-3, 3)
    _, a = _read(d.write_vtu(tmp_path / "s.vtu", time=3e-3))
    assert np.array_equal(a["sxx"], d.get_fields()[3])
