"""VTK output of a domain's fields (the role of bfam_vtk_write_file,
src/bfam.h:1453-1458): one VTK XML unstructured grid (.vtu) per call, every
element split at its LGL nodes into (Nq-1)^dim linear sub-cells (hexahedra
in 3D, quadrilaterals in 2D), the fields as point data.  Host-side file I/O
only: the state is downloaded through bfam_gpu_domain_get_fields.
"""
from __future__ import annotations

import base64
import struct
from pathlib import Path

import numpy as np

from . import FIELDS_2D, FIELDS_3D, lgl_operators

VTK_QUAD, VTK_HEXAHEDRON = 9, 12


def _subcells(dim: int, Nq: int) -> np.ndarray:
    """Node indices (element-local, i + Nq (j + Nq k)) of the sub-cells, in
    VTK's vertex order"""
    cells = []
    r = range(Nq - 1)
    if dim == 2:
        for j in r:
            for i in r:
                n = lambda a, b: (i + a) + Nq * (j + b)  # noqa: E731
                cells.append([n(0, 0), n(1, 0), n(1, 1), n(0, 1)])
    else:
        for k in r:
            for j in r:
                for i in r:
                    n = lambda a, b, c: (i + a) + Nq * ((j + b) + Nq * (k + c))  # noqa: E731
                    cells.append([n(0, 0, 0), n(1, 0, 0), n(1, 1, 0), n(0, 1, 0),
                                  n(0, 0, 1), n(1, 0, 1), n(1, 1, 1), n(0, 1, 1)])
    return np.array(cells, dtype=np.int64)


def _array(name, data: np.ndarray, ncomp: int, binary: bool) -> str:
    vtype = {np.dtype(np.float64): "Float64", np.dtype(np.int64): "Int64",
             np.dtype(np.uint8): "UInt8"}[data.dtype]
    head = f'<DataArray type="{vtype}" Name="{name}" NumberOfComponents="{ncomp}" '
    if binary:
        raw = np.ascontiguousarray(data).tobytes()
        enc = base64.b64encode(struct.pack("<Q", len(raw)) + raw).decode()
        return head + f'format="binary">{enc}</DataArray>\n'
    txt = " ".join(repr(float(x)) if data.dtype == np.float64 else str(int(x))
                   for x in data.ravel())
    return head + f'format="ascii">{txt}</DataArray>\n'


def write_vtu(path, mesh, q: np.ndarray, time: float | None = None,
              fields=None, binary: bool = True) -> Path:
    """Write fields q [nfields][K*Np] of `mesh` to `path` (.vtu)."""
    path = Path(path)
    dim, Nq, Np, K = mesh.dim, mesh.Nq, mesh.Np, mesh.K
    names = list(fields or (FIELDS_3D if dim == 3 else FIELDS_2D))
    q = np.asarray(q, dtype=np.float64).reshape(len(names), K * Np)
    x, y, z = mesh.node_coordinates(lgl_operators(mesh.N)[0])
    pts = np.stack([x, y, z if dim == 3 else np.zeros_like(x)], axis=1)
    local = _subcells(dim, Nq)
    conn = (local[None, :, :] + (np.arange(K, dtype=np.int64) * Np)[:, None, None])
    nvert = conn.shape[-1]
    conn = conn.reshape(-1, nvert)
    ncell = conn.shape[0]
    offsets = np.arange(1, ncell + 1, dtype=np.int64) * nvert
    types = np.full(ncell, VTK_HEXAHEDRON if dim == 3 else VTK_QUAD, dtype=np.uint8)
    with open(path, "w") as fh:
        fh.write('<?xml version="1.0"?>\n')
        fh.write('<VTKFile type="UnstructuredGrid" version="1.0" '
                 'byte_order="LittleEndian" header_type="UInt64">\n<UnstructuredGrid>\n')
        if time is not None:
            fh.write('<FieldData>\n' + _array("TIME", np.array([time]), 1, binary)
                     + '</FieldData>\n')
        fh.write(f'<Piece NumberOfPoints="{K * Np}" NumberOfCells="{ncell}">\n')
        fh.write('<Points>\n' + _array("Points", pts, 3, binary) + '</Points>\n')
        fh.write('<Cells>\n' + _array("connectivity", conn, 1, binary)
                 + _array("offsets", offsets, 1, binary)
                 + _array("types", types, 1, binary) + '</Cells>\n')
        fh.write(f'<PointData Scalars="{names[0]}">\n')
        for f, nm in enumerate(names):
            fh.write(_array(nm, q[f], 1, binary))
        fh.write('</PointData>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n')
    return path
