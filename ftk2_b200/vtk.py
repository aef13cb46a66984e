"""VTK XML output of extraction results from Python, byte for byte the files
include/ftk2b/vtk.hpp writes for the same complex (the reference's
write_complex_to_vtp / write_complex_to_vtu, utils/vtk.hpp:26-160, without
VTK).

One point per feature at sum_i (double)(float barycentric_i) * vertex
coordinates (mesh.vertex_coordinates), first three coordinates as Float32;
point arrays Scalar (Float32), TrackID (Int32), Type (Int32) and Time
(Float32: the last coordinate where the mesh's total dimension exceeds its
spatial one, else 0).  Connectivity: CPResult star edges (dimension 1),
ContourResult manifold cells (dimension = cell width - 1), or an explicit
`connectivity` list of (dimension, flat indices) on the result.  ASCII when
use_ascii is set or FTK_DEBUG is in the environment, else appended data in
base64 with UInt64 block headers and no compression, as the reference sets up
VTK's writer (utils/vtk.hpp:102-108, 150-156): per array the base64 of its
length header, then the base64 of its bytes, each padded on its own.  read_vtu loads an unstructured base mesh as the
reference's read_vtu does (utils/vtk.hpp:165-192), same result as the C++
header's.
"""
from __future__ import annotations

import base64
import io
import os
from typing import List, Tuple

import numpy as np

_VTK_TYPE = {0: 1, 1: 3, 2: 5, 3: 10}  # VERTEX, LINE, TRIANGLE, TETRA


def _connectivity(result) -> List[Tuple[int, np.ndarray]]:
    conn = getattr(result, "connectivity", None)
    if conn is not None:
        return [(int(d), np.asarray(i, np.uint32).reshape(-1)) for d, i in conn]
    cells = getattr(result, "cells", None)
    if cells is not None:
        c = np.asarray(cells)
        return [(c.shape[1] - 1, c.reshape(-1).astype(np.uint32))] if c.ndim == 2 and c.size else []
    e = np.asarray(getattr(result, "edges", np.zeros((0, 2), np.uint32)))
    return [(1, e.reshape(-1).astype(np.uint32))] if e.size else []


def complex_points(result, mesh):
    """(xyz (n, 3) float32, scalar, track, type, time) of a result's features."""
    simp = np.asarray(result.simplices, np.uint64)
    n = simp.shape[0]
    k = simp.shape[1] if simp.ndim == 2 else 1
    bary = np.asarray(result.bary, np.float32).reshape(n, k)
    td, sd = mesh.get_total_dimension(), mesh.get_spatial_dimension()
    pos = np.zeros((n, td), np.float64)
    if n:
        vc = mesh.vertex_coordinates(simp.reshape(n, k))
        for v in range(min(k, 5)):
            for j in range(min(td, vc.shape[-1])):
                pos[:, j] += bary[:, v].astype(np.float64) * vc[:, v, j]
    xyz = np.zeros((n, 3), np.float32)
    xyz[:, :min(3, td)] = pos[:, :3].astype(np.float32)
    time = pos[:, -1].astype(np.float32) if td > sd and td > 0 else np.zeros(n, np.float32)
    typ = getattr(result, "type", None)
    typ = np.zeros(n, np.int32) if typ is None else np.asarray(typ).astype(np.int64).astype(np.int32)
    track = np.asarray(result.track_id).astype(np.int64).astype(np.int32)
    return xyz.reshape(-1), np.asarray(result.scalar, np.float32), track, typ, time


class _Writer:
    def __init__(self, ascii_: bool):
        self.ascii = ascii_
        self.body = io.StringIO()
        self.appended = bytearray()

    def array(self, vtype: str, name: str, ncomp: int, a: np.ndarray, indent: str):
        w = self.body.write
        w(f'{indent}<DataArray type="{vtype}" Name="{name}"')
        if ncomp > 1:
            w(f' NumberOfComponents="{ncomp}"')
        if not self.ascii:
            w(f' format="appended" offset="{len(self.appended)}"/>\n')
            raw = np.ascontiguousarray(a).tobytes()
            self.appended += base64.b64encode(np.array([len(raw)], "<u8").tobytes()) + base64.b64encode(raw)
            return
        w(' format="ascii">\n')
        vals = ["%.9g" % float(v) for v in a] if vtype == "Float32" else [str(int(v)) for v in a]
        for i, s in enumerate(vals):
            if i % 6 == 0:
                w(indent + "  ")
            w(s + ("\n" if (i % 6 == 5 or i + 1 == len(vals)) else " "))
        w(f"{indent}</DataArray>\n")

    def save(self, path: str, vtype: str):
        with open(path, "wb") as f:
            f.write((f'<?xml version="1.0"?>\n<VTKFile type="{vtype}" version="1.0" byte_order="LittleEndian" '
                     f'header_type="UInt64">\n').encode())
            f.write(self.body.getvalue().encode())
            if not self.ascii:
                f.write(b'  <AppendedData encoding="base64">\n   _' + bytes(self.appended) + b"\n  </AppendedData>\n")
            f.write(b"</VTKFile>\n")


def _point_data(w: _Writer, pts):
    xyz, scalar, track, typ, time = pts
    w.body.write("      <PointData>\n")
    w.array("Float32", "Scalar", 1, scalar.astype("<f4"), "        ")
    w.array("Int32", "TrackID", 1, track.astype("<i4"), "        ")
    w.array("Int32", "Type", 1, typ.astype("<i4"), "        ")
    w.array("Float32", "Time", 1, time.astype("<f4"), "        ")
    w.body.write("      </PointData>\n      <CellData>\n      </CellData>\n      <Points>\n")
    w.array("Float32", "Points", 3, xyz.astype("<f4"), "        ")
    w.body.write("      </Points>\n")


def _cells(items):
    conn, offs, types = [], [], []
    total = 0
    for d, idx in items:
        w = d + 1
        m = len(idx) // w
        if m:
            conn.append(idx[:m * w].astype(np.int64))
            offs.append(total + w * np.arange(1, m + 1, dtype=np.int64))
            types.append(np.full(m, _VTK_TYPE.get(d, 0), np.uint8))
            total += m * w
    cat = (lambda a, dt: np.concatenate(a) if a else np.zeros(0, dt))
    return cat(conn, np.int64), cat(offs, np.int64), cat(types, np.uint8)


def _ascii(use_ascii: bool) -> bool:
    return bool(use_ascii) or "FTK_DEBUG" in os.environ


def write_complex_to_vtp(result, mesh, filename: str, target_dim: int = -1, use_ascii: bool = False) -> None:
    """write_complex_to_vtp (utils/vtk.hpp:75-115): dimension 0 / 1 / 2
    connectivity as verts / lines / polys."""
    pts = complex_points(result, mesh)
    conn = [(d, i) for d, i in _connectivity(result) if (target_dim == -1 or d == target_dim) and 0 <= d <= 2]
    secs = [_cells([(d, i) for d, i in conn if d == k]) for k in range(3)]
    w = _Writer(_ascii(use_ascii))
    w.body.write(f'  <PolyData>\n    <Piece NumberOfPoints="{len(pts[1])}" NumberOfVerts="{len(secs[0][2])}" '
                 f'NumberOfLines="{len(secs[1][2])}" NumberOfStrips="0" NumberOfPolys="{len(secs[2][2])}">\n')
    _point_data(w, pts)
    empty = (np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.uint8))
    for tag, c in (("Verts", secs[0]), ("Lines", secs[1]), ("Strips", empty), ("Polys", secs[2])):
        w.body.write(f"      <{tag}>\n")
        w.array("Int64", "connectivity", 1, c[0].astype("<i8"), "        ")
        w.array("Int64", "offsets", 1, c[1].astype("<i8"), "        ")
        w.body.write(f"      </{tag}>\n")
    w.body.write("    </Piece>\n  </PolyData>\n")
    w.save(filename, "PolyData")


def write_complex_to_vtu(result, mesh, filename: str, target_dim: int = -1, use_ascii: bool = False) -> None:
    """write_complex_to_vtu (utils/vtk.hpp:117-160): connectivity of
    dimension 0..3 as VERTEX / LINE / TRIANGLE / TETRA, or one VERTEX per
    feature for target_dim 0."""
    pts = complex_points(result, mesh)
    n = len(pts[1])
    if target_dim == 0:
        conn, offs, types = (np.arange(n, dtype=np.int64), np.arange(1, n + 1, dtype=np.int64),
                             np.ones(n, np.uint8))
    else:
        conn, offs, types = _cells([(d, i) for d, i in _connectivity(result)
                                    if (target_dim == -1 or d == target_dim) and 0 <= d <= 3])
    w = _Writer(_ascii(use_ascii))
    w.body.write(f'  <UnstructuredGrid>\n    <Piece NumberOfPoints="{n}" NumberOfCells="{len(types)}">\n')
    _point_data(w, pts)
    w.body.write("      <Cells>\n")
    w.array("Int64", "connectivity", 1, conn.astype("<i8"), "        ")
    w.array("Int64", "offsets", 1, offs.astype("<i8"), "        ")
    w.array("UInt8", "types", 1, types, "        ")
    w.body.write("      </Cells>\n    </Piece>\n  </UnstructuredGrid>\n")
    w.save(filename, "UnstructuredGrid")


# ---------------------------------------------------------------- reading

_NP = {"Float32": "<f4", "Float64": "<f8", "Int8": "i1", "UInt8": "u1", "Int16": "<i2", "UInt16": "<u2",
       "Int32": "<i4", "UInt32": "<u4", "Int64": "<i8", "UInt64": "<u8"}


def _attrs(tag: str) -> dict:
    import re
    return dict(re.findall(r'(\w+)="([^"]*)"', tag))


def _b64_stream(text: bytes, start: int, want: int) -> bytes:
    """Decode base64 quanta from start until want bytes are out; '=' padding
    may close a quantum mid-stream (a header encoded apart from its data)."""
    import binascii
    out, quantum, p = bytearray(), bytearray(), start
    while len(out) < want and p < len(text):
        c = text[p:p + 1]
        p += 1
        if c == b"<":
            break
        if c.isspace():
            continue
        quantum += c
        if len(quantum) == 4:
            out += binascii.a2b_base64(bytes(quantum))
            quantum.clear()
    return bytes(out)


def read_vtu(filename: str):
    """read_vtu (utils/vtk.hpp:165-192): points and the triangles and
    tetrahedra of a single-piece, little-endian, uncompressed VTU file (ASCII,
    inline base64, appended base64 or appended raw) as
    UnstructuredSimplicialMesh(cell_dim, cell_dim, coords, cells); cell_dim is
    that of the last triangle or tetrahedron.  None if the file cannot be
    opened."""
    import re
    from . import api
    try:
        data = open(filename, "rb").read()
    except OSError:
        return None
    m = re.search(rb"<VTKFile([^>]*)>", data)
    root = _attrs(m.group(1).decode()) if m else {}
    if root.get("type") != "UnstructuredGrid":
        raise ValueError(f"not a VTK UnstructuredGrid file: {filename}")
    if root.get("byte_order") == "BigEndian" or root.get("compressor"):
        raise ValueError("big-endian or compressed VTU")
    hb = 8 if root.get("header_type") == "UInt64" else 4
    app_at, raw = None, False
    am = re.search(rb"<AppendedData([^>]*)>", data)
    if am:
        raw = _attrs(am.group(1).decode()).get("encoding") == "raw"
        app_at = data.index(b"_", am.end()) + 1
    piece = _attrs(re.search(rb"<Piece([^>]*)>", data).group(1).decode())
    n_pts, n_cells = int(piece["NumberOfPoints"]), int(piece["NumberOfCells"])

    def array(section: bytes, name):
        s = data.index(b"<" + section, 0)
        e = data.index(b"</" + section + b">", s)
        for dm in re.finditer(rb"<DataArray([^>]*?)(/?)>", data[s:e]):
            a = _attrs(dm.group(1).decode())
            if name is None or a.get("Name") == name:
                return a, s + dm.end()
        raise ValueError(f"VTU lacks DataArray {name}")

    def values(a: dict, body: int, count: int) -> np.ndarray:
        dt = np.dtype(_NP[a["type"]])
        fmt = a.get("format", "ascii")
        if fmt == "ascii":
            txt = data[body:data.index(b"</DataArray>", body)].split()[:count]
            return np.array([float(t) for t in txt], np.float64).astype(dt)
        need = hb + count * dt.itemsize
        if fmt == "binary":
            b = _b64_stream(data, body, need)
        else:
            off = app_at + int(a["offset"])
            b = data[off:off + need] if raw else _b64_stream(data, off, need)
        if len(b) < need:
            raise ValueError("truncated DataArray in VTU")
        return np.frombuffer(b[hb:need], dt)

    pa, pb = array(b"Points", None)
    nc = int(pa.get("NumberOfComponents", "1") or 1)
    xyz = values(pa, pb, n_pts * nc).astype(np.float64).reshape(n_pts, nc)
    coords = np.zeros((n_pts, 3), np.float64)
    coords[:, :min(3, nc)] = xyz[:, :3]
    offs = values(*array(b"Cells", "offsets"), n_cells).astype(np.int64)
    types = values(*array(b"Cells", "types"), n_cells).astype(np.int64)
    conn = values(*array(b"Cells", "connectivity"), int(offs[-1]) if n_cells else 0).astype(np.uint64)
    cells, cell_dim = [], 0
    for i in range(n_cells):
        if types[i] == 5:
            cell_dim = 2
        elif types[i] == 10:
            cell_dim = 3
        else:
            continue
        cells.append(conn[(offs[i - 1] if i else 0):offs[i]])
    flat = np.concatenate(cells) if cells else np.zeros(0, np.uint64)
    if all(len(c) == cell_dim + 1 for c in cells):
        return api.UnstructuredSimplicialMesh(cell_dim, cell_dim, coords, flat)
    # triangles and tetrahedra mixed: the flat id list, as the reference keeps it
    mesh = api.UnstructuredSimplicialMesh.__new__(api.UnstructuredSimplicialMesh)
    mesh.spatial_dim, mesh.cell_dim, mesh.coords, mesh.cells = cell_dim, cell_dim, coords, flat
    return mesh
