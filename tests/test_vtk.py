"""VTK XML writers and reader of include/ftk2b/vtk.hpp, against the content
that utils/vtk.hpp:26-192 of the reference produces through VTK: one point per
feature at sum_i (double)(float barycentric_i) * vertex coordinates (stored as
Float32, first three coordinates), point arrays Scalar / TrackID / Type / Time
(time = last coordinate only where the mesh has more total than spatial
dimensions), verts / lines / polys (VTP) or VERTEX / LINE / TRIANGLE / TETRA
cells (VTU), the target_dim filter; and read_vtu on files in ASCII, inline
base64, appended base64 and appended raw form.  Expected values are computed
here from those formulas; the C++ header runs through tests/cpp/vtk_run.cpp
(host code only, no GPU)."""
import base64
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DT = {"Float32": "<f4", "Float64": "<f8", "Int32": "<i4", "Int64": "<i8", "UInt8": "u1", "UInt32": "<u4",
      "UInt64": "<u8"}


@pytest.fixture(scope="module")
def vtk_run(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ absent")
    exe = str(tmp_path_factory.mktemp("vtkbin") / "vtk_run")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "vtk_run.cpp"), "-o", exe], check=True)
    return exe


# ---------------------------------------------------------------- cases

def regular_case(rng):
    g = [5, 4, 3, 3]
    mesh = ("regular", g)
    n = 7
    feats = []
    for i in range(n):
        vid = np.sort(rng.choice(int(np.prod(g)), 4, replace=False)).astype(np.uint64)
        lam = rng.dirichlet(np.ones(4)).astype(np.float32)
        feats.append((3, vid, lam, int(rng.integers(0, 5)), int(rng.integers(0, 3)), np.float32(rng.normal())))
    conn = [(1, rng.integers(0, n, 8).astype(np.uint32)), (3, rng.integers(0, n, 8).astype(np.uint32)),
            (2, rng.integers(0, n, 6).astype(np.uint32)), (0, np.array([2, 5], np.uint32))]
    return mesh, feats, conn


def extruded_case(rng, spatial_dim):
    nv = 6
    coords = rng.normal(size=(nv, 3))
    cells = np.array([[0, 1, 2], [1, 2, 3], [2, 3, 4], [3, 4, 5]], np.uint64)
    mesh = ("extruded", spatial_dim, 2, coords, cells, 3)
    feats = []
    for i in range(5):
        vid = np.sort(rng.choice(nv * 4, 3, replace=False)).astype(np.uint64)
        lam = rng.dirichlet(np.ones(3)).astype(np.float32)
        feats.append((2, vid, lam, i // 2, 0, np.float32(0.25)))
    conn = [(1, np.array([0, 1, 1, 2, 3, 4], np.uint32)), (2, np.array([0, 1, 2, 2, 3, 4], np.uint32))]
    return mesh, feats, conn


def extruded_regular_case(rng):
    g = [4, 3]
    mesh = ("extruded_regular", g, 2)
    S = g[0] + g[0] * g[1]  # grid_index_to_id(global dims) of the spatial grid
    feats = []
    for i in range(4):
        vid = np.sort(rng.choice(S * 3, 3, replace=False)).astype(np.uint64)
        lam = rng.dirichlet(np.ones(3)).astype(np.float32)
        feats.append((2, vid, lam, 0, 1, np.float32(-1.5)))
    conn = [(1, np.array([0, 1, 2, 3], np.uint32))]
    return mesh, feats, conn


def case_text(mesh, feats, conn):
    out = []
    if mesh[0] == "regular":
        g = mesh[1]
        out += ["mesh regular", str(len(g)), " ".join(map(str, g)), " ".join("0" * len(g)), " ".join(map(str, g))]
    elif mesh[0] == "extruded":
        _, sd, cd, coords, cells, nl = mesh
        out += ["mesh extruded", f"{sd} {cd} {len(coords)}", " ".join(f"{v:.17g}" for v in coords.reshape(-1)),
                str(len(cells)), " ".join(map(str, cells.reshape(-1))), str(nl)]
    else:
        _, g, nl = mesh
        out += ["mesh extruded_regular", str(len(g)), " ".join(map(str, g)), str(nl)]
    out.append(f"features {len(feats)}")
    for dim, vid, lam, track, typ, sc in feats:
        out.append(" ".join([str(dim)] + [str(int(v)) for v in vid] + [f"{float(x):.9g}" for x in lam]
                            + [str(track), str(typ), f"{float(sc):.9g}"]))
    out.append(f"connectivity {len(conn)}")
    for dim, idx in conn:
        out.append(" ".join([str(dim), str(len(idx))] + [str(int(v)) for v in idx]))
    return "\n".join(out) + "\n"


def vertex_coords(mesh, vid):
    """get_vertex_coordinates (mesh.hpp:374-378, 714-720; unstructured_mesh.hpp:100-107)."""
    vid = int(vid)
    if mesh[0] == "regular":
        c = []
        for d in mesh[1]:
            c.append(float(vid % d))
            vid //= d
        return c
    if mesh[0] == "extruded":
        _, sd, _, coords, _, _ = mesh
        S = len(coords)
        return [float(x) for x in coords[vid % S][:sd]] + [float(vid // S)]
    g = mesh[1]
    S, mul = 0, 1
    for d in g:
        S += d * mul
        mul *= d
    s, c = vid % S, []
    for d in g:
        c.append(float(s % d))
        s //= d
    return c + [float(vid // S)]


def dims(mesh):
    """(total, spatial) dimension."""
    if mesh[0] == "regular":
        return len(mesh[1]), len(mesh[1])
    if mesh[0] == "extruded":
        return mesh[2] + 1, mesh[1]
    return len(mesh[1]) + 1, len(mesh[1])


def expected_points(mesh, feats):
    td, sd = dims(mesh)
    xyz = np.zeros((len(feats), 3), np.float32)
    time = np.zeros(len(feats), np.float32)
    for i, (dim, vid, lam, _, _, _) in enumerate(feats):
        pos = [0.0] * td
        for v in range(dim + 1):
            vc = vertex_coords(mesh, vid[v])
            for j in range(min(td, len(vc))):
                pos[j] += float(lam[v]) * vc[j]
        for j in range(min(3, td)):
            xyz[i, j] = np.float32(pos[j])
        time[i] = np.float32(pos[-1]) if td > sd else np.float32(0.0)
    return xyz, time


# ---------------------------------------------------------------- parsing

def parse_vtk(path):
    """{(section, name): array} and the Piece attributes of an ASCII or
    appended-base64 VTK XML file (each array's length header and its bytes
    encoded apart, as VTK's writer does without compression)."""
    data = open(path, "rb").read()
    head, sep, tail = data.partition(b'<AppendedData encoding="base64">')
    app = tail[tail.index(b"_") + 1:tail.index(b"\n  </AppendedData>")] if sep else None
    text = head.decode()
    piece = dict(re.findall(r'(\w+)="([^"]*)"', re.search(r"<Piece ([^>]*)>", text).group(1)))
    out, section = {}, None
    for m in re.finditer(r"<(PointData|CellData|Points|Verts|Lines|Strips|Polys|Cells)>|<DataArray ([^>]*?)(/?)>",
                         text):
        if m.group(1):
            section = m.group(1)
            continue
        at = dict(re.findall(r'(\w+)="([^"]*)"', m.group(2)))
        dt = np.dtype(DT[at["type"]])
        if at["format"] == "ascii":
            body = text[m.end():text.index("</DataArray>", m.end())]
            a = np.array(body.split(), dtype=np.float64).astype(dt) if body.split() else np.zeros(0, dt)
        else:
            off = int(at["offset"])
            nb = int(np.frombuffer(base64.b64decode(app[off:off + 12]), "<u8")[0])
            text = app[off + 12:off + 12 + 4 * ((nb + 2) // 3)]
            assert all(c in b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/=" for c in text)
            a = np.frombuffer(base64.b64decode(text), dt)
        out[(section, at["Name"])] = a
    return out, piece


def check_points(got, mesh, feats):
    xyz, time = expected_points(mesh, feats)
    assert np.array_equal(got[("Points", "Points")].reshape(-1, 3).view(np.uint32), xyz.view(np.uint32))
    assert np.array_equal(got[("PointData", "Time")].view(np.uint32), time.view(np.uint32))
    assert got[("PointData", "TrackID")].tolist() == [f[3] for f in feats]
    assert got[("PointData", "Type")].tolist() == [f[4] for f in feats]
    assert np.array_equal(got[("PointData", "Scalar")], np.array([f[5] for f in feats], np.float32))


def expected_cells(conn, dims_kept):
    ids, offs, types = [], [], []
    vtk_type = {0: 1, 1: 3, 2: 5, 3: 10}
    for dim, idx in conn:
        if dim not in dims_kept:
            continue
        for i in range(0, len(idx) - dim, dim + 1):
            ids += idx[i:i + dim + 1].tolist()
            offs.append(len(ids))
            types.append(vtk_type[dim])
    return ids, offs, types


CASES = {
    "regular_3d_t": lambda rng: regular_case(rng),
    "extruded_tri_2d": lambda rng: extruded_case(rng, 2),
    "extruded_tri_3d_coords": lambda rng: extruded_case(rng, 3),
    "extruded_regular_2d": lambda rng: extruded_regular_case(rng),
}


@pytest.mark.parametrize("name", list(CASES))
def test_writers_match_reference_content(vtk_run, tmp_path, name):
    mesh, feats, conn = CASES[name](np.random.default_rng(len(name)))
    (tmp_path / "case.txt").write_text(case_text(mesh, feats, conn))
    subprocess.run([vtk_run, "write", str(tmp_path / "case.txt"), str(tmp_path)], check=True)
    for f in ("all_ascii.vtp", "all_bin.vtp"):
        got, piece = parse_vtk(tmp_path / f)
        check_points(got, mesh, feats)
        for sec, dim in (("Verts", 0), ("Lines", 1), ("Polys", 2)):
            ids, offs, _ = expected_cells(conn, {dim})
            assert got[(sec, "connectivity")].tolist() == ids, (f, sec)
            assert got[(sec, "offsets")].tolist() == offs, (f, sec)
        assert got[("Strips", "connectivity")].size == 0
        assert int(piece["NumberOfLines"]) == len(expected_cells(conn, {1})[1])
    got, _ = parse_vtk(tmp_path / "dim1_ascii.vtp")
    assert got[("Lines", "connectivity")].tolist() == expected_cells(conn, {1})[0]
    assert got[("Verts", "connectivity")].size == 0 and got[("Polys", "connectivity")].size == 0
    for f, kept in (("all_ascii.vtu", {0, 1, 2, 3}), ("all_bin.vtu", {0, 1, 2, 3}), ("dim3_ascii.vtu", {3})):
        got, piece = parse_vtk(tmp_path / f)
        check_points(got, mesh, feats)
        ids, offs, types = expected_cells(conn, kept)
        assert got[("Cells", "connectivity")].tolist() == ids, f
        assert got[("Cells", "offsets")].tolist() == offs, f
        assert got[("Cells", "types")].tolist() == types, f
        assert int(piece["NumberOfCells"]) == len(types)
    got, piece = parse_vtk(tmp_path / "dim0_bin.vtu")
    n = len(feats)
    assert got[("Cells", "connectivity")].tolist() == list(range(n))
    assert got[("Cells", "types")].tolist() == [1] * n and got[("Cells", "offsets")].tolist() == list(range(1, n + 1))


def test_ftk_debug_forces_ascii(vtk_run, tmp_path):
    mesh, feats, conn = extruded_case(np.random.default_rng(3), 2)
    (tmp_path / "case.txt").write_text(case_text(mesh, feats, conn))
    subprocess.run([vtk_run, "write", str(tmp_path / "case.txt"), str(tmp_path)], check=True,
                   env=dict(os.environ, FTK_DEBUG="1"))
    assert b"AppendedData" not in (tmp_path / "all_bin.vtu").read_bytes()
    got, _ = parse_vtk(tmp_path / "all_bin.vtu")
    check_points(got, mesh, feats)


# ---------------------------------------------------------------- read_vtu

def make_vtu(points, cells, enc, header="UInt64", joint=False):
    """A VTU file as a VTK writer lays it out: enc is ascii, binary (inline
    base64), base64 (appended) or raw (appended); the base64 header is
    encoded apart from the data unless joint."""
    hdt = "<u8" if header == "UInt64" else "<u4"
    conn = np.concatenate([np.asarray(c, np.int64) for _, c in cells]) if cells else np.zeros(0, np.int64)
    offs = np.cumsum([len(c) for _, c in cells]).astype(np.int32)
    types = np.array([t for t, _ in cells], np.uint8)
    arrays = [("Points", "Points", "Float64", points.astype("<f8").reshape(-1), 3),
              ("Cells", "connectivity", "Int64", conn.astype("<i8"), 1),
              ("Cells", "offsets", "Int32", offs.astype("<i4"), 1),
              ("Cells", "types", "UInt8", types, 1)]
    blocks, appended = {}, b""
    for sec, name, typ, a, nc in arrays:
        raw = a.tobytes()
        hdr = np.array([len(raw)], hdt).tobytes()
        if enc == "ascii":
            blocks[name] = ('format="ascii">' + " ".join(repr(float(v)) if typ.startswith("Float") else str(int(v))
                                                        for v in a) + "</DataArray>")
        elif enc == "binary":
            b = base64.b64encode(hdr + raw) if joint else base64.b64encode(hdr) + base64.b64encode(raw)
            blocks[name] = 'format="binary">\n' + b.decode() + "\n</DataArray>"
        else:
            blocks[name] = f'format="appended" offset="{len(appended)}"/>'
            if enc == "raw":
                appended += hdr + raw
            else:
                appended += base64.b64encode(hdr + raw) if joint else base64.b64encode(hdr) + base64.b64encode(raw)

    def da(name, typ, nc):
        comp = f' NumberOfComponents="{nc}"' if nc > 1 else ""
        return f'<DataArray type="{typ}" Name="{name}"{comp} {blocks[name]}\n'

    s = (f'<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
         f'header_type="{header}">\n<UnstructuredGrid>\n<Piece NumberOfPoints="{len(points)}" '
         f'NumberOfCells="{len(cells)}">\n<PointData>\n</PointData>\n<Points>\n' + da("Points", "Float64", 3)
         + "</Points>\n<Cells>\n" + da("connectivity", "Int64", 1) + da("offsets", "Int32", 1)
         + da("types", "UInt8", 1) + "</Cells>\n</Piece>\n</UnstructuredGrid>\n").encode()
    if enc in ("raw", "base64"):
        s += f'<AppendedData encoding="{enc}">\n_'.encode() + appended + b"\n</AppendedData>\n"
    return s + b"</VTKFile>\n"


def run_read(vtk_run, path):
    out = subprocess.run([vtk_run, "read", str(path)], check=True, capture_output=True, text=True).stdout.split()
    sd, cd, nv, nc = (int(x) for x in out[:4])
    coords = np.array([float(x) for x in out[4:4 + 3 * nv]]).reshape(nv, 3)
    cells = np.array([int(x) for x in out[4 + 3 * nv:4 + 3 * nv + nc]], np.uint64)
    return sd, cd, coords, cells


@pytest.mark.parametrize("enc,header,joint", [("ascii", "UInt64", False), ("binary", "UInt32", False),
                                              ("binary", "UInt64", True), ("base64", "UInt64", False),
                                              ("base64", "UInt32", True), ("raw", "UInt32", False),
                                              ("raw", "UInt64", False)])
def test_read_vtu_encodings(vtk_run, tmp_path, enc, header, joint):
    """The C++ reader and the Python one (ftk2_b200.vtk.read_vtu)."""
    from ftk2_b200 import vtk
    rng = np.random.default_rng(11)
    pts = rng.normal(size=(7, 3))
    # triangles kept; a line and a quad skipped, as VTK's cell types other
    # than triangles and tetrahedra are (utils/vtk.hpp:181-185)
    cells = [(5, [0, 1, 2]), (3, [2, 3]), (5, [1, 2, 3]), (9, [3, 4, 5, 6]), (5, [4, 5, 6])]
    p = tmp_path / "m.vtu"
    p.write_bytes(make_vtu(pts, cells, enc, header, joint))
    sd, cd, coords, got = run_read(vtk_run, p)
    assert (sd, cd) == (2, 2)
    assert np.array_equal(coords, pts)
    assert got.tolist() == [0, 1, 2, 1, 2, 3, 4, 5, 6]
    m = vtk.read_vtu(str(p))
    assert (m.spatial_dim, m.cell_dim) == (2, 2) and np.array_equal(m.coords, pts)
    assert m.cells.reshape(-1).tolist() == got.tolist() and m.cells.shape == (3, 3)

    tets = [(10, [0, 1, 2, 3]), (10, [1, 2, 3, 4])]
    p.write_bytes(make_vtu(pts, tets, enc, header, joint))
    sd, cd, coords, got = run_read(vtk_run, p)
    assert (sd, cd) == (3, 3) and got.tolist() == [0, 1, 2, 3, 1, 2, 3, 4]
    m = vtk.read_vtu(str(p))
    assert m.cell_dim == 3 and m.cells.tolist() == [[0, 1, 2, 3], [1, 2, 3, 4]] and np.array_equal(m.coords, pts)


def test_read_vtu_round_trip_and_missing_file(vtk_run, tmp_path):
    mesh, feats, conn = regular_case(np.random.default_rng(5))
    (tmp_path / "case.txt").write_text(case_text(mesh, feats, conn))
    subprocess.run([vtk_run, "write", str(tmp_path / "case.txt"), str(tmp_path)], check=True)
    xyz, _ = expected_points(mesh, feats)
    for f in ("all_bin.vtu", "dim3_ascii.vtu"):
        sd, cd, coords, got = run_read(vtk_run, tmp_path / f)
        assert np.array_equal(coords, xyz.astype(np.float64))
        ids, _, types = expected_cells(conn, {3} if "dim3" in f else {2, 3})
        # the cell dimension is that of the last triangle or tetrahedron read
        last = [t for t in types if t in (5, 10)][-1]
        assert got.tolist() == ids and cd == (3 if last == 10 else 2)
    r = subprocess.run([vtk_run, "read", str(tmp_path / "absent.vtu")], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "none"
    from ftk2_b200 import vtk
    assert vtk.read_vtu(str(tmp_path / "absent.vtu")) is None
    m = vtk.read_vtu(str(tmp_path / "all_bin.vtu"))  # mixed triangles and tetrahedra: flat ids
    assert np.array_equal(m.coords, xyz.astype(np.float64))
    assert m.cells.tolist() == expected_cells(conn, {2, 3})[0]
    (tmp_path / "z.vtu").write_text('<?xml version="1.0"?>\n<VTKFile type="UnstructuredGrid" '
                                    'compressor="vtkZLibDataCompressor">\n</VTKFile>\n')
    r = subprocess.run([vtk_run, "read", str(tmp_path / "z.vtu")], capture_output=True, text=True)
    assert r.returncode == 2 and "compressed" in r.stderr


# ---------------------------------------------------------------- Python writer

def _py_result(feats, conn):
    from types import SimpleNamespace
    return SimpleNamespace(simplices=np.array([f[1] for f in feats], np.uint64),
                           bary=np.array([f[2] for f in feats], np.float32),
                           track_id=np.array([f[3] for f in feats], np.uint64),
                           type=np.array([f[4] for f in feats], np.uint32),
                           scalar=np.array([f[5] for f in feats], np.float32), connectivity=conn)


def _py_mesh(mesh):
    from ftk2_b200 import api
    if mesh[0] == "regular":
        return api.RegularSimplicialMesh(mesh[1])
    _, sd, cd, coords, cells, nl = mesh
    return api.ExtrudedSimplicialMesh(api.UnstructuredSimplicialMesh(sd, cd, coords, cells), nl)


@pytest.mark.parametrize("name", ["regular_3d_t", "extruded_tri_2d", "extruded_tri_3d_coords"])
def test_python_writer_is_byte_identical(vtk_run, tmp_path, name):
    """ftk2_b200.vtk writes the same bytes as the C++ header for the same
    complex, in every form the driver writes."""
    from ftk2_b200 import vtk
    mesh, feats, conn = CASES[name](np.random.default_rng(len(name)))
    (tmp_path / "case.txt").write_text(case_text(mesh, feats, conn))
    subprocess.run([vtk_run, "write", str(tmp_path / "case.txt"), str(tmp_path)], check=True)
    r, m = _py_result(feats, conn), _py_mesh(mesh)
    py = tmp_path / "py"
    py.mkdir()
    vtk.write_complex_to_vtp(r, m, str(py / "all_ascii.vtp"), -1, True)
    vtk.write_complex_to_vtp(r, m, str(py / "all_bin.vtp"))
    vtk.write_complex_to_vtp(r, m, str(py / "dim1_ascii.vtp"), 1, True)
    vtk.write_complex_to_vtu(r, m, str(py / "all_ascii.vtu"), -1, True)
    vtk.write_complex_to_vtu(r, m, str(py / "all_bin.vtu"))
    vtk.write_complex_to_vtu(r, m, str(py / "dim0_bin.vtu"), 0)
    vtk.write_complex_to_vtu(r, m, str(py / "dim3_ascii.vtu"), 3, True)
    for f in sorted(os.listdir(py)):
        assert (py / f).read_bytes() == (tmp_path / f).read_bytes(), f


def test_python_writer_takes_extraction_results(tmp_path):
    """CPResult star edges become lines; ContourResult cells become
    triangles or tetrahedra."""
    from ftk2_b200 import api, vtk
    mesh = api.RegularSimplicialMesh([4, 4, 3])
    cp = api.CPResult(simplices=np.array([[0, 1, 5], [1, 5, 21]], np.uint64), lam=np.zeros((2, 3)),
                      bary=np.array([[0.5, 0.25, 0.25], [0.125, 0.5, 0.375]], np.float32),
                      track_id=np.array([0, 0], np.uint64), type=np.zeros(2, np.uint32),
                      cp_class=np.zeros(2, np.uint32), scalar=np.zeros(2, np.float32),
                      edges=np.array([[0, 1]], np.uint32), n_tracks=1)
    vtk.write_complex_to_vtp(cp, mesh, str(tmp_path / "cp.vtp"), use_ascii=True)
    got, piece = parse_vtk(tmp_path / "cp.vtp")
    assert got[("Lines", "connectivity")].tolist() == [0, 1] and piece["NumberOfLines"] == "1"
    # vertex 21 = (1, 1, 1): point 2 = 0.125*(1,0,0) + 0.5*(1,1,0) + 0.375*(1,1,1)
    assert got[("Points", "Points")].reshape(-1, 3)[1].tolist() == [1.0, 0.875, 0.375]
    lv = api.ContourResult(simplices=np.array([[0, 1], [1, 2], [0, 4]], np.uint64), lam=np.zeros((3, 2)),
                           bary=np.full((3, 2), 0.5, np.float32), track_id=np.zeros(3, np.uint64),
                           scalar=np.full(3, 0.5, np.float32), cells=np.array([[0, 1, 2]], np.uint32))
    vtk.write_complex_to_vtu(lv, mesh, str(tmp_path / "lv.vtu"))
    got, _ = parse_vtk(tmp_path / "lv.vtu")
    assert got[("Cells", "types")].tolist() == [5] and got[("Cells", "connectivity")].tolist() == [0, 1, 2]
    assert got[("PointData", "Type")].tolist() == [0, 0, 0]
