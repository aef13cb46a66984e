"""ctypes bridge to the CPU oracles (TEST INFRASTRUCTURE ONLY).

Loads oracle/_ref/libftk2ref.so (the reference engine, built from the
reference's own headers) and oracle/_build/libcporacle.so (our C restatement,
cp_oracle.c); oracle/_ref/libftk2refcuda.so (the reference's own GPU engine)
is loaded only to time the incumbent GPU path.  Only tests/, the smoke check and bench.py's CPU-baseline leg
import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libftk2ref.so")
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libftk2refcuda.so")
# the same engine with its worker pool sized 1: the level-set oracle
REF1T_LIB = os.path.join(HERE, "_ref", "libftk2ref1t.so")
ORC_LIB = os.path.join(HERE, "_build", "libcporacle.so")

MESH_REGULAR, MESH_EXTRUDED = 0, 1
F32, F64 = 0, 1
LAYOUT_MULTI, LAYOUT_SEPARATE, LAYOUT_PER_VERTEX = 0, 1, 2


class OrcMesh(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("ndims", C.c_int),
        ("local_dims", C.c_uint64 * 4), ("offset", C.c_uint64 * 4), ("global_dims", C.c_uint64 * 4),
        ("n_base_verts", C.c_uint64), ("base_coords", C.c_void_p),
        ("n_base_cells", C.c_uint64), ("base_cells", C.c_void_p),
        ("base_cell_dim", C.c_int), ("n_layers", C.c_uint64),
    ]


class OrcField(C.Structure):
    _fields_ = [
        ("dtype", C.c_int), ("ncomp", C.c_int), ("layout", C.c_int),
        ("comp", C.c_void_p * 4), ("nd", C.c_int), ("dims", C.c_uint64 * 4),
        ("scalar", C.c_void_p), ("scalar_nd", C.c_int), ("scalar_dims", C.c_uint64 * 4),
        ("sos_q", C.c_double), ("n_threads", C.c_int),
        ("fiber", C.c_int), ("fiber_thr", C.c_double * 2),
    ]


class OrcResult(C.Structure):
    _fields_ = [
        ("m", C.c_int), ("n", C.c_uint64),
        ("simplices", C.POINTER(C.c_uint64)), ("bary", C.POINTER(C.c_float)),
        ("lambda_", C.POINTER(C.c_double)), ("track_id", C.POINTER(C.c_uint64)),
        ("type", C.POINTER(C.c_uint32)), ("scalar", C.POINTER(C.c_float)),
        ("n_edges", C.c_uint64), ("edges", C.POINTER(C.c_uint32)),
        ("n_tested", C.c_uint64), ("cp_class", C.POINTER(C.c_uint32)),
        ("cell_dim", C.c_int), ("n_cells", C.c_uint64), ("cells", C.POINTER(C.c_uint32)),
    ]


@dataclass
class CPResult:
    """Flattened FeatureComplex: features in canonical order plus edges."""
    simplices: np.ndarray   # (n, m+1) uint64
    bary: np.ndarray        # (n, m+1) float32
    lam: np.ndarray         # (n, m+1) float64
    track_id: np.ndarray    # (n,) uint64
    type: np.ndarray        # (n,) uint32
    scalar: np.ndarray      # (n,) float32
    edges: np.ndarray       # (e, 2) uint32
    n_tested: int = 0
    cp_class: np.ndarray | None = None  # (n,) uint32, restatement on regular meshes only
    cells: np.ndarray | None = None     # (c, 3) uint32 star-fan triangles, restated fiber surfaces only


_libs: dict[str, C.CDLL] = {}


def _load(path: str, prefix: str) -> C.CDLL:
    if path not in _libs:
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run __graft_entry__.build())")
        lib = C.CDLL(path)
        run = getattr(lib, prefix + "_run")
        run.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcField), C.POINTER(OrcResult)]
        run.restype = C.c_int
        free = getattr(lib, prefix + "_free")
        free.argtypes = [C.POINTER(OrcResult)]
        free.restype = None
        _libs[path] = lib
    return _libs[path]


def classify_jacobian(J: np.ndarray) -> int:
    """Class code of one spatial Jacobian (m x m, J[j][a] = d v_j / d x_a) by
    the restatement's FP64 classifier."""
    lib = _load(ORC_LIB, "cporacle")
    J = np.ascontiguousarray(J, dtype=np.float64)
    fn = lib.cporacle_classify_jacobian
    fn.argtypes = [C.c_int, C.POINTER(C.c_double)]
    fn.restype = C.c_uint32
    return int(fn(J.shape[0], J.ctypes.data_as(C.POINTER(C.c_double))))


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def make_regular_mesh(local_dims, offset=None, global_dims=None) -> OrcMesh:
    nd = len(local_dims)
    offset = list(offset) if offset is not None else [0] * nd
    global_dims = list(global_dims) if global_dims is not None else list(local_dims)
    m = OrcMesh()
    m.kind = MESH_REGULAR
    m.ndims = nd
    for i in range(nd):
        m.local_dims[i] = int(local_dims[i])
        m.offset[i] = int(offset[i])
        m.global_dims[i] = int(global_dims[i])
    return m


def make_extruded_mesh(coords: np.ndarray, cells: np.ndarray, n_layers: int, keep: list) -> OrcMesh:
    coords = np.ascontiguousarray(coords, dtype=np.float64)
    cells = np.ascontiguousarray(cells, dtype=np.uint64)
    keep += [coords, cells]
    m = OrcMesh()
    m.kind = MESH_EXTRUDED
    m.ndims = cells.shape[1]  # base cell dim + 1 (time)
    m.n_base_verts = coords.shape[0]
    m.base_coords = coords.ctypes.data
    m.n_base_cells = cells.shape[0]
    m.base_cells = cells.ctypes.data
    m.base_cell_dim = cells.shape[1] - 1
    m.n_layers = int(n_layers)
    return m


def make_field(arrays, layout: int, ncomp: int, scalar=None, sos_q: float = 1e6,
               n_threads: int = 0, keep: list | None = None, fiber_thr=None) -> OrcField:
    """arrays: MULTI -> one numpy array whose memory is [M, dims...] Fortran
    (C-order shape (..reversed dims.., M)); SEPARATE / PER_VERTEX -> list of M
    arrays (C-order shape reversed dims).  fiber_thr = (a, b): the
    restatement runs FiberPredicate<T> with those thresholds (ncomp 2)."""
    keep = keep if keep is not None else []
    f = OrcField()
    first = arrays if layout == LAYOUT_MULTI else arrays[0]
    f.dtype = F64 if first.dtype == np.float64 else F32
    f.ncomp = ncomp
    f.layout = layout
    if layout == LAYOUT_MULTI:
        a = np.ascontiguousarray(arrays)
        keep.append(a)
        f.comp[0] = a.ctypes.data
        dims = a.shape[::-1][1:]
    else:
        dims = None
        for j, a in enumerate(arrays):
            a = np.ascontiguousarray(a)
            keep.append(a)
            f.comp[j] = a.ctypes.data
            dims = a.shape[::-1]
    f.nd = len(dims)
    for i, d in enumerate(dims):
        f.dims[i] = int(d)
    if scalar is not None:
        s = np.ascontiguousarray(scalar)
        keep.append(s)
        f.scalar = s.ctypes.data
        f.scalar_nd = s.ndim
        for i, d in enumerate(s.shape[::-1]):
            f.scalar_dims[i] = int(d)
    f.sos_q = float(sos_q)
    f.n_threads = int(n_threads)
    if fiber_thr is not None:
        f.fiber = 1
        f.fiber_thr[0], f.fiber_thr[1] = float(fiber_thr[0]), float(fiber_thr[1])
    return f


def _run(path: str, prefix: str, mesh: OrcMesh, field: OrcField) -> CPResult:
    lib = _load(path, prefix)
    res = OrcResult()
    rc = getattr(lib, prefix + "_run")(C.byref(mesh), C.byref(field), C.byref(res))
    if rc != 0:
        raise RuntimeError(f"{prefix}_run failed with status {rc}")
    try:
        n, k, e = int(res.n), int(res.m) + 1, int(res.n_edges)

        def arr(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        return CPResult(
            simplices=arr(res.simplices, n * k, np.uint64).reshape(n, k),
            bary=arr(res.bary, n * k, np.float32).reshape(n, k),
            lam=arr(res.lambda_, n * k, np.float64).reshape(n, k),
            track_id=arr(res.track_id, n, np.uint64),
            type=arr(res.type, n, np.uint32),
            scalar=arr(res.scalar, n, np.float32),
            edges=arr(res.edges, 2 * e, np.uint32).reshape(e, 2),
            n_tested=int(res.n_tested),
            cp_class=arr(res.cp_class, n, np.uint32) if res.cp_class else None,
            cells=arr(res.cells, int(res.n_cells) * (int(res.cell_dim) + 1), np.uint32).reshape(
                int(res.n_cells), int(res.cell_dim) + 1) if res.cells else None,
        )
    finally:
        getattr(lib, prefix + "_free")(C.byref(res))


def run_reference(mesh: OrcMesh, field: OrcField) -> CPResult:
    """The reference's own engine (execute + get_complex)."""
    return _run(REF_LIB, "ftk2ref", mesh, field)


def _ref_cuda() -> C.CDLL:
    lib = _load(REF_CUDA_LIB, "ftk2refcuda")
    if not hasattr(lib, "_typed"):
        lib.ftk2refcuda_run.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcField), C.POINTER(OrcResult),
                                        C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.ftk2refcuda_time_kernel.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcField), C.c_int,
                                                C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.ftk2refcuda_time_kernel.restype = C.c_int
        lib._typed = True
    return lib


def run_reference_cuda(mesh: OrcMesh, field: OrcField):
    """The reference's own GPU engine: execute_cuda + get_complex on separate
    component arrays of a regular mesh (engine.hpp:273-425).  Returns the
    complex and the wall times of execute_cuda and get_complex in ms.  The
    reference ends the process on a CUDA error, so callers run this in a
    child process."""
    lib = _ref_cuda()
    res = OrcResult()
    ex, cx = C.c_double(0), C.c_double(0)
    rc = lib.ftk2refcuda_run(C.byref(mesh), C.byref(field), C.byref(res), C.byref(ex), C.byref(cx))
    if rc != 0:
        raise RuntimeError(f"ftk2refcuda_run failed with status {rc}")
    try:
        n, k, e = int(res.n), int(res.m) + 1, int(res.n_edges)

        def arr(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        out = CPResult(
            simplices=arr(res.simplices, n * k, np.uint64).reshape(n, k),
            bary=arr(res.bary, n * k, np.float32).reshape(n, k),
            lam=np.full((n, k), np.nan),
            track_id=arr(res.track_id, n, np.uint64),
            type=arr(res.type, n, np.uint32),
            scalar=arr(res.scalar, n, np.float32),
            edges=arr(res.edges, 2 * e, np.uint32).reshape(e, 2),
        )
    finally:
        lib.ftk2refcuda_free(C.byref(res))
    return out, ex.value, cx.value


def time_reference_cuda_kernel(mesh: OrcMesh, field: OrcField, reps: int = 3):
    """Mean CUDA-event time (ms) of the reference's extraction kernel
    (cuda_engine.hpp:366-493) over `reps` launches, and its node count."""
    lib = _ref_cuda()
    ms, nn = C.c_double(0), C.c_int(0)
    rc = lib.ftk2refcuda_time_kernel(C.byref(mesh), C.byref(field), int(reps), C.byref(ms), C.byref(nn))
    if rc != 0:
        raise RuntimeError(f"ftk2refcuda_time_kernel failed with status {rc}")
    return ms.value, int(nn.value)


class OrcConn(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_uint64), ("idx", C.POINTER(C.c_uint32))]


def run_reference_contour(mesh: OrcMesh, field: OrcField, threshold: float, one_thread: bool = True):
    """The reference's own engine with ContourPredicate<T> on a regular mesh
    (execute + get_complex): the features (mesh edges) and the manifold cells,
    an (n, dim+1) array of feature indices.  By default the one-worker build:
    with several workers the reference's patching races on its node map."""
    lib = _load(REF1T_LIB if one_thread else REF_LIB, "ftk2ref")
    fn = lib.ftk2ref_run_contour
    fn.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcField), C.c_double, C.POINTER(OrcResult), C.POINTER(OrcConn)]
    fn.restype = C.c_int
    lib.ftk2ref_free_conn.argtypes = [C.POINTER(OrcConn)]
    res, conn = OrcResult(), OrcConn()
    rc = fn(C.byref(mesh), C.byref(field), float(threshold), C.byref(res), C.byref(conn))
    if rc != 0:
        raise RuntimeError(f"ftk2ref_run_contour failed with status {rc}")
    try:
        n, k = int(res.n), int(conn.dim) + 1

        def arr(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        out = CPResult(
            simplices=arr(res.simplices, 2 * n, np.uint64).reshape(n, 2),
            bary=arr(res.bary, 2 * n, np.float32).reshape(n, 2),
            lam=arr(res.lambda_, 2 * n, np.float64).reshape(n, 2),
            track_id=arr(res.track_id, n, np.uint64),
            type=arr(res.type, n, np.uint32),
            scalar=arr(res.scalar, n, np.float32),
            edges=np.zeros((0, 2), dtype=np.uint32),
        )
        cells = arr(conn.idx, int(conn.n) * k, np.uint32).reshape(-1, k)
    finally:
        lib.ftk2ref_free(C.byref(res))
        lib.ftk2ref_free_conn(C.byref(conn))
    return out, cells


def run_reference_fiber(mesh: OrcMesh, field: OrcField, thresholds, one_thread: bool = False) -> CPResult:
    """The reference's own engine with FiberPredicate<T> on a regular 2D+t
    mesh: field.comp[0], comp[1] are the two scalar arrays."""
    lib = _load(REF1T_LIB if one_thread else REF_LIB, "ftk2ref")
    fn = lib.ftk2ref_run_fiber
    fn.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcField), C.POINTER(C.c_double), C.POINTER(OrcResult)]
    fn.restype = C.c_int
    thr = (C.c_double * 2)(float(thresholds[0]), float(thresholds[1]))
    res = OrcResult()
    rc = fn(C.byref(mesh), C.byref(field), thr, C.byref(res))
    if rc != 0:
        raise RuntimeError(f"ftk2ref_run_fiber failed with status {rc}")
    try:
        n, e = int(res.n), int(res.n_edges)

        def arr(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        return CPResult(
            simplices=arr(res.simplices, 3 * n, np.uint64).reshape(n, 3),
            bary=arr(res.bary, 3 * n, np.float32).reshape(n, 3),
            lam=arr(res.lambda_, 3 * n, np.float64).reshape(n, 3),
            track_id=arr(res.track_id, n, np.uint64),
            type=arr(res.type, n, np.uint32),
            scalar=arr(res.scalar, n, np.float32),
            edges=arr(res.edges, 2 * e, np.uint32).reshape(e, 2),
        )
    finally:
        lib.ftk2ref_free(C.byref(res))


def run_reference_fiber_surface(mesh: OrcMesh, field: OrcField, thresholds, one_thread: bool = False):
    """The reference's own engine with FiberPredicate<T> on a regular 3D+t
    mesh or an extruded mesh over tets: the triangle features and the
    star-fan triangles of get_complex, an (n, 3) array of feature indices.
    one_thread: the engine built to run its loops on one worker (on extruded
    meshes the triangles found while patching are numbered in the order the
    workers meet them, which only one worker makes deterministic)."""
    lib = _load(REF1T_LIB if one_thread else REF_LIB, "ftk2ref")
    fn = lib.ftk2ref_run_fiber_surface
    fn.argtypes = [C.POINTER(OrcMesh), C.POINTER(OrcField), C.POINTER(C.c_double), C.POINTER(OrcResult),
                   C.POINTER(OrcConn)]
    fn.restype = C.c_int
    lib.ftk2ref_free_conn.argtypes = [C.POINTER(OrcConn)]
    thr = (C.c_double * 2)(float(thresholds[0]), float(thresholds[1]))
    res, conn = OrcResult(), OrcConn()
    rc = fn(C.byref(mesh), C.byref(field), thr, C.byref(res), C.byref(conn))
    if rc != 0:
        raise RuntimeError(f"ftk2ref_run_fiber_surface failed with status {rc}")
    try:
        n = int(res.n)

        def arr(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        out = CPResult(
            simplices=arr(res.simplices, 3 * n, np.uint64).reshape(n, 3),
            bary=arr(res.bary, 3 * n, np.float32).reshape(n, 3),
            lam=arr(res.lambda_, 3 * n, np.float64).reshape(n, 3),
            track_id=arr(res.track_id, n, np.uint64),
            type=arr(res.type, n, np.uint32),
            scalar=arr(res.scalar, n, np.float32),
            edges=np.zeros((0, 2), dtype=np.uint32),
        )
        cells = arr(conn.idx, int(conn.n) * 3, np.uint32).reshape(-1, 3)
    finally:
        lib.ftk2ref_free(C.byref(res))
        lib.ftk2ref_free_conn(C.byref(conn))
    return out, cells


def run_restatement(mesh: OrcMesh, field: OrcField) -> CPResult:
    """Our exact C restatement of the same algorithm."""
    return _run(ORC_LIB, "cporacle", mesh, field)


class OrcTracked(C.Structure):
    _fields_ = [
        ("dtype", C.c_int), ("m", C.c_int), ("dims", C.c_uint64 * 3), ("nt", C.c_uint64),
        ("vec", C.c_void_p), ("n_attr", C.c_int),
        ("attr_data", C.c_void_p * 16), ("attr_nd", C.c_int * 16), ("attr_dims", (C.c_uint64 * 6) * 16),
        ("attr_magnitude", C.c_int * 16), ("attr_component", C.c_int * 16),
    ]


def run_reference_tracked(vec: np.ndarray, attrs=()):
    """The reference high-level caller's critical-point flow: its engine on
    ExtrudedSimplicialMesh(RegularSimplicialMesh(spatial dims), nt - 1) with
    the multicomponent array ``vec`` (C-order shape (nt, [nz,] ny, nx, m), the
    bytes of a Fortran [m, nx, ny, (nz,) nt] array) and attributes given as
    (array, magnitude, component) with arrays in C order (reversed Fortran
    shape).  Returns (CPResult, attributes (n, 16) float32)."""
    lib = _load(REF_LIB, "ftk2ref")
    if not hasattr(lib, "_tracked_bound"):
        lib.ftk2ref_run_tracked.argtypes = [C.POINTER(OrcTracked), C.POINTER(OrcResult),
                                            C.POINTER(C.POINTER(C.c_float))]
        lib.ftk2ref_run_tracked.restype = C.c_int
        lib.ftk2ref_free_attrs.argtypes = [C.POINTER(C.c_float)]
        lib._tracked_bound = True
    vec = np.ascontiguousarray(vec)
    m = vec.shape[-1]
    t = OrcTracked()
    t.dtype = F64 if vec.dtype == np.float64 else F32
    t.m = m
    sp = vec.shape[1:-1][::-1]  # Fortran spatial dims
    for i, d in enumerate(sp):
        t.dims[i] = int(d)
    t.nt = int(vec.shape[0])
    t.vec = vec.ctypes.data
    keep = [vec]
    t.n_attr = len(attrs)
    for a, (arr, mag, comp) in enumerate(attrs):
        arr = np.ascontiguousarray(arr, dtype=vec.dtype)
        keep.append(arr)
        t.attr_data[a] = arr.ctypes.data
        fd = arr.shape[::-1]
        t.attr_nd[a] = len(fd)
        for i, d in enumerate(fd):
            t.attr_dims[a][i] = int(d)
        t.attr_magnitude[a] = int(bool(mag))
        t.attr_component[a] = int(comp)
    res = OrcResult()
    out = C.POINTER(C.c_float)()
    rc = lib.ftk2ref_run_tracked(C.byref(t), C.byref(res), C.byref(out))
    if rc != 0:
        raise RuntimeError(f"ftk2ref_run_tracked failed with status {rc}")
    try:
        n, k, e = int(res.n), int(res.m) + 1, int(res.n_edges)

        def arr_(ptr, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

        r = CPResult(
            simplices=arr_(res.simplices, n * k, np.uint64).reshape(n, k),
            bary=arr_(res.bary, n * k, np.float32).reshape(n, k),
            lam=arr_(res.lambda_, n * k, np.float64).reshape(n, k),
            track_id=arr_(res.track_id, n, np.uint64),
            type=arr_(res.type, n, np.uint32),
            scalar=arr_(res.scalar, n, np.float32),
            edges=arr_(res.edges, 2 * e, np.uint32).reshape(e, 2),
            n_tested=0, cp_class=None)
        at = arr_(out, n * 16, np.float32).reshape(n, 16)
        return r, at
    finally:
        lib.ftk2ref_free(C.byref(res))
        lib.ftk2ref_free_attrs(out)
