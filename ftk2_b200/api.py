"""Python binding of the C ABI in include/ftk2b.h (ctypes), plus a mirror of
the reference's engine interface for this path:

    mesh   = RegularSimplicialMesh([nx, ny, nt])              # mesh.hpp:256-265
    pred   = CriticalPointPredicate(2, vector_var_name="v")   # predicate.hpp:49-64
    engine = SimplicialEngine(mesh, pred)                     # engine.hpp:84-85
    engine.execute({"v": array})                              # engine.hpp:96-99
    fc     = engine.get_complex()                             # engine.hpp:822-996

Arrays follow the reference's ndarray memory layout (Fortran order, first
index fastest): a numpy array of C-order shape (nt, ny, nx, M) holds the
reference's [M, nx, ny, nt] multicomponent array.  CUDA tensors (torch) are
passed by device pointer without a copy.

There is no CPU fallback: without the built library or a CUDA device every
call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libftk2b.so")
# the build with the device bounds checks compiled in (FTK2B_CHECKED=1 loads it)
CHECKED_LIB_PATH = os.path.join(HERE, "_lib", "checked", "libftk2b.so")

# enums of include/ftk2b.h
OK, INVALID_ARG, OOM, CUDA_ERROR, TIMEOUT, OVERFLOW_RETRY, NO_DEVICE, UNSUPPORTED, BUSY, INTERNAL = range(10)
STATUS_NAMES = ["OK", "INVALID_ARG", "OOM", "CUDA_ERROR", "TIMEOUT", "OVERFLOW_RETRY", "NO_DEVICE",
                "UNSUPPORTED", "BUSY", "INTERNAL"]
MESH_REGULAR, MESH_EXTRUDED = 0, 1
F32, F64 = 0, 1
LAYOUT_MULTICOMPONENT, LAYOUT_SEPARATE, LAYOUT_PER_VERTEX = 0, 1, 2
HOST, DEVICE = 0, 1
PRECISION_EXACT, PRECISION_REFINED = 0, 1
OPT_FEATURE_CAPACITY, OPT_TIME_CHUNK, OPT_DISABLE_TMA, OPT_USE_GRAPHS = 1, 2, 3, 4
INFO_LAST_TMA = 100
INFO_LAST_CULL_MODE = 101
INFO_LAST_BATCH_TIME_CHUNK = 102
INFO_LAST_CANDIDATES = 103
INFO_LAST_TESTED = 104
OPT_BLOCKING_SYNC = 5
OPT_CULL_MODE = 6
OPT_BATCH_TIME_CHUNK = 7
OPT_TEST_STALL_POLLS = 8
CLASS_NAMES = ["none", "degenerate", "source", "sink", "saddle", "spiral_source", "spiral_sink",
               "center"]


class Ftk2bError(RuntimeError):
    def __init__(self, status: int, msg: str):
        name = STATUS_NAMES[status] if 0 <= status < len(STATUS_NAMES) else str(status)
        super().__init__(f"{name}: {msg}")
        self.status = status


class MeshDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("ndims", C.c_int),
        ("local_dims", C.c_uint64 * 4), ("offset", C.c_uint64 * 4), ("global_dims", C.c_uint64 * 4),
        ("n_base_verts", C.c_uint64), ("base_cells", C.c_void_p), ("n_base_cells", C.c_uint64),
        ("base_cell_dim", C.c_int), ("n_layers", C.c_uint64),
    ]


class FieldDesc(C.Structure):
    _fields_ = [
        ("dtype", C.c_int), ("ncomp", C.c_int), ("layout", C.c_int), ("location", C.c_int),
        ("comp", C.c_void_p * 3), ("nd", C.c_int), ("dims", C.c_uint64 * 4),
        ("scalar", C.c_void_p), ("scalar_nd", C.c_int), ("scalar_dims", C.c_uint64 * 4),
    ]


class CPParams(C.Structure):
    _fields_ = [("sos_q", C.c_double), ("precision", C.c_int), ("want_edges", C.c_int),
                ("classify", C.c_int)]


class CPResultC(C.Structure):
    _fields_ = [
        ("m", C.c_int), ("n_features", C.c_uint64),
        ("simplices", C.POINTER(C.c_uint64)), ("lambda_", C.POINTER(C.c_double)),
        ("barycentric", C.POINTER(C.c_float)), ("track_id", C.POINTER(C.c_uint64)),
        ("type", C.POINTER(C.c_uint32)), ("cp_class", C.POINTER(C.c_uint32)),
        ("scalar", C.POINTER(C.c_float)),
        ("n_edges", C.c_uint64), ("edges", C.POINTER(C.c_uint32)),
        ("n_tracks", C.c_uint64), ("n_simplices", C.c_uint64), ("device_ms", C.c_double),
    ]


class RequestC(C.Structure):
    _fields_ = [("kind", C.c_int), ("mesh", MeshDesc), ("field", FieldDesc), ("params", CPParams),
                ("stream", C.c_uint64)]


class RequestStatsC(C.Structure):
    _fields_ = [("status", C.c_int), ("slot", C.c_int), ("queue_ms", C.c_double), ("run_ms", C.c_double),
                ("latency_ms", C.c_double), ("n_features", C.c_uint64), ("n_simplices", C.c_uint64),
                ("phase_ms", C.c_double * 4)]


class ServerStatsC(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("rejected", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("max_ms", C.c_double), ("mean_ms", C.c_double), ("elapsed_s", C.c_double),
                ("simplices", C.c_uint64), ("hbm_budget", C.c_uint64), ("hbm_reserved_peak", C.c_uint64),
                ("max_in_flight", C.c_int)]


class ContourResultC(C.Structure):
    _fields_ = [
        ("n_features", C.c_uint64), ("simplices", C.POINTER(C.c_uint64)), ("lambda_", C.POINTER(C.c_double)),
        ("barycentric", C.POINTER(C.c_float)), ("track_id", C.POINTER(C.c_uint64)),
        ("scalar", C.POINTER(C.c_float)), ("cell_dim", C.c_int), ("n_cells", C.c_uint64),
        ("cells", C.POINTER(C.c_uint32)), ("n_tracks", C.c_uint64), ("n_simplices", C.c_uint64),
        ("device_ms", C.c_double),
    ]


class FiberSurfaceResultC(C.Structure):
    _fields_ = [
        ("n_features", C.c_uint64), ("simplices", C.POINTER(C.c_uint64)), ("lambda_", C.POINTER(C.c_double)),
        ("barycentric", C.POINTER(C.c_float)), ("track_id", C.POINTER(C.c_uint64)),
        ("scalar", C.POINTER(C.c_float)), ("n_cells", C.c_uint64), ("cells", C.POINTER(C.c_uint32)),
        ("n_tracks", C.c_uint64), ("n_simplices", C.c_uint64), ("device_ms", C.c_double),
    ]


REQ_EXTRACT, REQ_STREAM_PUSH = 0, 1


ATTR_VALUE, ATTR_COMPONENT, ATTR_MAGNITUDE = 0, 1, 2


class AttributeDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("component", C.c_int), ("slot", C.c_int), ("location", C.c_int),
                ("data", C.c_void_p), ("nd", C.c_int), ("dims", C.c_uint64 * 6)]


# name -> (restype, argtypes); every symbol include/ftk2b.h declares
SIGNATURES = {
    "ftk2b_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "ftk2b_ctx_destroy": (None, [C.c_void_p]),
    "ftk2b_last_error": (C.c_char_p, [C.c_void_p]),
    "ftk2b_ctx_stream": (C.c_void_p, [C.c_void_p]),
    "ftk2b_cp_params_default": (CPParams, []),
    "ftk2b_ctx_set_option": (C.c_int, [C.c_void_p, C.c_int, C.c_int64]),
    "ftk2b_ctx_get_option": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]),
    "ftk2b_mesh_simplex_count": (C.c_uint64, [C.POINTER(MeshDesc), C.c_int]),
    "ftk2b_cp_extract": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                   C.POINTER(CPParams), C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_cp_result_free": (None, [C.POINTER(CPResultC)]),
    "ftk2b_contour_extract": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc), C.c_double,
                                        C.c_double, C.POINTER(C.POINTER(ContourResultC))]),
    "ftk2b_contour_result_free": (None, [C.POINTER(ContourResultC)]),
    "ftk2b_fiber_extract": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                      C.POINTER(C.c_double), C.c_double, C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_fiber_surface_extract": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                              C.POINTER(C.c_double), C.c_double,
                                              C.POINTER(C.POINTER(FiberSurfaceResultC))]),
    "ftk2b_fiber_surface_result_free": (None, [C.POINTER(FiberSurfaceResultC)]),
    "ftk2b_cp_run": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                               C.POINTER(CPParams), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "ftk2b_cp_fetch": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_ctx_last_phases": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "ftk2b_ctx_last_timing": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_uint64)]),
    "ftk2b_stream_checkpoint": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint64)]),
    "ftk2b_stream_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(C.c_void_p)]),
    "ftk2b_stream_open": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                    C.POINTER(CPParams), C.POINTER(C.c_void_p)]),
    "ftk2b_stream_push": (C.c_int, [C.c_void_p, C.POINTER(FieldDesc), C.POINTER(C.c_uint64)]),
    "ftk2b_stream_result": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_stream_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                    C.POINTER(C.c_double)]),
    "ftk2b_stream_close": (None, [C.c_void_p]),
    "ftk2b_server_create": (C.c_int, [C.c_int, C.c_int, C.c_uint64, C.c_int, C.POINTER(C.c_void_p)]),
    "ftk2b_server_stream_open": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                           C.POINTER(CPParams), C.POINTER(C.c_uint64)]),
    "ftk2b_server_submit": (C.c_int, [C.c_void_p, C.POINTER(RequestC), C.POINTER(C.c_uint64)]),
    "ftk2b_server_warm": (C.c_int, [C.c_void_p, C.POINTER(RequestC)]),
    "ftk2b_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(C.POINTER(CPResultC)),
                                    C.POINTER(RequestStatsC)]),
    "ftk2b_server_stream_result": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_server_stream_close": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ftk2b_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStatsC)]),
    "ftk2b_server_last_error": (C.c_char_p, [C.c_void_p]),
    "ftk2b_server_destroy": (None, [C.c_void_p]),
    "ftk2b_cp_attributes": (C.c_int, [C.c_void_p, C.POINTER(MeshDesc), C.POINTER(C.c_uint64), C.c_uint32,
                                      C.POINTER(AttributeDesc), C.c_void_p]),
    "ftk2b_cp_run_batch": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                     C.POINTER(CPParams), C.POINTER(C.c_uint64)]),
    "ftk2b_cp_fetch_batch": (C.c_int, [C.c_void_p, C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_cp_extract_batch": (C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(MeshDesc), C.POINTER(FieldDesc),
                                         C.POINTER(CPParams), C.POINTER(C.POINTER(CPResultC))]),
    "ftk2b_cp_features_noalloc": (C.c_int, [C.POINTER(MeshDesc), C.POINTER(FieldDesc), C.c_double,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                            C.c_void_p, C.POINTER(C.c_uint64)]),
}

_lib: Optional[C.CDLL] = None


def load_library(path: Optional[str] = None) -> C.CDLL:
    """Load libftk2b.so and bind every exported entry point (the checked build
    when the environment sets FTK2B_CHECKED=1).  Raises if the library has
    not been built: the path has no CPU fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = CHECKED_LIB_PATH if os.environ.get("FTK2B_CHECKED") == "1" else LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library not built: {path} (run __graft_entry__.build())")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


# ---------------------------------------------------------------------------
# descriptors


def regular_mesh_desc(local_dims, offset=None, global_dims=None) -> MeshDesc:
    nd = len(local_dims)
    offset = list(offset) if offset is not None else [0] * nd
    global_dims = list(global_dims) if global_dims is not None else list(local_dims)
    m = MeshDesc()
    m.kind = MESH_REGULAR
    m.ndims = nd
    for i in range(nd):
        m.local_dims[i] = int(local_dims[i])
        m.offset[i] = int(offset[i])
        m.global_dims[i] = int(global_dims[i])
    return m


def extruded_mesh_desc(n_base_verts: int, cells: np.ndarray, n_layers: int, keep: list) -> MeshDesc:
    cells = np.ascontiguousarray(cells, dtype=np.uint64)
    keep.append(cells)
    m = MeshDesc()
    m.kind = MESH_EXTRUDED
    m.ndims = cells.shape[1]
    m.n_base_verts = int(n_base_verts)
    m.base_cells = cells.ctypes.data
    m.n_base_cells = cells.shape[0]
    m.base_cell_dim = cells.shape[1] - 1
    m.n_layers = int(n_layers)
    return m


def _is_torch_cuda(a) -> bool:
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


def _ptr_dtype_shape(a, keep: list):
    if _is_torch_cuda(a):
        if not a.is_contiguous():
            raise ValueError("device arrays must be contiguous")
        import torch
        dt = {torch.float64: F64, torch.float32: F32}.get(a.dtype)
        if dt is None:
            raise ValueError(f"unsupported dtype {a.dtype}")
        keep.append(a)
        return a.data_ptr(), dt, tuple(a.shape), DEVICE
    a = np.ascontiguousarray(a)
    if a.dtype not in (np.float64, np.float32):
        raise ValueError(f"unsupported dtype {a.dtype}")
    keep.append(a)
    return a.ctypes.data, (F64 if a.dtype == np.float64 else F32), a.shape, HOST


def field_desc(arrays, layout: int, ncomp: int, scalar=None, keep: Optional[list] = None) -> FieldDesc:
    """MULTICOMPONENT: one array of C-order shape (..reversed dims.., M).
    SEPARATE / PER_VERTEX: a sequence of M arrays of C-order shape reversed dims."""
    keep = keep if keep is not None else []
    f = FieldDesc()
    f.ncomp = ncomp
    f.layout = layout
    if layout == LAYOUT_MULTICOMPONENT:
        p, dt, shape, loc = _ptr_dtype_shape(arrays, keep)
        if shape[-1] != ncomp:
            raise ValueError("multicomponent arrays carry the component axis last (fastest)")
        f.comp[0] = p
        dims = tuple(shape[::-1][1:])
    else:
        dims = None
        loc = dt = None
        for j, a in enumerate(arrays):
            p, dtj, shape, locj = _ptr_dtype_shape(a, keep)
            f.comp[j] = p
            dims = tuple(shape[::-1])
            dt, loc = dtj, locj
    f.dtype, f.location = dt, loc
    f.nd = len(dims)
    for i, d in enumerate(dims):
        f.dims[i] = int(d)
    if scalar is not None:
        p, _, shape, _ = _ptr_dtype_shape(scalar, keep)
        f.scalar = p
        f.scalar_nd = len(shape)
        for i, d in enumerate(shape[::-1]):
            f.scalar_dims[i] = int(d)
    return f


def params(sos_q: float = 1e6, precision: int = PRECISION_EXACT, want_edges: bool = True,
           classify: bool = False) -> CPParams:
    p = CPParams()
    p.sos_q = float(sos_q)
    p.precision = int(precision)
    p.want_edges = int(bool(want_edges))
    p.classify = int(bool(classify))
    return p


@dataclass
class CPResult:
    """Flattened FeatureComplex (complex.hpp:14-58) of one extraction."""
    simplices: np.ndarray      # (n, m+1) uint64 sorted vertex ids, canonical order
    lam: np.ndarray            # (n, m+1) float64 barycentrics
    bary: np.ndarray           # (n, m+1) float32 as FeatureElement stores them
    track_id: np.ndarray       # (n,) uint64
    type: np.ndarray           # (n,) uint32 (0)
    cp_class: np.ndarray       # (n,) uint32
    scalar: np.ndarray         # (n,) float32
    edges: np.ndarray          # (e, 2) uint32
    n_tracks: int = 0
    n_simplices: int = 0
    device_ms: float = 0.0


def _result_from_c(r: CPResultC) -> CPResult:
    n, k, e = int(r.n_features), int(r.m) + 1, int(r.n_edges)

    def arr(ptr, count, dt):
        if count == 0:
            return np.zeros(0, dtype=dt)
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

    return CPResult(
        simplices=arr(r.simplices, n * k, np.uint64).reshape(n, k),
        lam=arr(r.lambda_, n * k, np.float64).reshape(n, k),
        bary=arr(r.barycentric, n * k, np.float32).reshape(n, k),
        track_id=arr(r.track_id, n, np.uint64),
        type=arr(r.type, n, np.uint32),
        cp_class=arr(r.cp_class, n, np.uint32),
        scalar=arr(r.scalar, n, np.float32),
        edges=arr(r.edges, 2 * e, np.uint32).reshape(e, 2),
        n_tracks=int(r.n_tracks), n_simplices=int(r.n_simplices), device_ms=float(r.device_ms))


@dataclass
class ContourResult:
    """Flattened FeatureComplex of a level-set (ContourPredicate) or
    fiber-surface (FiberPredicate on 3D+t) extraction: features are mesh
    edges or triangles, cells the manifold cells of get_complex.  The arrays
    are views of the library's result memory, freed with the last of them."""
    simplices: np.ndarray      # (n, m+1) uint64 vertex ids, simplex order (m = 1 edges, 2 triangles)
    lam: np.ndarray            # (n, m+1) float64 barycentrics in the field precision
    bary: np.ndarray           # (n, m+1) float32 as FeatureElement stores them
    track_id: np.ndarray       # (n,) uint64
    scalar: np.ndarray         # (n,) float32 (the threshold)
    cells: np.ndarray          # (c, cell_dim + 1) uint32 feature indices
    n_tracks: int = 0
    n_simplices: int = 0
    device_ms: float = 0.0


class _CResultOwner:
    """Owns one result the library allocated (its host arrays are plain heap
    or huge-page memory, independent of the context) and frees it with the
    library's free function once the last numpy view of it is gone.  Level
    sets return gigabytes; the views spare the host a second copy."""

    __slots__ = ("_free", "_ptr")

    def __init__(self, free, ptr):
        self._free, self._ptr = free, ptr

    def __del__(self):
        if self._ptr is not None and self._ptr:
            self._free(self._ptr)
        self._ptr = None


def _view(owner: _CResultOwner, ptr, count: int, dt) -> np.ndarray:
    """A writable numpy view of count elements at ptr that keeps owner alive."""
    if count == 0 or not ptr:
        return np.zeros(0, dtype=dt)
    buf = (C.c_uint8 * (count * np.dtype(dt).itemsize)).from_address(C.cast(ptr, C.c_void_p).value)
    buf._owner = owner
    return np.frombuffer(buf, dtype=dt)


def _contour_from_c(r: ContourResultC, owner: _CResultOwner) -> ContourResult:
    n, k, c = int(r.n_features), int(r.cell_dim) + 1, int(r.n_cells)
    return ContourResult(
        simplices=_view(owner, r.simplices, 2 * n, np.uint64).reshape(n, 2),
        lam=_view(owner, r.lambda_, 2 * n, np.float64).reshape(n, 2),
        bary=_view(owner, r.barycentric, 2 * n, np.float32).reshape(n, 2),
        track_id=_view(owner, r.track_id, n, np.uint64),
        scalar=_view(owner, r.scalar, n, np.float32),
        cells=_view(owner, r.cells, k * c, np.uint32).reshape(c, k),
        n_tracks=int(r.n_tracks), n_simplices=int(r.n_simplices), device_ms=float(r.device_ms))


def _fiber_surface_from_c(r: FiberSurfaceResultC, owner: _CResultOwner) -> ContourResult:
    n, c = int(r.n_features), int(r.n_cells)
    return ContourResult(
        simplices=_view(owner, r.simplices, 3 * n, np.uint64).reshape(n, 3),
        lam=_view(owner, r.lambda_, 3 * n, np.float64).reshape(n, 3),
        bary=_view(owner, r.barycentric, 3 * n, np.float32).reshape(n, 3),
        track_id=_view(owner, r.track_id, n, np.uint64),
        scalar=_view(owner, r.scalar, n, np.float32),
        cells=_view(owner, r.cells, 3 * c, np.uint32).reshape(c, 3),
        n_tracks=int(r.n_tracks), n_simplices=int(r.n_simplices), device_ms=float(r.device_ms))


class Context:
    """One ftk2b_ctx: a device, a CUDA stream and reusable device buffers."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.ftk2b_ctx_create(int(device), C.byref(h))
        if st != OK:
            raise Ftk2bError(st, "ftk2b_ctx_create failed")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ftk2b_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def stream_ptr(self) -> int:
        return int(self.lib.ftk2b_ctx_stream(self.h) or 0)

    def set_option(self, option: int, value: int):
        self._check(self.lib.ftk2b_ctx_set_option(self.h, int(option), int(value)))

    def get_option(self, option: int) -> int:
        v = C.c_int64()
        self._check(self.lib.ftk2b_ctx_get_option(self.h, int(option), C.byref(v)))
        return int(v.value)

    def last_error(self) -> str:
        return (self.lib.ftk2b_last_error(self.h) or b"").decode()

    def _check(self, st: int):
        if st != OK:
            raise Ftk2bError(st, self.last_error())

    def extract(self, mesh: MeshDesc, field: FieldDesc, prm: Optional[CPParams] = None) -> CPResult:
        prm = prm or params()
        out = C.POINTER(CPResultC)()
        self._check(self.lib.ftk2b_cp_extract(self.h, C.byref(mesh), C.byref(field), C.byref(prm),
                                              C.byref(out)))
        try:
            self._last_n = int(out.contents.n_features)
            return _result_from_c(out.contents)
        finally:
            self.lib.ftk2b_cp_result_free(out)

    def contour(self, mesh: MeshDesc, field, threshold: float = 0.0, sos_q: float = 1e6) -> ContourResult:
        """Level sets (ContourPredicate<T>) on a regular mesh.  field: a
        FieldDesc (ncomp 1, LAYOUT_SEPARATE), or the scalar array itself (numpy
        or torch, C-order of reversed Fortran shape)."""
        keep: list = []
        if not isinstance(field, FieldDesc):
            field = field_desc([field], LAYOUT_SEPARATE, 1, keep=keep)
        out = C.POINTER(ContourResultC)()
        self._check(self.lib.ftk2b_contour_extract(self.h, C.byref(mesh), C.byref(field), float(threshold),
                                                   float(sos_q), C.byref(out)))
        return _contour_from_c(out.contents, _CResultOwner(self.lib.ftk2b_contour_result_free, out))

    def fiber(self, mesh: MeshDesc, field: FieldDesc, thresholds=(0.0, 0.0), sos_q: float = 1e6) -> CPResult:
        """Fibers (FiberPredicate<T>) of two scalar fields on a regular 2D+t
        mesh; field carries the two arrays as its two components."""
        thr = (C.c_double * 2)(float(thresholds[0]), float(thresholds[1]))
        out = C.POINTER(CPResultC)()
        self._check(self.lib.ftk2b_fiber_extract(self.h, C.byref(mesh), C.byref(field), thr, float(sos_q),
                                                 C.byref(out)))
        try:
            self._last_n = int(out.contents.n_features)
            return _result_from_c(out.contents)
        finally:
            self.lib.ftk2b_cp_result_free(out)

    def fiber_surface(self, mesh: MeshDesc, field: FieldDesc, thresholds=(0.0, 0.0),
                      sos_q: float = 1e6) -> ContourResult:
        """Fiber surfaces (FiberPredicate<T>) of two scalar fields on a regular
        3D+t mesh or an extruded mesh over tets (per-vertex arrays): triangle
        features (simplices (n, 3)) and the star-fan triangles of get_complex
        (cells (c, 3))."""
        thr = (C.c_double * 2)(float(thresholds[0]), float(thresholds[1]))
        out = C.POINTER(FiberSurfaceResultC)()
        self._check(self.lib.ftk2b_fiber_surface_extract(self.h, C.byref(mesh), C.byref(field), thr,
                                                         float(sos_q), C.byref(out)))
        return _fiber_surface_from_c(out.contents, _CResultOwner(self.lib.ftk2b_fiber_surface_result_free, out))

    def run(self, mesh: MeshDesc, field: FieldDesc, prm: Optional[CPParams] = None):
        """Device pipeline only; results stay on the device until fetch()."""
        prm = prm or params()
        n, ne = C.c_uint64(), C.c_uint64()
        self._check(self.lib.ftk2b_cp_run(self.h, C.byref(mesh), C.byref(field), C.byref(prm),
                                          C.byref(n), C.byref(ne)))
        self._last_n = int(n.value)
        return int(n.value), int(ne.value)

    def last_timing(self):
        """(extraction kernel ms, whole pipeline ms, kernels launched so far)."""
        x, t, k = C.c_double(), C.c_double(), C.c_uint64()
        self._check(self.lib.ftk2b_ctx_last_timing(self.h, C.byref(x), C.byref(t), C.byref(k)))
        return float(x.value), float(t.value), int(k.value)

    def fetch(self) -> CPResult:
        out = C.POINTER(CPResultC)()
        self._check(self.lib.ftk2b_cp_fetch(self.h, C.byref(out)))
        try:
            return _result_from_c(out.contents)
        finally:
            self.lib.ftk2b_cp_result_free(out)


    def attributes(self, mesh: MeshDesc, attrs, base_grid_dims=None) -> np.ndarray:
        """Attributes at the features of the last run (ftk2b_cp_attributes).
        attrs: list of (kind, array, component, slot); arrays in C order
        (reversed Fortran shape), host numpy or device torch.  Returns
        (n_features, 16) float32."""
        n = self._last_n
        keep = []
        descs = (AttributeDesc * max(1, len(attrs)))()
        for i, (kind, arr, comp, slot) in enumerate(attrs):
            d = descs[i]
            d.kind, d.component, d.slot = int(kind), int(comp), int(slot)
            if hasattr(arr, "data_ptr"):
                d.location, d.data = DEVICE, arr.data_ptr()
                shape = tuple(arr.shape)
            else:
                arr = np.ascontiguousarray(arr)
                d.location, d.data = HOST, arr.ctypes.data
                shape = arr.shape
            keep.append(arr)
            d.nd = len(shape)
            for q, v in enumerate(shape[::-1]):
                d.dims[q] = int(v)
        out = np.zeros((max(n, 1), 16), dtype=np.float32)
        bg = None
        if base_grid_dims is not None:
            bg = (C.c_uint64 * 3)(*[int(x) for x in base_grid_dims] + [0] * (3 - len(base_grid_dims)))
        self._check(self.lib.ftk2b_cp_attributes(self.h, C.byref(mesh), bg, len(attrs), descs,
                                                 out.ctypes.data))
        return out[:n]

    # ---- batches (ftk2b_cp_*_batch): n fields of uneven sizes in one pass
    @staticmethod
    def _batch_arrays(meshes, fields, prms):
        n = len(meshes)
        if len(fields) != n or (prms is not None and len(prms) != n):
            raise ValueError("meshes, fields and params must have the same length")
        ma = (MeshDesc * n)(*meshes)
        fa = (FieldDesc * n)(*fields)
        pa = (CPParams * n)(*prms) if prms is not None else None
        return n, ma, fa, pa

    def run_batch(self, meshes, fields, prms=None) -> int:
        """Device pipeline of a batch; results stay on the device until
        fetch_batch().  Returns the number of features of the whole batch."""
        n, ma, fa, pa = self._batch_arrays(meshes, fields, prms)
        tot = C.c_uint64()
        self._check(self.lib.ftk2b_cp_run_batch(self.h, n, ma, fa, pa, C.byref(tot)))
        self._batch_n = n
        return int(tot.value)

    def fetch_batch(self) -> list:
        n = getattr(self, "_batch_n", 0)
        outs = (C.POINTER(CPResultC) * max(n, 1))()
        self._check(self.lib.ftk2b_cp_fetch_batch(self.h, outs))
        try:
            return [_result_from_c(outs[i].contents) for i in range(n)]
        finally:
            for i in range(n):
                self.lib.ftk2b_cp_result_free(outs[i])

    def extract_batch(self, meshes, fields, prms=None) -> list:
        """One result per field, each identical to extract() on that field."""
        n, ma, fa, pa = self._batch_arrays(meshes, fields, prms)
        outs = (C.POINTER(CPResultC) * n)()
        self._check(self.lib.ftk2b_cp_extract_batch(self.h, n, ma, fa, pa, outs))
        try:
            return [_result_from_c(outs[i].contents) for i in range(n)]
        finally:
            for i in range(n):
                self.lib.ftk2b_cp_result_free(outs[i])


class Stream:
    """A time stream on a context (ftk2b_stream_*): push one timestep at a
    time; result() equals Context.extract on all timesteps pushed so far."""

    def __init__(self, ctx: Context, mesh: MeshDesc, template: FieldDesc, prm: Optional[CPParams] = None):
        self.ctx = ctx
        self.lib = ctx.lib
        prm = prm or params()
        h = C.c_void_p()
        ctx._check(self.lib.ftk2b_stream_open(ctx.h, C.byref(mesh), C.byref(template), C.byref(prm),
                                              C.byref(h)))
        self.h = h

    def push(self, step: FieldDesc) -> int:
        n = C.c_uint64()
        self.ctx._check(self.lib.ftk2b_stream_push(self.h, C.byref(step), C.byref(n)))
        return int(n.value)

    def result(self) -> CPResult:
        out = C.POINTER(CPResultC)()
        self.ctx._check(self.lib.ftk2b_stream_result(self.h, C.byref(out)))
        try:
            return _result_from_c(out.contents)
        finally:
            self.lib.ftk2b_cp_result_free(out)

    def info(self):
        """(timesteps pushed, features so far, device ms of the last push)."""
        t, n, ms = C.c_uint64(), C.c_uint64(), C.c_double()
        self.ctx._check(self.lib.ftk2b_stream_info(self.h, C.byref(t), C.byref(n), C.byref(ms)))
        return int(t.value), int(n.value), float(ms.value)

    def checkpoint(self) -> bytes:
        """The stream's whole state as bytes (ftk2b_stream_checkpoint)."""
        n = C.c_uint64()
        self.ctx._check(self.lib.ftk2b_stream_checkpoint(self.h, None, C.byref(n)))
        buf = C.create_string_buffer(max(1, n.value))
        self.ctx._check(self.lib.ftk2b_stream_checkpoint(self.h, buf, C.byref(n)))
        return buf.raw[:n.value]

    @classmethod
    def restore(cls, ctx: Context, blob: bytes) -> "Stream":
        """A stream on ctx resumed from checkpoint() bytes (ftk2b_stream_restore)."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        data = C.create_string_buffer(bytes(blob), len(blob))
        ctx._check(self.lib.ftk2b_stream_restore(ctx.h, data, len(blob), C.byref(h)))
        self.h = h
        return self

    def close(self):
        if getattr(self, "h", None):
            self.lib.ftk2b_stream_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Server:
    """Request loop over worker slots (ftk2b_server_*): extraction requests and
    stream pushes are admitted in arrival order as workers and HBM budget
    free up; their device work overlaps across slots.  Arrays referenced by a
    request must stay alive until its wait() returns (pass `keep`)."""

    def __init__(self, device: int = 0, n_slots: int = 4, hbm_budget: int = 0, queue_limit: int = 0):
        self.lib = load_library()
        h = C.c_void_p()
        st = self.lib.ftk2b_server_create(int(device), int(n_slots), int(hbm_budget), int(queue_limit),
                                          C.byref(h))
        if st != OK:
            raise Ftk2bError(st, "ftk2b_server_create failed")
        self.h = h
        self._keep: dict = {}

    def _check(self, st: int):
        if st != OK:
            raise Ftk2bError(st, (self.lib.ftk2b_server_last_error(self.h) or b"").decode())

    def open_stream(self, mesh: MeshDesc, template: FieldDesc, prm: Optional[CPParams] = None) -> int:
        sid = C.c_uint64()
        self._check(self.lib.ftk2b_server_stream_open(self.h, C.byref(mesh), C.byref(template),
                                                      C.byref(prm or params()), C.byref(sid)))
        return int(sid.value)

    def _submit(self, req: RequestC, keep) -> int:
        t = C.c_uint64()
        self._check(self.lib.ftk2b_server_submit(self.h, C.byref(req), C.byref(t)))
        self._keep[int(t.value)] = keep
        return int(t.value)

    def submit_extract(self, mesh: MeshDesc, field: FieldDesc, prm: Optional[CPParams] = None,
                       keep=None) -> int:
        r = RequestC()
        r.kind = REQ_EXTRACT
        r.mesh = mesh
        r.field = field
        r.params = prm or params()
        return self._submit(r, keep)

    def warm(self, mesh: MeshDesc, field: FieldDesc, prm: Optional[CPParams] = None):
        """Runs one extraction on every slot (buffers and graphs sized for it)."""
        r = RequestC()
        r.kind = REQ_EXTRACT
        r.mesh = mesh
        r.field = field
        r.params = prm or params()
        self._check(self.lib.ftk2b_server_warm(self.h, C.byref(r)))

    def submit_push(self, stream_id: int, step: FieldDesc, keep=None) -> int:
        r = RequestC()
        r.kind = REQ_STREAM_PUSH
        r.field = step
        r.params = params()
        r.stream = int(stream_id)
        return self._submit(r, keep)

    def wait(self, ticket: int, timeout: float = -1.0, want_result: bool = True):
        """(CPResult or None, stats dict); raises on a failed request."""
        out = C.POINTER(CPResultC)()
        stc = RequestStatsC()
        st = self.lib.ftk2b_server_wait(self.h, int(ticket), float(timeout),
                                        C.byref(out) if want_result else None, C.byref(stc))
        self._keep.pop(int(ticket), None)
        self._check(st)
        res = None
        if want_result and out:
            try:
                res = _result_from_c(out.contents)
            finally:
                self.lib.ftk2b_cp_result_free(out)
        stats = {k: getattr(stc, k) for k, _ in RequestStatsC._fields_}
        stats["phase_ms"] = list(stc.phase_ms)
        return res, stats

    def stream_result(self, stream_id: int) -> CPResult:
        out = C.POINTER(CPResultC)()
        self._check(self.lib.ftk2b_server_stream_result(self.h, int(stream_id), C.byref(out)))
        try:
            return _result_from_c(out.contents)
        finally:
            self.lib.ftk2b_cp_result_free(out)

    def close_stream(self, stream_id: int):
        self._check(self.lib.ftk2b_server_stream_close(self.h, int(stream_id)))

    def stats(self) -> dict:
        s = ServerStatsC()
        self._check(self.lib.ftk2b_server_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in ServerStatsC._fields_}

    def close(self):
        if getattr(self, "h", None):
            self.lib.ftk2b_server_destroy(self.h)
            self.h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def simplex_count(mesh: MeshDesc, m: int) -> int:
    return int(load_library().ftk2b_mesh_simplex_count(C.byref(mesh), int(m)))


# ---------------------------------------------------------------------------
# mirror of the reference's engine interface


class RegularSimplicialMesh:
    """RegularSimplicialMesh(dims, offset, global_dims) (mesh.hpp:256-265)."""

    def __init__(self, dims: Sequence[int], offset: Optional[Sequence[int]] = None,
                 global_dims: Optional[Sequence[int]] = None):
        self.dims = list(dims)
        self.offset = list(offset) if offset else [0] * len(dims)
        self.global_dims = list(global_dims) if global_dims else list(dims)

    def get_total_dimension(self) -> int:
        return len(self.dims)

    def get_spatial_dimension(self) -> int:
        return len(self.dims)

    def vertex_coordinates(self, ids: np.ndarray) -> np.ndarray:
        """get_vertex_coordinates (mesh.hpp:374-378) of many ids: the global
        grid index per axis, (..., nd) float64."""
        ids = np.asarray(ids, dtype=np.uint64)
        out = np.empty(ids.shape + (len(self.global_dims),), np.float64)
        r = ids.copy()
        for i, d in enumerate(self.global_dims):
            out[..., i] = (r % np.uint64(d)).astype(np.float64)
            r //= np.uint64(d)
        return out

    def desc(self, keep: list) -> MeshDesc:
        return regular_mesh_desc(self.dims, self.offset, self.global_dims)


class UnstructuredSimplicialMesh:
    """UnstructuredSimplicialMesh(spatial_dim, cell_dim, coords, cells)
    (unstructured_mesh.hpp:16-76); coords are (n, 3), cells (n_cells, cell_dim+1)."""

    def __init__(self, spatial_dim: int, cell_dim: int, coords: np.ndarray, cells: np.ndarray):
        self.spatial_dim = spatial_dim
        self.cell_dim = cell_dim
        self.coords = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
        self.cells = np.asarray(cells, dtype=np.uint64).reshape(-1, cell_dim + 1)

    def get_total_dimension(self) -> int:
        return self.cell_dim

    def get_spatial_dimension(self) -> int:
        return self.spatial_dim

    def vertex_coordinates(self, ids: np.ndarray) -> np.ndarray:
        """get_vertex_coordinates (unstructured_mesh.hpp:100-107): the first
        spatial_dim stored coordinates, (..., spatial_dim) float64."""
        return self.coords[np.asarray(ids, dtype=np.int64)][..., :self.spatial_dim]


class ExtrudedSimplicialMesh:
    """ExtrudedSimplicialMesh(base, n_layers) (mesh.hpp:542-562)."""

    def __init__(self, base: UnstructuredSimplicialMesh, n_layers: int):
        self.base = base
        self.n_layers = int(n_layers)

    def get_total_dimension(self) -> int:
        return self.base.get_total_dimension() + 1

    def get_spatial_dimension(self) -> int:
        return self.base.get_spatial_dimension()

    def vertex_coordinates(self, ids: np.ndarray) -> np.ndarray:
        """get_vertex_coordinates (mesh.hpp:714-720): the base vertex's
        coordinates, then the layer of vertex id s + t * n_base_vertices."""
        ids = np.asarray(ids, dtype=np.uint64)
        S = np.uint64(self.base.coords.shape[0])
        base = self.base.vertex_coordinates((ids % S).astype(np.int64))
        return np.concatenate([base, (ids // S).astype(np.float64)[..., None]], axis=-1)

    def desc(self, keep: list) -> MeshDesc:
        return extruded_mesh_desc(self.base.coords.shape[0], self.base.cells, self.n_layers, keep)


@dataclass
class CriticalPointPredicate:
    """CriticalPointPredicate<M,T> knobs (predicate.hpp:22-64)."""
    M: int
    vector_var_name: str = ""
    var_names: list = field(default_factory=list)
    scalar_var_name: str = ""
    use_multicomponent: bool = True
    sos_q: float = 1e6
    precision: int = PRECISION_EXACT
    classify: bool = False


@dataclass
class ContourPredicate:
    """ContourPredicate<T> knobs (predicate.hpp:135-183): level sets of one
    scalar field."""
    var_name: str = ""
    threshold: float = 0.0
    sos_q: float = 1e6


@dataclass
class FiberPredicate:
    """FiberPredicate<T> knobs (predicate.hpp:341-362): fibers of two scalar
    fields (points of 2D+t meshes, surfaces of 3D+t meshes)."""
    var_names: list = field(default_factory=lambda: ["", ""])
    thresholds: tuple = (0.0, 0.0)
    sos_q: float = 1e6


class SimplicialEngine:
    """SimplicialEngine<T, Predicate> (engine.hpp:79-996) on the GPU, for
    CriticalPointPredicate, ContourPredicate and FiberPredicate."""

    def __init__(self, mesh, pred, ctx: Optional[Context] = None):
        self.mesh = mesh
        self.pred = pred
        self.ctx = ctx or Context(0)
        self._result = None

    def _field(self, data: dict, keep: list) -> FieldDesc:
        p = self.pred
        scalar = data[p.scalar_var_name] if p.scalar_var_name else None
        if p.use_multicomponent and p.vector_var_name:
            return field_desc(data[p.vector_var_name], LAYOUT_MULTICOMPONENT, p.M, scalar, keep)
        arrays = [data[n] for n in p.var_names[:p.M]]
        layout = LAYOUT_PER_VERTEX if isinstance(self.mesh, ExtrudedSimplicialMesh) else LAYOUT_SEPARATE
        return field_desc(arrays, layout, p.M, scalar, keep)

    def execute(self, data: dict, var_names=None):
        keep: list = []
        mesh = self.mesh.desc(keep)
        p = self.pred
        if isinstance(p, ContourPredicate):
            name = var_names[0] if var_names else p.var_name
            fld = field_desc([data[name]], LAYOUT_SEPARATE, 1, keep=keep)
            self._result = self.ctx.contour(mesh, fld, p.threshold, p.sos_q)
            return
        if isinstance(p, FiberPredicate):
            names = list(var_names[:2]) if var_names and len(var_names) >= 2 else list(p.var_names[:2])
            layout = LAYOUT_PER_VERTEX if isinstance(self.mesh, ExtrudedSimplicialMesh) else LAYOUT_SEPARATE
            fld = field_desc([data[n] for n in names], layout, 2, keep=keep)
            if self.mesh.get_total_dimension() == 4:
                self._result = self.ctx.fiber_surface(mesh, fld, p.thresholds, p.sos_q)
            else:
                self._result = self.ctx.fiber(mesh, fld, p.thresholds, p.sos_q)
            return
        fld = self._field(data, keep)
        prm = params(p.sos_q, p.precision, True, p.classify)
        self._result = self.ctx.extract(mesh, fld, prm)

    execute_cuda = execute

    def get_complex(self):
        """CPResult (critical points, 2D+t fibers) or ContourResult (level
        sets, fiber surfaces)."""
        if self._result is None:
            raise RuntimeError("execute() has not run")
        return self._result
