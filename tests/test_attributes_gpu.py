"""ftk2b_cp_attributes on regular meshes, against a step-by-step numpy
restatement of the reference's attribute recording (engine.hpp:1143-1199):
per feature, the sum over its vertices of the stored float barycentric times
the source value there, accumulated in the field precision operation by
operation, then rounded to float.  Multicomponent sources are read as one
component or as the magnitude; other arrays at the vertex's grid coordinates
minus the mesh offset, or by vertex id when 1-D."""
import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S

pytestmark = pytest.mark.gpu


def vertex_coords(vid, gdims):
    c = []
    for d in gdims:
        c.append(int(vid % d))
        vid //= d
    return c


def fort(a, idx):
    """ndarray f(i0, i1, ...) on a C-order array of reversed Fortran shape."""
    dims = a.shape[::-1]
    o, mul = 0, 1
    for k, i in enumerate(idx):
        o += i * mul
        mul *= dims[k] if k < len(dims) else 1
    return a.reshape(-1)[o]


def expected(res, kind, arr, comp, gdims, offset, T):
    n, k = res.simplices.shape
    out = np.zeros(n, dtype=np.float32)
    for i in range(n):
        acc = T(0)
        for v in range(k):
            vid = int(res.simplices[i, v])
            c = vertex_coords(vid, gdims)
            if kind == api.ATTR_COMPONENT:
                val = T(fort(arr, [comp] + c))
            elif kind == api.ATTR_MAGNITUDE:
                sq = T(0)
                for cc in range(arr.shape[-1]):
                    cv = T(fort(arr, [cc] + c))
                    sq = T(sq + T(cv * cv))
                val = T(np.sqrt(sq))
            elif arr.ndim == 1:
                val = T(arr[vid])
            else:
                val = T(fort(arr, [a - b for a, b in zip(c, offset)]))
            acc = T(acc + T(T(res.bary[i, v]) * val))
        out[i] = np.float32(acc)
    return out


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_attributes_match_reference_rules(ctx, dtype):
    T = dtype
    gd = [30, 28, 6]
    g = S.gaussian_sum_gradient((30, 28), 6, seed=9, n_blobs=14, dtype=dtype, sigma=(2, 6))  # (6, 28, 30, 2)
    local, off = [24, 20, 5], [3, 4, 1]
    keep: list = []
    mesh = api.regular_mesh_desc(local, off, gd)
    res = ctx.extract(mesh, api.field_desc(g, api.LAYOUT_MULTICOMPONENT, 2, keep=keep), api.params(1e6))
    assert len(res.track_id) > 0
    rng = np.random.default_rng(2)
    scal = rng.standard_normal((6, 28, 30)).astype(dtype)           # Fortran [30, 28, 6]
    pv = rng.standard_normal(30 * 28 * 6).astype(dtype)              # per vertex id
    specs = [(api.ATTR_COMPONENT, g, 1, 0), (api.ATTR_MAGNITUDE, g, -1, 3), (api.ATTR_VALUE, scal, -1, 5),
             (api.ATTR_VALUE, pv, -1, 15)]
    got = ctx.attributes(mesh, specs)
    assert got.shape == (len(res.track_id), 16)
    for kind, arr, comp, slot in specs:
        want = expected(res, kind, arr, comp, gd, off, T)
        assert np.array_equal(got[:, slot].view(np.uint32), want.view(np.uint32)), (kind, slot)
    untouched = [s for s in range(16) if s not in (0, 3, 5, 15)]
    assert not got[:, untouched].any()
