"""Time-slab sharding on the GPU: the slabs of a field extracted one after
another on one B200 (ftk2_b200.sharded.extract_local) and merged give exactly
the one-call result on the whole mesh (features, barycentrics, tracks,
edges), for 2D+t and 3D+t fields and several slab counts."""
import numpy as np
import pytest

from ftk2_b200 import api, sharded
from ftk2_b200 import synthetic as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [2, 3, 5])
def test_sharded_2d_equals_one_call(ctx, n):
    v = S.analytic_2d(64, 64, 10)
    dims = [64, 64, 10]
    keep: list = []
    whole = ctx.extract(api.regular_mesh_desc(dims), api.field_desc(v, api.LAYOUT_MULTICOMPONENT, 2, keep=keep),
                        api.params(1e6))
    got = sharded.extract_local(ctx, dims, v, 2, n, api.params(1e6))
    assert len(whole.track_id) > 0
    assert np.array_equal(got.simplices, whole.simplices)
    assert np.array_equal(got.lam.view(np.uint64), whole.lam.view(np.uint64))
    assert np.array_equal(got.track_id, whole.track_id)
    assert np.array_equal(got.edges, whole.edges)


@pytest.mark.parametrize("n", [2, 4])
def test_sharded_3d_equals_one_call(ctx, n):
    torch = pytest.importorskip("torch")
    from ftk2_b200 import generate
    dims = [64, 64, 64, 8]
    dev = generate.gaussian_field_device((64, 64, 64), 8, seed=1234, n_blobs=32, dtype=torch.float64)
    keep: list = []
    whole = ctx.extract(api.regular_mesh_desc(dims),
                        api.field_desc(dev, api.LAYOUT_MULTICOMPONENT, 3, keep=keep), api.params(2.0 ** 20))
    got = sharded.extract_local(ctx, dims, dev, 3, n, api.params(2.0 ** 20))
    assert len(whole.track_id) > 100
    assert np.array_equal(got.simplices, whole.simplices)
    assert np.array_equal(got.lam.view(np.uint64), whole.lam.view(np.uint64))
    assert np.array_equal(got.track_id, whole.track_id)
    assert np.array_equal(got.edges, whole.edges)
