"""Time-slab sharding (ftk2_b200/sharded.py) on the CPU: the merge of slab
results equals the result of the whole mesh, in one process for 1 to 4 slabs
and across world_size 2 and 3 gloo process groups.  Each slab is extracted by
the restatement (oracle/cp_oracle.c) here, standing in for the rank's GPU;
the GPU form is tests/test_sharded_gpu.py."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from ftk2_b200 import api, sharded
from ftk2_b200 import synthetic as S
from oracle import bridge


def orc_extract(field, m, q):
    def run(mesh_desc, t0=None, t1=None):
        nd = mesh_desc.ndims
        om = bridge.make_regular_mesh([mesh_desc.local_dims[i] for i in range(nd)],
                                      [mesh_desc.offset[i] for i in range(nd)],
                                      [mesh_desc.global_dims[i] for i in range(nd)])
        keep: list = []
        r = bridge.run_restatement(om, bridge.make_field(field, bridge.LAYOUT_MULTI, m, sos_q=q, keep=keep))
        n = len(r.track_id)
        return api.CPResult(simplices=r.simplices, lam=r.lam, bary=r.bary, track_id=r.track_id, type=r.type,
                            cp_class=r.cp_class if r.cp_class is not None else np.zeros(n, np.uint32),
                            scalar=r.scalar, edges=r.edges, n_tracks=int(len(set(r.track_id.tolist()))))
    return run


FIELDS = {
    "2d_analytic": lambda: (S.analytic_2d(40, 36, 9), [40, 36, 9], 2, 1e6),
    "3d_gauss": lambda: (S.gaussian_sum_gradient((18, 16, 14), 7, seed=3, n_blobs=9, sigma=(2, 5)),
                         [18, 16, 14, 7], 3, 2.0 ** 20),
}


def same(a, b):
    assert np.array_equal(a.simplices, b.simplices)
    assert np.array_equal(a.lam.view(np.uint64), b.lam.view(np.uint64))
    assert np.array_equal(a.bary.view(np.uint32), b.bary.view(np.uint32))
    assert np.array_equal(a.track_id, b.track_id)
    assert np.array_equal(a.edges, b.edges)


def test_slab_bounds_cover_and_share_one_step():
    for nt in (2, 3, 9, 16):
        for n in (1, 2, 3, 4, 8):
            b = sharded.slab_bounds(nt, n)
            assert b[0][0] == 0 and b[-1][1] == nt - 1
            for (a0, a1), (c0, c1) in zip(b, b[1:]):
                assert a1 == c0 and a0 < a1
            assert len(b) == min(n, nt - 1)


@pytest.mark.parametrize("name", list(FIELDS))
@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_merge_of_slabs_equals_whole_mesh(name, n):
    field, dims, m, q = FIELDS[name]()
    run = orc_extract(field, m, q)
    whole = run(api.regular_mesh_desc(dims))
    assert len(whole.track_id) > 0
    bounds = sharded.slab_bounds(dims[-1], n)
    parts = [run(sharded.slab_mesh(dims, t0, t1)) for t0, t1 in bounds]
    same(sharded.merge(parts, bounds, dims), whole)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, name, out_path):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        field, dims, m, q = FIELDS[name]()
        res = sharded.extract_distributed(dims, None, m, extractor=lambda mesh, t0, t1: orc_extract(field, m, q)(mesh))
        if rank == 0:
            np.savez(out_path, simplices=res.simplices, lam=res.lam, bary=res.bary, track_id=res.track_id,
                     edges=res.edges)
        else:
            assert res is None
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", list(FIELDS))
def test_distributed_gloo_ranks(tmp_path, world, name):
    import torch.multiprocessing as mp
    out = str(tmp_path / "merged.npz")
    mp.start_processes(_rank_main, args=(world, _free_port(), name, out), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    field, dims, m, q = FIELDS[name]()
    whole = orc_extract(field, m, q)(api.regular_mesh_desc(dims))
    assert np.array_equal(got["simplices"], whole.simplices)
    assert np.array_equal(got["lam"].view(np.uint64), whole.lam.view(np.uint64))
    assert np.array_equal(got["track_id"], whole.track_id)
    assert np.array_equal(got["edges"], whole.edges)
