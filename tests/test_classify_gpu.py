"""GPU critical-point classification (a field the reference does not fill:
type = 0 always, predicate.hpp:80) against the oracle's FP64 classifier.

* every feature of the regular golden and medium cases: the CUDA class equals
  the oracle's class exactly, while type stays 0 like the reference;
* near-singular linear fields whose Jacobian determinant is lost in FP32
  (1 + 1e-8 rounds to 1): the FP64 fallback decides, so the class is source
  for det > 0 and saddle for det < 0, exactly as the oracle says.
"""
import numpy as np
import pytest

from ftk2_b200 import api
from ftk2_b200 import synthetic as S
from oracle import bridge
import cases

pytestmark = pytest.mark.gpu

SOURCE, SADDLE = 2, 4


def run_both(ctx, case):
    keep: list = []
    mesh, fld = cases.gpu_inputs(case, keep)
    g = ctx.extract(mesh, fld, api.params(case.sos_q, classify=True))
    om, of = cases.oracle_inputs(case, keep)
    o = bridge.run_restatement(om, of)
    return g, o


def _cases():
    out = [cases.GOLDEN_CASES[n]() for n in sorted(cases.GOLDEN_CASES) if not n.startswith("extruded")]
    g = S.gaussian_sum_gradient((40, 36, 32), 5, seed=7, n_blobs=24, dtype=np.float32, noise=1e-3,
                                sigma=(3, 8))
    out.append(cases.Case("g3d_f32_noise", "regular", 3, cases.MULTI, g, 2.0 ** 20, [40, 36, 32, 5]))
    g = S.gaussian_sum_gradient((200, 150), 12, seed=3, n_blobs=40, sigma=(3, 9))
    out.append(cases.Case("g2d_f64", "regular", 2, cases.MULTI, g, 1e6, [200, 150, 12]))
    return out


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c.name)
def test_classes_match_oracle(ctx, case):
    g, o = run_both(ctx, case)
    assert np.array_equal(g.simplices, o.simplices)
    assert o.cp_class is not None and len(o.cp_class) == len(g.cp_class)
    assert np.array_equal(g.cp_class, o.cp_class)
    assert np.all(g.type == 0)
    assert np.all((g.cp_class >= 1) & (g.cp_class <= 7))


def linear_field(A, dims, nt, centre, drift):
    """v(x, t) = A (x - c(t)) on the grid, multicomponent layout."""
    m = len(dims)
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in dims[::-1]], indexing="ij")
    X = np.stack(grids[::-1], -1)  # (..reversed dims.., m): X[..., a] = coordinate a
    out = np.empty((nt,) + tuple(dims[::-1]) + (m,), dtype=np.float64)
    for t in range(nt):
        c = np.asarray(centre) + t * np.asarray(drift)
        out[t] = (X - c) @ np.asarray(A).T
    return out


@pytest.mark.parametrize("m,delta,want", [(2, 1e-8, SOURCE), (2, -1e-8, SADDLE),
                                          (3, 1e-8, SOURCE), (3, -1e-8, SADDLE)])
def test_fp64_fallback_near_singular(ctx, m, delta, want):
    if m == 2:
        A = [[1.0, 1.0], [1.0, 1.0 + delta]]
        dims, centre, drift = (12, 12), (5.3, 6.1), (0.2, 0.1)
    else:
        A = [[1.0, 1.0, 0.0], [1.0, 1.0 + delta, 0.0], [0.0, 0.0, 1.0]]
        dims, centre, drift = (10, 10, 10), (4.3, 5.1, 4.7), (0.2, 0.1, 0.15)
    v = linear_field(A, dims, 3, centre, drift)
    case = cases.Case(f"lin{m}", "regular", m, cases.MULTI, v, 1e12, list(dims) + [3])
    g, o = run_both(ctx, case)
    assert len(g.cp_class) > 0
    assert np.array_equal(g.cp_class, o.cp_class)
    assert np.all(g.cp_class == want), np.unique(g.cp_class)
