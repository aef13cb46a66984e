"""The oracle's FP64 critical-point classifier (the checker for the CUDA
classification, which the reference does not have: type = 0 always,
predicate.hpp:80) against eigenvalues computed by numpy."""
import numpy as np
import pytest

from oracle import bridge

DEGENERATE, SOURCE, SINK, SADDLE, SPIRAL_SOURCE, SPIRAL_SINK, CENTER = range(1, 8)


def expected(J):
    ev = np.linalg.eigvals(J)
    if np.min(np.abs(ev)) < 1e-9:
        return DEGENERATE
    re = ev.real
    cpx = np.any(np.abs(ev.imag) > 1e-9)
    if np.all(re > 0):
        return SPIRAL_SOURCE if cpx else SOURCE
    if np.all(re < 0):
        return SPIRAL_SINK if cpx else SINK
    if len(ev) == 2 and cpx and np.all(np.abs(re) < 1e-12):
        return CENTER
    return SADDLE


@pytest.mark.parametrize("J,want", [
    (np.eye(2) * 2, SOURCE),                        # Hessian of x^2 + y^2: minimum
    (-np.eye(2), SINK),                             # maximum
    (np.diag([1.0, -1.0]), SADDLE),
    ([[0.1, -1.0], [1.0, 0.1]], SPIRAL_SOURCE),
    ([[-0.1, -1.0], [1.0, -0.1]], SPIRAL_SINK),
    ([[0.0, -1.0], [1.0, 0.0]], CENTER),
    ([[1.0, 2.0], [2.0, 4.0]], DEGENERATE),
    (np.zeros((2, 2)), DEGENERATE),
    (np.eye(3), SOURCE),
    (-np.eye(3) * 3, SINK),
    (np.diag([1.0, 1.0, -1.0]), SADDLE),            # h = 0 with a real pair
    (np.diag([1.0, 2.0, -3.0]), SADDLE),            # trace 0
    ([[0.1, -1, 0], [1, 0.1, 0], [0, 0, 0.5]], SPIRAL_SOURCE),
    ([[-0.1, -1, 0], [1, -0.1, 0], [0, 0, -0.5]], SPIRAL_SINK),
    ([[0.0, -1, 0], [1, 0.0, 0], [0, 0, 1.0]], CENTER),  # h = 0 with an imaginary pair
    (np.diag([1.0, 0.0, 1.0]), DEGENERATE),
    (np.array([[1.0, 2.0], [3.0, 4.0]]) * 1e300, SADDLE),   # scaled without overflow
    (np.array([[1.0, 0.5], [0.5, 1.0]]) * 1e-300, SOURCE),  # and without underflow
])
def test_known_jacobians(J, want):
    assert bridge.classify_jacobian(np.asarray(J, dtype=np.float64)) == want


@pytest.mark.parametrize("m", [2, 3])
def test_random_jacobians_match_eigenvalues(m):
    rng = np.random.default_rng(m)
    n = 0
    for _ in range(3000):
        J = rng.standard_normal((m, m))
        if rng.random() < 0.3:
            J = J + J.T  # a Hessian: real spectrum
        ev = np.linalg.eigvals(J)
        # keep away from the boundaries of the classes, where the eigenvalue
        # solver and the exact signs may legitimately disagree
        if np.min(np.abs(ev.real)) < 1e-6 or np.any((np.abs(ev.imag) > 0) & (np.abs(ev.imag) < 1e-6)):
            continue
        assert bridge.classify_jacobian(J) == expected(J), J
        n += 1
    assert n > 2500


def test_hessians_are_extrema_or_saddles():
    rng = np.random.default_rng(7)
    for _ in range(500):
        A = rng.standard_normal((3, 3))
        c = bridge.classify_jacobian(A + A.T)
        assert c in (SOURCE, SINK, SADDLE, DEGENERATE)
