"""The exact-rational yardstick for the residual step (tests/helpers.py:
exact_residual), checked on the CPU: a float64 residual of the symmetric
scatter product (ops.hpp:25-45, then VectorSubtract, ops.hpp:88-96) lies
within the standard summation bound gamma_k = k u / (1 - k u) of it, k the
terms in a row."""
import numpy as np

from mpir_b200 import kkt
from helpers import exact_residual, residual_error_ratios


def test_exact_residual_bounds_float64_residual():
    s = kkt.illcond3d(grid=5, seed=3)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(s.n)
    r64 = s.b - kkt.symmetric_matvec(s.n, s.Ap, s.Ai, s.Ax, x)
    ex, mag = exact_residual(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
    k = int(np.max(np.diff(s.Ap))) * 2 + 2
    u = 2.0 ** -53
    ratios = residual_error_ratios(r64, ex, mag)
    assert np.all(ratios <= k * u / (1 - k * u))
    # and the yardstick is not trivially loose: float64 misses by more than
    # double-double's bound somewhere
    assert np.max(ratios) > 2.0 ** -90
