"""Refactorization paths of one solver: the first factorization of a
solver's buffers runs its launches directly, the second records them as a
CUDA graph and every later one replays it.  Each path must give the same
factor bit for bit (the same kernels in the same order): factor A1, then A2
(recorded), then A1 again (replayed) and compare with the first."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt

pytestmark = pytest.mark.gpu


def test_plain_recorded_and_replayed_factors_agree():
    s = kkt.grid3d(grid=12, seed=3)
    rng = np.random.default_rng(0)
    cols = np.repeat(np.arange(s.n), np.diff(s.Ap))
    A2 = s.Ax.copy()
    diag_h = (s.Ai == cols) & (cols < s.n1)
    A2[diag_h] += rng.uniform(0.0, 0.1, int(diag_h.sum()))
    g = mp.GmresLDLIR()
    g.analyze(s.Ap, s.Ai, s.Ax)
    g.factor(s.Ax)
    first = g.export_factor()
    x1 = g.Solve(s.b)
    g.factor(A2)
    second = g.export_factor()
    g.factor(s.Ax)
    third = g.export_factor()
    x3 = g.Solve(s.b)
    g.factor(A2)
    fourth = g.export_factor()
    g.close()
    for a, b in zip(first, third):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(second, fourth):
        np.testing.assert_array_equal(a, b)
    assert np.max(np.abs(x1 - x3)) <= 1e-14 * np.max(np.abs(x1))
    assert not np.array_equal(first[2], second[2])
