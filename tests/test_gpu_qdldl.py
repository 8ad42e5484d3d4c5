"""QDLDL drop-in solves on the GPU beyond QDLDL_solve itself.

* QDLDL_Lsolve / QDLDL_Ltsolve (qdldl.hpp:362-400) on their own, against the
  reference's factor and a float64 triangular solve with the same L (1e-12
  normwise relative: the GPU accumulates in float64 as the reference does
  with XPREC = double).
* Repeated QDLDL_solve calls with one factor, as LUIR_QDLDL makes them
  (luir.hpp:165-205): the analysed, uploaded factor is reused, results are
  bitwise the same from call to call, and a factor rewritten in place is
  picked up (it hashes differently) and solved exactly as a fresh one."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import mpir_b200 as mp
from mpir_b200 import kkt
from helpers import rel_norm_diff

pytestmark = pytest.mark.gpu


def _unit_lower(n, Lp, Li, Lx):
    cols = np.repeat(np.arange(n), np.diff(Lp))
    L = sp.csr_matrix((Lx.astype(np.float64), (Li, cols)), shape=(n, n))
    return (L + sp.identity(n)).tocsr()


@pytest.mark.parametrize("grid", [8, 12])
def test_lsolve_and_ltsolve_alone(ref_lib, grid):
    s = kkt.grid3d(grid=grid, seed=9)
    out = mp.analyze_host(s.Ap, s.Ai, s.Ax)
    from helpers import permuted_upper
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, out["perm"])
    st, Lp, Li, Lx, D, Dinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float32)
    L = _unit_lower(s.n, Lp, Li, Lx)
    b = np.random.default_rng(grid).standard_normal(s.n)
    x = b.copy()
    mp.QDLDL_Lsolve(s.n, Lp, Li, Lx, x)
    assert rel_norm_diff(x, spla.spsolve_triangular(L, b, lower=True)) <= 1e-12
    y = b.copy()
    mp.QDLDL_Ltsolve(s.n, Lp, Li, Lx, y)
    assert rel_norm_diff(y, spla.spsolve_triangular(L.T.tocsr(), b, lower=False)) <= 1e-12
    # the three phases compose to QDLDL_solve
    z = b.copy()
    mp.QDLDL_Lsolve(s.n, Lp, Li, Lx, z)
    z *= Dinv.astype(np.float64)
    mp.QDLDL_Ltsolve(s.n, Lp, Li, Lx, z)
    w = b.copy()
    mp.QDLDL_solve(s.n, Lp, Li, Lx, Dinv, w)
    assert rel_norm_diff(z, w) <= 1e-13


def test_repeated_solves_reuse_the_factor(ref_lib):
    s = kkt.grid3d(grid=10, seed=4)
    out = mp.analyze_host(s.Ap, s.Ai, s.Ax)
    from helpers import permuted_upper
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, out["perm"])
    st, Lp, Li, Lx, D, Dinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float32)
    b = np.random.default_rng(1).standard_normal(s.n)
    first = mp.QDLDL_solve(s.n, Lp, Li, Lx, Dinv, b.copy())
    for _ in range(3):
        np.testing.assert_array_equal(mp.QDLDL_solve(s.n, Lp, Li, Lx, Dinv, b.copy()), first)
    assert rel_norm_diff(first, ref_lib.solve(s.n, Lp, Li, Lx, Dinv, b)) <= 1e-10
    # the same arrays rewritten in place: a new factor, solved as such
    Lx *= 0.5
    Dinv *= 2.0
    again = mp.QDLDL_solve(s.n, Lp, Li, Lx, Dinv, b.copy())
    assert rel_norm_diff(again, ref_lib.solve(s.n, Lp, Li, Lx, Dinv, b)) <= 1e-10
    assert rel_norm_diff(again, first) > 1e-3
