"""The residual step of GmresLDLIR::Solve (gmres_ir.hpp:550-551:
MatrixMultiply<UR> then VectorSubtract<UR>, ops.hpp:25-45 and :88-96) on the
device, against exact rational arithmetic.

With UR = double-double the device adds exact products (two_prod) in
double-double and rounds the sum to float64 once.  Bound, per row i with k
terms and m_i = |b_i| + sum_j |k_ij x_j|: after the final rounding's half
ulp, |r_i - exact_i| <= 2^-96 m_i (k <= 2^8 double-double additions of
relative error 2^-104 each).  The float64 mode keeps the standard bound
gamma_k m_i.  The cases: a near-solution from GMRES-IR (the residual is
15-16 orders below m_i, so float64 keeps no correct digit while
double-double must) and a random x."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt
from helpers import exact_residual, residual_error_ratios

pytestmark = pytest.mark.gpu

DD_BOUND = 2.0 ** -96


@pytest.mark.parametrize("name,s", [("small2d", kkt.small2d(seed=4)),
                                    ("illcond3d-6", kkt.illcond3d(grid=6, seed=2))])
def test_dd_residual_against_exact_rationals(name, s):
    solver = mp.GmresLDLIR(ur="dd")
    solver.Compute(s.Ap, s.Ai, s.Ax, 0)
    x_near = solver.Solve(s.b)
    x_rand = np.random.default_rng(1).standard_normal(s.n)
    k = int(np.max(np.diff(s.Ap))) * 2 + 2
    gamma = k * 2.0 ** -53 / (1 - k * 2.0 ** -53)
    for x in (x_near, x_rand):
        ex, mag = exact_residual(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
        r_dd = solver.residual(s.b, x, "dd")
        r_64 = solver.residual(s.b, x, "f64")
        dd_ratio = residual_error_ratios(r_dd, ex, mag)
        f64_ratio = residual_error_ratios(r_64, ex, mag)
        assert np.max(dd_ratio) <= DD_BOUND, (name, np.max(dd_ratio))
        assert np.max(f64_ratio) <= gamma, (name, np.max(f64_ratio))
    # at the near-solution float64 loses what double-double keeps
    ex, mag = exact_residual(s.n, s.Ap, s.Ai, s.Ax, x_near, s.b)
    f64_ratio = residual_error_ratios(solver.residual(s.b, x_near, "f64"), ex, mag)
    assert np.max(f64_ratio) > DD_BOUND
    solver.close()


def test_residual_entry_errors():
    s = kkt.small2d(seed=5)
    solver = mp.GmresLDLIR()
    solver.analyze(s.Ap, s.Ai, s.Ax)
    with pytest.raises(mp.MpirError) as e:
        solver.residual(s.b, s.b, "dd")
    assert e.value.code == -8
    solver.factor(s.Ax)
    with pytest.raises(mp.MpirError) as e:
        solver.residual(s.b, s.b, "f32")
    assert e.value.code == -6
    r = solver.residual(s.b, np.zeros(s.n), "dd")
    np.testing.assert_array_equal(r, s.b)
    solver.close()
