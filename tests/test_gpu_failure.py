"""Failure detection on the GPU without a GPU fault.

* A bounded wait of the triangular solves made to run out: the test withholds
  the block result of one forward work item (a value that nothing then
  writes) and shortens the waits to 2^10 polls; the solve must return
  MPIR_ERR_TIMEOUT (-5), and the next solve with the controls cleared must
  succeed on the same solver.
* A non-finite right-hand side: the solve ends with stop reason 4 (r is not
  finite) and status 0, and the next solve is unaffected.
* A zero pivot: factor returns -1 and a solve before a good factor is a call
  out of order."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt

pytestmark = pytest.mark.gpu


def test_wait_timeout_is_reported_and_recovered():
    s = kkt.grid3d(grid=12, seed=8)
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax)
    assert solver.info()["max_front"] > 256  # the ticketed block kernels run
    x = solver.Solve(s.b)
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14
    solver.set_wait_controls(poll_log2=10, withhold_item=0)
    with pytest.raises(mp.MpirError) as ei:
        solver.Solve(s.b)
    assert ei.value.code == -5
    # the several-vector kernels report it the same way
    with pytest.raises(mp.MpirError) as ei:
        solver.SolveBatch(np.stack([s.b, s.b]))
    assert ei.value.code == -5
    solver.set_wait_controls(0, -1)
    x2 = solver.Solve(s.b)
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x2, s.b) <= 1e-14
    X = solver.SolveBatch(np.stack([s.b, s.b]))
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X[1], s.b) <= 1e-14
    solver.close()


def test_nonfinite_rhs_stops_with_reason_4():
    s = kkt.small2d()
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax)
    b = s.b.copy()
    b[7] = np.nan
    solver.Solve(b)
    assert solver.last_report["status"] == 0
    assert solver.last_report["stop_reason"] == 4
    x = solver.Solve(s.b)
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14
    solver.close()


def test_zero_pivot_then_state_error():
    n = 2
    Ap, Ai = np.array([0, 1, 3]), np.array([0, 0, 1])
    solver = mp.GmresLDLIR()
    solver.analyze(Ap, Ai, np.array([1.0, 1.0, 1.0]))
    assert solver.factor(np.array([1.0, 1.0, 1.0])) == -1
    with pytest.raises(mp.MpirError) as ei:
        solver.Solve(np.ones(n))
    assert ei.value.code == -8
    solver.close()
