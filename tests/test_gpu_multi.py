"""Several right-hand sides per factor on the GPU (through the C ABI).

* The several-vector triangular solve against the single-vector one, column
  by column, on fronts of every kind (warp-solved fronts only, and the
  ticketed 128-row block kernels): within 1e-12 normwise relative (the block
  kernels add in another order; the warp-solved fronts are bitwise equal).
* Lockstep GMRES-IR of up to 16 right-hand sides against one-at-a-time
  solves: every column at backward error <= 1e-14, its forward error within
  10x of the single solve's, and the two solutions within 20x of the single
  solve's forward error.
* The same-pattern batch (one analysis, a refactorization per instance, 16
  right-hand sides per instance)."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt
from helpers import rel_norm_diff

pytestmark = pytest.mark.gpu


def _factored(s):
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax)
    return solver


@pytest.mark.parametrize("name,make", [
    ("small2d", lambda: kkt.small2d()),
    ("grid3d_12", lambda: kkt.grid3d(grid=12, seed=4)),
    ("grid3d_20", lambda: kkt.grid3d(grid=20, seed=6)),
])
@pytest.mark.parametrize("nrhs", [3, 8, 16])
def test_apply_factor_multi_matches_single(name, make, nrhs):
    s = make()
    solver = _factored(s)
    rng = np.random.default_rng(nrhs)
    X = rng.standard_normal((nrhs, s.n))
    Y = solver.apply_factor(X)
    for k in range(nrhs):
        y1 = solver.apply_factor(X[k:k + 1])[0]
        assert rel_norm_diff(Y[k], y1) <= 1e-12, (name, k)
    solver.close()


def test_apply_factor_multi_bitwise_on_warp_fronts():
    # small2d's fronts are all solved by one warp each: the several-vector
    # kernels do per vector exactly the single kernels' operations
    s = kkt.small2d()
    solver = _factored(s)
    info = solver.info()
    X = np.random.default_rng(1).standard_normal((5, s.n))
    Y = solver.apply_factor(X)
    if info["max_front"] <= 64:
        for k in range(5):
            np.testing.assert_array_equal(Y[k], solver.apply_factor(X[k:k + 1])[0])
    solver.close()


@pytest.mark.parametrize("name,make", [
    ("small2d", lambda: kkt.small2d()),
    ("grid3d_16", lambda: kkt.grid3d(grid=16, seed=2)),
])
def test_solve_batch_matches_single_solves(name, make):
    s = make()
    solver = _factored(s)
    rng = np.random.default_rng(3)
    nrhs = 16
    Xt = rng.uniform(-1, 1, size=(nrhs, s.n))
    B = np.stack([kkt.symmetric_matvec(s.n, s.Ap, s.Ai, s.Ax, xt) for xt in Xt])
    X = solver.SolveBatch(B)
    reps = solver.last_reports
    assert len(reps) == nrhs
    for k in range(nrhs):
        be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X[k], B[k])
        assert be <= 1e-14, (k, be, reps[k])
        assert reps[k]["backward_error"] <= 1e-14
        x1 = solver.Solve(B[k])
        fe1 = kkt.forward_error(x1, Xt[k])
        fe = kkt.forward_error(X[k], Xt[k])
        assert fe <= max(10 * fe1, 1e-12), (k, fe, fe1)
        assert np.max(np.abs(X[k] - x1)) / np.max(np.abs(x1)) <= max(20 * fe1, 1e-12)
    # SolveMany goes through the same batches
    X2 = solver.SolveMany(B[:5])
    for k in range(5):
        assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X2[k], B[k]) <= 1e-14
    solver.close()


def test_same_pattern_batch_refactor_and_multi_rhs():
    insts = kkt.batch2d(instances=3, grid=24, nrhs=16, seed=5)
    solver = mp.GmresLDLIR()
    solver.analyze(insts[0].Ap, insts[0].Ai, insts[0].Ax)
    for s in insts:
        assert solver.factor(s.Ax) == 0
        X = solver.SolveBatch(s.b)
        for k in range(s.b.shape[0]):
            be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X[k], s.b[k])
            assert be <= 1e-14, (k, be)
    solver.close()


def test_solve_batch_argument_errors():
    s = kkt.small2d()
    solver = _factored(s)
    with pytest.raises(mp.MpirError):
        solver.SolveBatch(np.zeros((17, s.n)))
    assert solver.SolveBatch(np.zeros((2, s.n - 1))).size == 0
    solver.close()


def test_factor_group_one_launch_matches_solo_factors():
    """Same-pattern instances refactorized together by one graph launch give
    the factors (and so the solutions) each gets alone."""
    insts = kkt.batch2d(instances=3, grid=24, nrhs=4, seed=7)
    base = mp.GmresLDLIR()
    base.analyze(insts[0].Ap, insts[0].Ai, insts[0].Ax)
    grp = mp.FactorGroup(base, len(insts))
    for rounds in range(2):  # the recorded launch is replayed for new values
        if rounds:
            insts = insts[::-1]
        npos = grp.factor([s.Ax for s in insts])
        assert grp.last_status == 0 and np.all(npos > 0)
        for i, s in enumerate(insts):
            X = grp.SolveBatch(i, s.b)
            solo = mp.GmresLDLIR()
            solo.Compute(s.Ap, s.Ai, s.Ax)
            for k in range(s.b.shape[0]):
                assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X[k], s.b[k]) <= 1e-14
                x1 = grp.Solve(i, s.b[k])
                xs = solo.Solve(s.b[k])
                assert np.max(np.abs(x1 - xs)) / np.max(np.abs(xs)) <= 1e-13
            solo.close()
    grp.close()
    base.close()
