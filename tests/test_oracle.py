"""The oracle (oracle/oracle.c) pinned against the reference's own code
compiled from its headers (oracle/_ref) and against the reference's
known-answer tests (the doctest cases of include/MPIR/ops.hpp)."""
import numpy as np
import pytest

from mpir_b200 import kkt


# Known answers from the reference's doctests (ops.hpp:63-351).
def test_ops_known_answers_oracle(oracle_lib):
    O = oracle_lib
    assert O.dot([1.1, 2.2, 3.3], [4.4, 5.5, 6.6]) == pytest.approx(38.72)
    assert O.dot([1.5, 2.5, 3.5], [4.5, 5.5, 6.5]) == pytest.approx(43.25)
    assert O.dot([], []) == 0.0
    assert O.dnrm2([3.0, 4.0]) == pytest.approx(5.0)
    assert O.dnrm2([1.0, 2.0, 2.0]) == pytest.approx(3.0)
    assert O.dnrm2([0.0, 0.0, 0.0]) == 0.0
    assert O.dnrm2([5.5]) == pytest.approx(5.5)
    assert O.dnrm2([3.14, 2.71, 1.41]) == pytest.approx(np.sqrt(3.14**2 + 2.71**2 + 1.41**2))
    assert O.dnrm2([0.577] * 3) == pytest.approx(np.sqrt(3 * 0.577**2))
    assert O.dnrm2([]) == 0.0
    assert O.infnrm([3.0, -4.0, 5.5, -6.1]) == pytest.approx(6.1)
    assert O.infnrm([-1.1, -2.2, -3.3]) == pytest.approx(3.3)
    assert O.infnrm([0.0, 0.0, 0.0]) == 0.0
    assert O.infnrm([7.5]) == pytest.approx(7.5)
    assert O.infnrm([-3.14, 2.71, -1.41, 5.89]) == pytest.approx(5.89)


def test_ops_known_answers_reference(ref_lib):
    R = ref_lib
    np.testing.assert_allclose(R.vector_op(0, [5.5, 6.6, 7.7], [1.1, 2.2, 3.3]), [6.6, 8.8, 11.0])
    np.testing.assert_allclose(R.vector_op(1, [5.5, 6.6, 7.7], [1.1, 2.2, 3.3]), [4.4, 4.4, 4.4])
    np.testing.assert_allclose(R.vector_op(2, [1.1, 2.2, 3.3], [4.4, 5.5, 6.6]), [4.84, 12.1, 21.78])
    np.testing.assert_allclose(R.vector_op(3, [1.1, 2.2, 3.3], 2.0), [2.2, 4.4, 6.6])
    assert R.dot([1.1, 2.2, 3.3], [4.4, 5.5, 6.6]) == pytest.approx(38.72)
    assert R.dnrm2([3.0, 4.0]) == pytest.approx(5.0)
    assert R.infnrm([3.0, -4.0, 5.5, -6.1]) == pytest.approx(6.1)


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 5, 7, 8, 9, 31, 1000])
def test_oracle_ops_bitexact(oracle_lib, ref_lib, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal(n)
    b = rng.standard_normal(n)
    assert oracle_lib.dot(a, b) == ref_lib.dot(a, b)
    if n:
        assert oracle_lib.dnrm2(a) == ref_lib.dnrm2(a)
        assert oracle_lib.infnrm(a) == ref_lib.infnrm(a)


def _systems():
    yield "small2d", kkt.small2d()
    yield "grid3d_8", kkt.grid3d(grid=8, seed=3)
    yield "illcond3d_8", kkt.illcond3d(grid=8, seed=4)
    yield "batch2d_16", kkt.batch2d(instances=1, grid=16, nrhs=1, seed=5)[0]


@pytest.mark.parametrize("name,s", list(_systems()))
def test_oracle_qdldl_bitexact(oracle_lib, ref_lib, name, s):
    a = oracle_lib.etree(s.n, s.Ap, s.Ai)
    b = ref_lib.etree(s.n, s.Ap, s.Ai)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])
    for dt in (np.float32, np.float64):
        fa = oracle_lib.factor(s.n, s.Ap, s.Ai, s.Ax, dt)
        fb = ref_lib.factor(s.n, s.Ap, s.Ai, s.Ax, dt)
        assert fa[0] == fb[0]
        for x, y in zip(fa[1:], fb[1:]):
            np.testing.assert_array_equal(x, y)
        rhs = s.b if s.b.ndim == 1 else s.b[0]
        xa = oracle_lib.solve(s.n, fa[1], fa[2], fa[3], fa[5], rhs)
        xb = ref_lib.solve(s.n, fb[1], fb[2], fb[3], fb[5], rhs)
        np.testing.assert_array_equal(xa, xb)
    y = oracle_lib.matmul(s.n, s.Ap, s.Ai, s.Ax, s.x_true if s.x_true.ndim == 1 else s.x_true[0])
    z = ref_lib.matmul(s.n, s.Ap, s.Ai, s.Ax, s.x_true if s.x_true.ndim == 1 else s.x_true[0])
    np.testing.assert_array_equal(y, z)


@pytest.mark.parametrize("uf", [np.float32, np.float64])
def test_oracle_gmres_ir_bitexact(oracle_lib, ref_lib, uf):
    """The restated GMRES-IR driver, fed the same TriangularSolve form the
    harness injects into GmresLDLIR, reproduces the reference bit for bit."""
    s = kkt.small2d()
    xr, AD, info = ref_lib.gmres_ir(s.n, s.Ap, s.Ai, s.Ax, s.b, uf=uf)
    xo, st = oracle_lib.gmres_ir(s.n, s.Ap, s.Ai, s.Ax, s.b, uf=uf, form=1)
    np.testing.assert_array_equal(xo, xr)
    assert st["ir_steps"] == info["ir_steps"]
    ADo, _ = oracle_lib.scale(s.n, s.Ap, s.Ai, s.Ax,
                              float(np.finfo(uf).eps))
    np.testing.assert_array_equal(ADo, AD)
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, xr, s.b) <= 1e-14


def test_oracle_gmres_ir_qdldl_form(oracle_lib):
    """QDLDL_solve-form preconditioner (the GPU path's form) converges to the
    same backward-error bar."""
    for s in (kkt.small2d(), kkt.grid3d(grid=8, seed=1)):
        x, st = oracle_lib.gmres_ir(s.n, s.Ap, s.Ai, s.Ax, s.b, form=0)
        assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14
        assert kkt.forward_error(x, s.x_true) < 1e-9


def test_oracle_error_codes(oracle_lib, ref_lib):
    # empty column
    Ap = np.array([0, 1, 1, 2])
    Ai = np.array([0, 2])
    for L in (oracle_lib, ref_lib):
        assert L.etree(3, Ap, Ai)[0] == -1
    # entry below the diagonal
    Ap = np.array([0, 2, 3])
    Ai = np.array([0, 1, 1])
    for L in (oracle_lib, ref_lib):
        assert L.etree(2, Ap, Ai)[0] == -1
    # zero pivot: [[1, 1], [1, 1]]
    Ap = np.array([0, 1, 3])
    Ai = np.array([0, 0, 1])
    Ax = np.array([1.0, 1.0, 1.0])
    for L in (oracle_lib, ref_lib):
        assert L.factor(2, Ap, Ai, Ax, np.float64)[0] == -1


@pytest.mark.parametrize("maxiter", [0, 1, 10])
def test_oracle_luir_bitexact(oracle_lib, ref_lib, maxiter):
    """LUIR_QDLDL<float,double,double,double> (qdldl-luir/luir.hpp): the
    restatement equals the compiled reference bit for bit, including the
    stop test's step count."""
    for s in (kkt.small2d(), kkt.grid3d(grid=6, seed=3)):
        xo, io = oracle_lib.luir(s.n, s.Ap, s.Ai, s.Ax, s.b, maxiter)
        xr, ir = ref_lib.luir(s.n, s.Ap, s.Ai, s.Ax, s.b, maxiter)
        np.testing.assert_array_equal(xo, xr)
        assert io == ir
