"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference compiled from its headers, on the same seeded inputs.

Tolerances: symbolic results bit-exact; the float32 L and D within 1e-5
normwise relative of the reference's float32 QDLDL factor of the same matrix
(the GPU factor adds in a different order); solves within 1e-10 normwise
relative of the reference's solve with the same factor; the GMRES-IR
solution at normwise backward error <= 1e-14."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt
from helpers import permuted_upper, rel_norm_diff

pytestmark = pytest.mark.gpu

FLT_EPS = float(np.finfo(np.float32).eps)


def small_systems():
    yield "small2d", kkt.small2d()
    yield "grid3d_10", kkt.grid3d(grid=10, seed=1)
    yield "illcond3d_10", kkt.illcond3d(grid=10, seed=2)
    yield "batch2d_32", kkt.batch2d(instances=1, grid=32, nrhs=1, seed=3)[0]


# ---------------------------------------------------------------- QDLDL drop-in
@pytest.mark.parametrize("name,s", list(small_systems())[:2])
def test_qdldl_factor_matches_reference(ref_lib, name, s):
    tot, Lnz, et = mp.QDLDL_etree(s.n, s.Ap, s.Ai)
    st, Lp, Li, Lx, D, Dinv = mp.QDLDL_factor(s.n, s.Ap, s.Ai, s.Ax, Lnz, et)
    rs, rLp, rLi, rLx, rD, rDinv = ref_lib.factor(s.n, s.Ap, s.Ai, s.Ax, np.float32)
    assert st == rs
    np.testing.assert_array_equal(Lp, rLp)
    np.testing.assert_array_equal(Li, rLi)
    assert rel_norm_diff(Lx, rLx) <= 1e-5
    assert rel_norm_diff(D, rD) <= 1e-5
    assert rel_norm_diff(Dinv, rDinv) <= 1e-5


def test_qdldl_factor_permuted_and_16bit(ref_lib):
    s = kkt.grid3d(grid=8, seed=7)
    out = mp.analyze_host(s.Ap, s.Ai, s.Ax)
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, out["perm"])
    tot, Lnz, et = mp.QDLDL_etree(s.n, Cp, Ci)
    st, Lp, Li, Lx, D, Dinv = mp.QDLDL_factor(s.n, Cp, Ci, Cx, Lnz, et)
    rs, rLp, rLi, rLx, rD, rDinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float32)
    assert st == rs
    np.testing.assert_array_equal(Li, rLi)
    assert rel_norm_diff(Lx, rLx) <= 1e-5
    assert rel_norm_diff(D, rD) <= 1e-5
    # 16-bit storage is the float32 factor rounded to nearest
    import torch
    for prec, tdt in (("bf16", torch.bfloat16), ("f16", torch.float16)):
        st2, _, _, Lx2, D2, _ = mp.QDLDL_factor(s.n, Cp, Ci, Cx, Lnz, et, fact_prec=prec)
        assert st2 == st
        want = torch.from_numpy(Lx).to(tdt).view(torch.int16).numpy().view(np.uint16)
        np.testing.assert_array_equal(Lx2, want)


def test_qdldl_zero_pivot_and_errors():
    Ap, Ai, Ax = np.array([0, 1, 3]), np.array([0, 0, 1]), np.array([1.0, 1.0, 1.0])
    tot, Lnz, et = mp.QDLDL_etree(2, Ap, Ai)
    assert mp.QDLDL_factor(2, Ap, Ai, Ax, Lnz, et)[0] == -1
    with pytest.raises(mp.MpirError):
        mp.QDLDL_factor(2, Ap, Ai, Ax, Lnz, et, fact_prec="f64")


@pytest.mark.parametrize("name,s", list(small_systems())[:2])
def test_qdldl_solve_matches_reference(ref_lib, name, s):
    rs, Lp, Li, Lx, D, Dinv = ref_lib.factor(s.n, s.Ap, s.Ai, s.Ax, np.float32)
    xr = ref_lib.solve(s.n, Lp, Li, Lx, Dinv, s.b)
    x = s.b.copy()
    mp.QDLDL_solve(s.n, Lp, Li, Lx, Dinv, x)
    assert rel_norm_diff(x, xr) <= 1e-10
    # float32 vectors
    x32 = s.b.astype(np.float32)
    mp.QDLDL_solve(s.n, Lp, Li, Lx, Dinv, x32)
    xr32 = ref_lib.solve(s.n, Lp, Li, Lx, Dinv, s.b.astype(np.float32), xdtype=np.float32)
    assert rel_norm_diff(x32, xr32) <= 1e-4


# ---------------------------------------------------------------- GMRES-IR
@pytest.mark.parametrize("name,s", list(small_systems()))
def test_gmres_ir_matches_reference(ref_lib, name, s):
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax, 0)
    x = solver.Solve(s.b)
    rep = solver.last_report
    be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
    assert be <= 1e-14, (be, rep)
    assert rep["backward_error"] <= 1e-14
    assert abs(rep["backward_error"] - be) <= 1e-15 + 0.5 * be
    # the reference's GMRES-IR on the same ordering (its QDLDL on P K P^T)
    sym = solver.symbolic()
    perm = sym["perm"]
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, perm)
    bp = s.b[perm]
    xr_p, AD, info = ref_lib.gmres_ir(s.n, Cp, Ci, Cx, bp)
    xr = np.empty_like(xr_p)
    xr[perm] = xr_p
    fe_gpu = kkt.forward_error(x, s.x_true)
    fe_ref = kkt.forward_error(xr, s.x_true)
    assert fe_gpu <= max(10 * fe_ref, 1e-12), (fe_gpu, fe_ref)
    assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) <= max(20 * fe_ref, 1e-12)


def test_factor_matches_reference_on_scaled_permuted_matrix(oracle_lib, ref_lib):
    s = kkt.grid3d(grid=10, seed=5)
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax)
    sym = solver.symbolic()
    AD, Axs = oracle_lib.scale(s.n, s.Ap, s.Ai, s.Ax, FLT_EPS)
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, Axs, sym["perm"])
    np.testing.assert_array_equal(sym["Cp"], Cp)
    np.testing.assert_array_equal(sym["Ci"], Ci)
    tot, Lnz, et = ref_lib.etree(s.n, Cp, Ci)
    np.testing.assert_array_equal(sym["Lnz"], Lnz)
    np.testing.assert_array_equal(sym["etree"], et)
    Lp, Li, Lx, D, Dinv = solver.export_factor()
    rs, rLp, rLi, rLx, rD, rDinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float32)
    np.testing.assert_array_equal(Lp, rLp)
    np.testing.assert_array_equal(Li, rLi)
    assert rel_norm_diff(Lx, rLx) <= 1e-5
    assert rel_norm_diff(D, rD) <= 1e-5


def test_gmres_ir_settings_and_edges():
    s = kkt.small2d()
    solver = mp.GmresLDLIR()
    solver.SetMaxIRIterations(0)
    solver.SetMaxGmresIterations(30)
    solver.SetTolerance(1e-14)
    solver.Compute(s.Ap, s.Ai, s.Ax)
    x0 = solver.Solve(s.b)  # GMRES only, no refinement step
    assert solver.last_report["ir_iterations"] == 0
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x0, s.b) < 1e-10
    assert solver.Solve(s.b[:-1]).size == 0  # size mismatch -> empty
    # zero right-hand side
    z = solver.Solve(np.zeros(s.n))
    assert np.all(z == 0)
    # new values on the same pattern
    solver.SetMaxIRIterations(10)
    Ax2 = s.Ax * 2.0
    assert solver.factor(Ax2) == 0
    x2 = solver.Solve(s.b)
    np.testing.assert_allclose(x2, s.x_true / 2.0, rtol=0, atol=1e-10)


def test_gmres_ir_double_double_residual():
    s = kkt.illcond3d(grid=8, seed=11)
    a = mp.GmresLDLIR(ur="f64")
    a.Compute(s.Ap, s.Ai, s.Ax)
    xa = a.Solve(s.b)
    b = mp.GmresLDLIR(ur="dd")
    b.Compute(s.Ap, s.Ai, s.Ax)
    xb = b.Solve(s.b)
    for x in (xa, xb):
        assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14


def test_zero_pivot_reported():
    # K = [[1, 1], [1, 1]] is singular: the factor hits D = 0.
    Ap, Ai, Ax = np.array([0, 1, 3]), np.array([0, 0, 1]), np.array([1.0, 1.0, 1.0])
    solver = mp.GmresLDLIR()
    with pytest.raises(mp.MpirError) as e:
        solver.Compute(Ap, Ai, Ax)
    assert e.value.code == -1


def test_tiny_systems():
    for n in (1, 2, 3):
        Ap = np.arange(n + 1)
        Ai = np.arange(n)
        Ax = np.arange(1.0, n + 1)
        solver = mp.GmresLDLIR()
        solver.Compute(Ap, Ai, Ax)
        b = np.ones(n)
        x = solver.Solve(b)
        np.testing.assert_allclose(x, 1.0 / Ax, rtol=1e-15)


# ---------------------------------------------------------------- several right-hand sides
def test_same_pattern_batch_many_rhs():
    """The same-pattern batch (several instances sharing Ap/Ai, each with
    several right-hand sides): one analysis, a refactorization per instance,
    SolveMany per instance; every column at backward error <= 1e-14 and within
    rounding of the single-right-hand-side solve of that column (SolveMany
    runs the columns in lockstep through the several-vector triangular
    solves, which add in another order: 1e-12 normwise relative)."""
    batch = kkt.batch2d(instances=3, grid=24, nrhs=4, seed=6)
    solver = mp.GmresLDLIR()
    solver.analyze(batch[0].Ap, batch[0].Ai, batch[0].Ax)
    for s in batch:
        assert solver.factor(s.Ax) == 0
        X = solver.SolveMany(s.b)
        assert X.shape == s.b.shape
        for k in range(s.b.shape[0]):
            assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X[k], s.b[k]) <= 1e-14
        assert rel_norm_diff(X[1], solver.Solve(s.b[1])) <= 1e-12
        assert len(solver.last_reports) == s.b.shape[0]


# ---------------------------------------------------------------- log and driver
def test_dump_log_schema():
    """DumpLog: one gmres_ir event per solve with the reference's VERBOSE
    fields (gmres_ir.hpp:539-632), then the settings; cleared by the dump."""
    s = kkt.grid3d(grid=8, seed=2)
    solver = mp.GmresLDLIR(ur="dd")
    solver.SetTolerance(1e-15)
    solver.Compute(s.Ap, s.Ai, s.Ax)
    solver.Solve(s.b)
    solver.Solve(2 * s.b)
    log = solver.DumpLog()
    assert len(log["events"]) == 2
    assert log["max_outer_iterations"] == 10 and log["tolerance"] == 1e-15
    ev = log["events"][0]
    assert ev["name"] == "gmres_ir"
    assert ev["total_iterations"] == len(ev["iterations"])
    for it in ev["iterations"]:
        assert set(it) == {"iteration", "residual", "d_norm", "timestamp_ms", "inner_time_ms"}
    assert ev["stop_reason"] in ("max_iterations_reached", "converged_small_update",
                                 "converged_residual_stagnation", "exact_residual")
    assert solver.DumpLog()["events"] == []


def test_example_driver_on_matrix_market_file(tmp_path, capsys):
    """The example driver (examples/example.cpp) end to end on a Matrix
    Market file: b = A ones solved to the reference driver's residual level,
    and the JSON log written beside the matrix."""
    from mpir_b200 import example
    from mpir_b200.mmio import write_matrix_market
    s = kkt.small2d()
    p = tmp_path / "small2d.mtx"
    write_matrix_market(p, s.n, s.Ap, s.Ai, s.Ax)
    assert example.main([str(p), "--log"]) == 0
    out = capsys.readouterr().out
    assert out.splitlines()[0] == "symmetric"
    logs = list(tmp_path.glob("small2d_*.json"))
    assert len(logs) == 1
    import json
    log = json.loads(logs[0].read_text())
    assert log["matrix"] == "small2d" and log["ilu_k"] == 0
    assert log["residual_precision"] == "quadruple"
    assert log["relative_residual"] <= 1e-14
    assert log["relative_error"] <= 1e-10
    assert len(log["events"]) == 1


# ---------------------------------------------------------------- plain IR
@pytest.mark.parametrize("name,s", list(small_systems())[:3])
def test_luir_matches_reference(ref_lib, name, s):
    """LUIR_QDLDL on the GPU against the reference's LUIR_QDLDL on the same
    system: both refine to a relative residual at float64 rounding level; the
    GPU factor (permuted, scaled, different summation order) may take one
    refinement step more or less; solutions agree to the reference's forward
    error."""
    x, st = mp.LUIR_QDLDL(s.n, s.Ap, s.Ai, s.Ax, s.b, fact_prec="f32", maxiter=10)
    xr, ir = ref_lib.luir(s.n, s.Ap, s.Ai, s.Ax, s.b, 10)
    rel = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
    assert st["relative_residual_"] <= max(10 * ir["relres"], 1e-14), (st, ir)
    assert rel <= 1e-14
    assert abs(st["num_refinement_steps_"] - ir["steps"]) <= 1, (st, ir)
    fe_gpu, fe_ref = kkt.forward_error(x, s.x_true), kkt.forward_error(xr, s.x_true)
    assert fe_gpu <= max(10 * fe_ref, 1e-12), (fe_gpu, fe_ref)


def test_luir_single_solve_and_solver_handle():
    """maxiter = 0 is one solve (no refinement step); the solver handle's
    luir() refines with the factor it holds."""
    s = kkt.small2d()
    x0, st0 = mp.LUIR_QDLDL(s.n, s.Ap, s.Ai, s.Ax, s.b, maxiter=0)
    assert st0["num_refinement_steps_"] == 0
    assert st0["relative_residual_"] < 1e-4
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax)
    x = solver.luir(s.b, maxiter=10)
    assert solver.last_report["ir_iterations"] >= 1
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14


# ---------------------------------------------------------------- tensor cores
@pytest.fixture
def update_engine(monkeypatch):
    def set_engine(name):
        monkeypatch.setenv("MPIR_UPDATE", name)
    return set_engine


@pytest.mark.parametrize("engine", ["tf32x3", "simt"])
def test_update_engine_matches_reference(oracle_lib, ref_lib, update_engine, engine):
    """3xTF32 tensor-core trailing updates (the float32 default) and the
    float32 SIMT updates both keep the float32 factor within the same 1e-5 of
    the reference's float32 QDLDL factor.  grid 12 has fronts wider than one
    128-column block, so the left-looking updates and the split K run."""
    update_engine(engine)
    s = kkt.grid3d(grid=12, seed=9)
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax)
    sym = solver.symbolic()
    AD, Axs = oracle_lib.scale(s.n, s.Ap, s.Ai, s.Ax, FLT_EPS)
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, Axs, sym["perm"])
    Lp, Li, Lx, D, Dinv = solver.export_factor()
    rs, rLp, rLi, rLx, rD, rDinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float32)
    np.testing.assert_array_equal(Li, rLi)
    assert rel_norm_diff(Lx, rLx) <= 1e-5
    assert rel_norm_diff(D, rD) <= 1e-5
    x = solver.Solve(s.b)
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14


@pytest.mark.parametrize("uf", ["bf16", "f16"])
def test_low_precision_factor_tier_converges(uf):
    """16-bit tensor-core trailing updates: a rougher preconditioner, same
    float64 backward error after refinement."""
    for s in (kkt.grid3d(grid=12, seed=4), kkt.illcond3d(grid=10, seed=5)):
        solver = mp.GmresLDLIR(uf=uf)
        solver.SetMaxGmresIterations(50)
        solver.SetMaxIRIterations(30)
        solver.Compute(s.Ap, s.Ai, s.Ax)
        x = solver.Solve(s.b)
        be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
        assert be <= 1e-14, (uf, be, solver.last_report)
        # the report names the tier the factor was computed in
        assert solver.last_report["factor_prec"] == mp._PREC[uf]
        # lockstep solves read the same 16-bit L through the several-vector
        # kernels
        X = solver.SolveBatch(np.stack([s.b, 2 * s.b, -s.b]))
        for k, scale in enumerate((1, 2, -1)):
            assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, X[k], scale * s.b) <= 1e-14
        Y = np.random.default_rng(2).standard_normal((4, s.n))
        Z = solver.apply_factor(Y)
        for k in range(4):
            assert rel_norm_diff(Z[k], solver.apply_factor(Y[k:k + 1])[0]) <= 1e-12


@pytest.mark.parametrize("name,s", list(small_systems())[:3])
def test_forward_error_against_fp64_direct_ldlt(ref_lib, name, s):
    """Forward error of the GPU GMRES-IR solution against an FP64 direct
    LDL^T solution: the reference's QDLDL_factor<double> and QDLDL_solve on
    the same permuted matrix."""
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax, 0)
    x = solver.Solve(s.b)
    perm = solver.symbolic()["perm"]
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, perm)
    st, Lp, Li, Lx, D, Dinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float64)
    xd_p = ref_lib.solve(s.n, Lp, Li, Lx, Dinv, s.b[perm])
    xd = np.empty_like(xd_p)
    xd[perm] = xd_p
    fe_direct = kkt.forward_error(xd, s.x_true)
    fe = float(np.max(np.abs(x - xd)) / np.max(np.abs(xd)))
    assert fe <= max(10 * fe_direct, 1e-12), (fe, fe_direct)
    assert kkt.forward_error(x, s.x_true) <= max(10 * fe_direct, 1e-12)


def test_bf16x3_update_engine(oracle_lib, ref_lib):
    """3xBF16 trailing updates of a float32 factor (bfloat16 high and low
    parts, three products): about 16 significant bits per product, so L and D
    within 1e-4 normwise of the reference's float32 factor; GMRES-IR with it
    still reaches backward error <= 1e-14."""
    s = kkt.grid3d(grid=12, seed=9)
    solver = mp.GmresLDLIR()
    solver.set_update("bf16x3")
    solver.Compute(s.Ap, s.Ai, s.Ax)
    sym = solver.symbolic()
    AD, Axs = oracle_lib.scale(s.n, s.Ap, s.Ai, s.Ax, FLT_EPS)
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, Axs, sym["perm"])
    Lp, Li, Lx, D, Dinv = solver.export_factor()
    rs, rLp, rLi, rLx, rD, rDinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float32)
    np.testing.assert_array_equal(Li, rLi)
    assert rel_norm_diff(Lx, rLx) <= 1e-4
    assert rel_norm_diff(D, rD) <= 1e-4
    x = solver.Solve(s.b)
    assert kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b) <= 1e-14
    # the default engine again on the same solver: float32-level factor
    solver.set_update("tf32x3")
    solver.factor(s.Ax)
    Lp, Li, Lx, D, Dinv = solver.export_factor()
    assert rel_norm_diff(Lx, rLx) <= 1e-5
