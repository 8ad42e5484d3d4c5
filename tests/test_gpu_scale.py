"""GPU parity at a size where the factorization takes the paths the benchmark
takes: the 3-D KKT generator on 24^3 (n = 17,280; root front 4,096 rows, so
the 128-column left-looking steps, the tensor-core updates with K splits, the
ticketed triangular solves with chains of diagonal blocks and the one-CTA
extend-add all run).

The reference's own code (oracle/_ref: QDLDL_etree, QDLDL_factor<float> and
GmresLDLIR<float,double,double>::Solve preconditioned by that factor) runs
once on the same scaled, permuted matrix.  Tolerances: the symbolic pattern
bit-exact; the float32 L and D within 1e-5 normwise relative (the GPU factor
adds in another order); the GMRES-IR solution at backward error <= 1e-14
with a forward error within 10x of the reference's, and within 20x of the
reference's forward error of the reference's solution."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt
from helpers import permuted_upper, rel_norm_diff

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def grid24(ref_lib):
    s = kkt.grid3d(grid=24, seed=11)
    solver = mp.GmresLDLIR()
    solver.Compute(s.Ap, s.Ai, s.Ax, 0)
    x = solver.Solve(s.b)
    rep = solver.last_report
    sym = solver.symbolic()
    Lp, Li, Lx, D, Dinv = solver.export_factor()
    info = solver.info()
    solver.close()
    perm = sym["perm"]
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, perm)
    xr_p, AD, rinfo, rLx, rD = ref_lib.gmres_ir_with_factor(s.n, Cp, Ci, Cx, s.b[perm])
    xr = np.empty_like(xr_p)
    xr[perm] = xr_p
    return dict(s=s, x=x, rep=rep, sym=sym, Cp=Cp, Ci=Ci, Lp=Lp, Li=Li, Lx=Lx, D=D,
                info=info, xr=xr, rinfo=rinfo, rLx=rLx, rD=rD)


def test_grid24_takes_the_large_front_paths(grid24):
    # the root front is wide enough for the blocked, ticketed kernels
    assert grid24["info"]["max_front"] >= 4000
    assert grid24["info"]["levels"] >= 8


def test_grid24_pattern_bitexact(grid24, ref_lib):
    g = grid24
    n = g["s"].n
    tot, Lnz, et = ref_lib.etree(n, g["Cp"], g["Ci"])
    np.testing.assert_array_equal(g["sym"]["Lnz"], Lnz)
    np.testing.assert_array_equal(g["sym"]["etree"], et)
    np.testing.assert_array_equal(g["Lp"], np.concatenate([[0], np.cumsum(Lnz)]))
    assert g["Li"].size == tot == g["rLx"].size


def test_grid24_factor_within_1e5(grid24):
    g = grid24
    assert rel_norm_diff(g["Lx"], g["rLx"]) <= 1e-5
    assert rel_norm_diff(g["D"], g["rD"]) <= 1e-5
    # same inertia as the reference's factor (QDLDL_factor's return value)
    assert int(np.sum(g["D"] > 0)) == int(g["rinfo"]["npos"])


def test_grid24_gmres_ir_matches_reference(grid24):
    g = grid24
    s, x, xr = g["s"], g["x"], g["xr"]
    be = kkt.backward_error(s.n, s.Ap, s.Ai, s.Ax, x, s.b)
    assert be <= 1e-14, (be, g["rep"])
    fe_gpu = kkt.forward_error(x, s.x_true)
    fe_ref = kkt.forward_error(xr, s.x_true)
    assert fe_gpu <= max(10 * fe_ref, 1e-12), (fe_gpu, fe_ref)
    assert np.max(np.abs(x - xr)) / np.max(np.abs(xr)) <= max(20 * fe_ref, 1e-12)
