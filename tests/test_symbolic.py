"""Host symbolic analysis (product code, no GPU): bit-exact with the
reference's QDLDL_etree and QDLDL_factor pattern on the same matrices."""
import numpy as np
import pytest

import mpir_b200 as mp
from mpir_b200 import kkt
from helpers import permuted_upper


def _systems():
    yield kkt.small2d()
    yield kkt.grid3d(grid=10, seed=1)
    yield kkt.illcond3d(grid=8, seed=2)
    yield kkt.batch2d(instances=1, grid=24, nrhs=1, seed=3)[0]


@pytest.mark.parametrize("s", list(_systems()))
def test_qdldl_etree_bitexact(ref_lib, s):
    a = mp.QDLDL_etree(s.n, s.Ap, s.Ai)
    b = ref_lib.etree(s.n, s.Ap, s.Ai)
    assert a[0] == b[0]
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])


@pytest.mark.parametrize("s", list(_systems()))
@pytest.mark.parametrize("ordering", [mp.ORDER_NATURAL, mp.ORDER_AUTO])
def test_analysis_matches_reference_on_permuted_matrix(ref_lib, s, ordering):
    out = mp.analyze_host(s.Ap, s.Ai, s.Ax, ordering=ordering, pattern=True)
    perm = out["perm"]
    assert np.array_equal(np.sort(perm), np.arange(s.n))
    if ordering == mp.ORDER_NATURAL:
        assert np.array_equal(perm, np.arange(s.n))
    Cp, Ci, Cx = permuted_upper(s.n, s.Ap, s.Ai, s.Ax, perm)
    np.testing.assert_array_equal(out["Cp"], Cp)
    np.testing.assert_array_equal(out["Ci"], Ci)
    tot, Lnz, et = ref_lib.etree(s.n, Cp, Ci)
    assert tot == out["info"]["nnz_L"]
    np.testing.assert_array_equal(out["Lnz"], Lnz)
    np.testing.assert_array_equal(out["etree"], et)
    st, Lp, Li, Lx, D, Dinv = ref_lib.factor(s.n, Cp, Ci, Cx, np.float64)
    assert st >= 0
    np.testing.assert_array_equal(out["Lp"], Lp)
    np.testing.assert_array_equal(out["Li"], Li)


def test_positive_block_first_and_fill_reduction():
    s = kkt.grid3d(grid=12, seed=0)
    nat = mp.analyze_host(s.Ap, s.Ai, s.Ax, ordering=mp.ORDER_NATURAL)
    aut = mp.analyze_host(s.Ap, s.Ai, s.Ax, ordering=mp.ORDER_AUTO)
    assert aut["info"]["nnz_L"] < 0.5 * nat["info"]["nnz_L"]
    # H unknowns (positive diagonal) are eliminated before the constraints.
    assert np.all(aut["perm"][: s.n1] < s.n1)
    assert aut["info"]["levels"] < 40


def test_error_codes_and_edge_sizes():
    # empty column -> -1, entry below the diagonal -> -1 (qdldl.hpp:64-78)
    assert mp.QDLDL_etree(3, [0, 1, 1, 2], [0, 2])[0] == -1
    assert mp.QDLDL_etree(2, [0, 2, 3], [0, 1, 1])[0] == -1
    with pytest.raises(mp.MpirError) as e:
        mp.analyze_host(np.array([0, 1, 1, 2]), np.array([0, 2]))
    assert e.value.code == -1
    # n = 0 and n = 1
    assert mp.QDLDL_etree(0, [0], [])[0] == 0
    r = mp.QDLDL_etree(1, [0, 1], [0])
    assert r[0] == 0 and r[2][0] == -1
    out = mp.analyze_host(np.array([0]), np.array([], np.int64))
    assert out["info"]["n"] == 0
    # diagonal only: no fill, every column its own root
    n = 50
    out = mp.analyze_host(np.arange(n + 1), np.arange(n), np.ones(n), pattern=True)
    assert out["info"]["nnz_L"] == 0 and np.all(out["etree"] == -1)


def test_dense_block():
    """A fully dense upper triangle: one supernode, nnz(L) = n(n-1)/2."""
    n = 70
    Ap = np.concatenate([[0], np.cumsum(np.arange(1, n + 1))]).astype(np.int64)
    Ai = np.concatenate([np.arange(j + 1) for j in range(n)]).astype(np.int64)
    out = mp.analyze_host(Ap, Ai, ordering=mp.ORDER_NATURAL, pattern=True)
    assert out["info"]["nnz_L"] == n * (n - 1) // 2
    assert out["info"]["supernodes"] == 1
