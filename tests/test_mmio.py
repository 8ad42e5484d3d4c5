"""Matrix Market ingest (the reference example driver's reading rules,
examples/example.cpp:86-145): round trips and the rejected cases."""
import numpy as np
import pytest

from mpir_b200 import kkt
from mpir_b200.mmio import MatrixMarketError, read_matrix_market, write_matrix_market


def test_symmetric_round_trip(tmp_path):
    s = kkt.small2d()
    p = tmp_path / "small2d.mtx"
    write_matrix_market(p, s.n, s.Ap, s.Ai, s.Ax, comment="seeded KKT, n = 1280")
    n, Ap, Ai, Ax, sym = read_matrix_market(p)
    assert n == s.n and sym == "symmetric"
    np.testing.assert_array_equal(Ap, s.Ap)
    np.testing.assert_array_equal(Ai, s.Ai)
    np.testing.assert_array_equal(Ax, s.Ax)


def test_general_file_keeps_both_triangles(tmp_path):
    # a general file stores both triangles: the swapped read puts entries
    # below the diagonal, which the solver rejects as QDLDL_etree does
    p = tmp_path / "g.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n% c\n2 2 4\n"
                 "1 1 4.0\n2 1 1.0\n1 2 1.0\n2 2 3.0\n")
    n, Ap, Ai, Ax, sym = read_matrix_market(p)
    assert sym == "general"
    np.testing.assert_array_equal(Ap, [0, 2, 4])
    np.testing.assert_array_equal(Ai, [0, 1, 0, 1])
    assert np.any(Ai[Ap[0]:Ap[1]] > 0)


def test_pattern_and_errors(tmp_path):
    p = tmp_path / "p.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 3\n1 1\n2 2\n3 3\n")
    n, Ap, Ai, Ax, _ = read_matrix_market(p)
    np.testing.assert_array_equal(Ax, [1.0, 1.0, 1.0])
    bad = tmp_path / "b.mtx"
    bad.write_text("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n")
    with pytest.raises(MatrixMarketError):
        read_matrix_market(bad)
    rect = tmp_path / "r.mtx"
    rect.write_text("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1.0\n")
    with pytest.raises(MatrixMarketError):
        read_matrix_market(rect)
