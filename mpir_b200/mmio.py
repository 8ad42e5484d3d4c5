"""Matrix Market ingest for the solver, as the reference's example driver
does it (examples/example.cpp:86-145).

The driver reads the coordinate file with rows and columns swapped (so the
lower triangle that a symmetric file stores becomes the upper triangle the
solver takes), sorts the entries by column and then row, and builds the CSC
column pointers; values are cast to float64.  A file with entries on both
sides of the diagonal (a "general" matrix) therefore yields a CSC with
entries below the diagonal, which the solver rejects as the reference's
QDLDL_etree does (-1).

Supported: coordinate format, fields real, integer and pattern (pattern
entries read as 1.0), symmetry general, symmetric, skew-symmetric; comment
lines (%) anywhere before the data.
"""
from __future__ import annotations

import numpy as np


class MatrixMarketError(ValueError):
    pass


def read_matrix_market(path):
    """Returns (n, Ap, Ai, Ax, symmetry) with Ap, Ai int64 and Ax float64,
    the upper-triangle CSC the example driver builds."""
    with open(path, "r") as f:
        header = f.readline().split()
        if len(header) < 5 or header[0].lower() != "%%matrixmarket":
            raise MatrixMarketError(f"{path}: not a Matrix Market file")
        obj, fmt, field, symmetry = (h.lower() for h in header[1:5])
        if obj != "matrix" or fmt != "coordinate":
            raise MatrixMarketError(f"{path}: only coordinate matrices are supported")
        if field not in ("real", "integer", "pattern", "double"):
            raise MatrixMarketError(f"{path}: field '{field}' is not supported")
        line = f.readline()
        while line and line.lstrip().startswith("%"):
            line = f.readline()
        dims = line.split()
        if len(dims) != 3:
            raise MatrixMarketError(f"{path}: bad size line")
        nrows, ncols, nnz = (int(v) for v in dims)
        if nrows != ncols:
            raise MatrixMarketError(f"{path}: the matrix is not square")
        cols_per = 2 if field == "pattern" else 3
        data = np.loadtxt(f, comments="%", ndmin=2, max_rows=nnz,
                          usecols=range(cols_per)) if nnz else np.zeros((0, cols_per))
    if data.shape[0] != nnz:
        raise MatrixMarketError(f"{path}: {data.shape[0]} entries, header says {nnz}")
    # rows and columns swapped, as the reference reads the triplets
    cs = data[:, 0].astype(np.int64) - 1
    rs = data[:, 1].astype(np.int64) - 1
    vs = data[:, 2].astype(np.float64) if field != "pattern" else np.ones(nnz)
    order = np.lexsort((rs, cs))  # by column, then row
    Ai, cols, Ax = rs[order], cs[order], vs[order]
    Ap = np.zeros(nrows + 1, np.int64)
    np.add.at(Ap, cols + 1, 1)
    Ap = np.cumsum(Ap)
    return nrows, Ap, Ai, Ax, symmetry


def write_matrix_market(path, n, Ap, Ai, Ax, comment=None):
    """Writes an upper-triangle CSC as a symmetric coordinate file (the
    lower triangle, 1-based), the form the reader above turns back into the
    same CSC."""
    Ap, Ai, Ax = np.asarray(Ap), np.asarray(Ai), np.asarray(Ax, np.float64)
    cols = np.repeat(np.arange(n), np.diff(Ap))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real symmetric\n")
        if comment:
            for ln in str(comment).splitlines():
                f.write(f"% {ln}\n")
        f.write(f"{n} {n} {len(Ai)}\n")
        for c, r, v in zip(cols, Ai, Ax):
            # upper entry (r, c), r <= c, written as the lower entry (c, r)
            f.write(f"{c + 1} {r + 1} {v:.17g}\n")
