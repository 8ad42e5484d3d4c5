"""Seeded synthetic quasi-definite KKT systems K = [[H, A^T], [A, -delta I]].

The reference measures only on SuiteSparse matrices, which are not available
here; these generators stand in with the shapes, sizes and value
distributions of the five workloads the solver is benchmarked on:

* ``small2d``  H = 5-point Laplacian on 32x32 + 1e-2 I, A 256x1024 with 4
  N(0,1) entries per row at distinct uniform columns, delta = 1e-4 (n = 1280).
* ``grid3d``   H = 7-point Laplacian on 48^3 + 1e-2 I, A 27,648 x 110,592 with
  6 entries per row, delta = 1e-6 (n = 138,240).
* ``illcond3d`` H = D L3D(64^3) D + 1e-8 I with D log-uniform in [1e-3, 1e3],
  A 65,536 x 262,144 with 8 entries per row, delta = 1e-8.
* ``batch2d``  64 instances on one pattern: H = L2D(256^2) + diag(s) with s
  log-uniform in [1e-6, 1e2], A 16,384 x 65,536 with 4 entries per row,
  delta = 1e-8, 16 right-hand sides each.

Every system is returned as the upper triangle in CSC (int64 column pointers
and row indices, float64 values, row indices ascending within each column,
no duplicates), the form QDLDL_etree/QDLDL_factor take (qdldl.hpp:12-47).
Unknowns are ordered H block first, then the constraint block.  The right-hand
side is b = K x_true with x_true ~ U(-1, 1).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp


@dataclass
class KKT:
    n: int
    Ap: np.ndarray
    Ai: np.ndarray
    Ax: np.ndarray
    n1: int
    m: int
    x_true: np.ndarray
    b: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.Ap[-1])


def laplacian(nx: int, dim: int) -> sp.csc_matrix:
    """Dirichlet 5-point (dim=2) or 7-point (dim=3) Laplacian on nx^dim."""
    one = sp.diags([-np.ones(nx - 1), 2 * np.ones(nx), -np.ones(nx - 1)], [-1, 0, 1], format="csr")
    eye = sp.identity(nx, format="csr")
    if dim == 2:
        L = sp.kron(eye, one) + sp.kron(one, eye)
    elif dim == 3:
        L = (sp.kron(sp.kron(eye, eye), one) + sp.kron(sp.kron(eye, one), eye)
             + sp.kron(sp.kron(one, eye), eye))
    else:
        raise ValueError(dim)
    return sp.csc_matrix(L)


def random_rows(rng: np.random.Generator, m: int, ncols: int, k: int) -> np.ndarray:
    """m x k column indices, distinct within each row, uniform over ncols."""
    cols = rng.integers(0, ncols, size=(m, k))
    while True:
        s = np.sort(cols, axis=1)
        dup = np.any(s[:, 1:] == s[:, :-1], axis=1) if k > 1 else np.zeros(m, bool)
        if not dup.any():
            return cols
        cols[dup] = rng.integers(0, ncols, size=(int(dup.sum()), k))


def upper_csc(M: sp.spmatrix):
    """Upper triangle of a symmetric sparse matrix as sorted int64 CSC."""
    U = sp.triu(M, format="csc")
    U.sum_duplicates()
    U.sort_indices()
    return (U.indptr.astype(np.int64), U.indices.astype(np.int64),
            U.data.astype(np.float64))


def symmetric_matvec(n, Ap, Ai, Ax, x):
    """y = K x for K given by its upper triangle (vectorised, float64)."""
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(Ap))
    y = np.bincount(cols, weights=Ax * x[Ai], minlength=n)
    off = Ai != cols
    y += np.bincount(Ai[off], weights=Ax[off] * x[cols[off]], minlength=n)
    return y


def assemble(H: sp.spmatrix, A_rows: np.ndarray, A_vals: np.ndarray, delta: float,
             rng: np.random.Generator, nrhs: int = 1, meta=None) -> KKT:
    n1 = H.shape[0]
    m, k = A_rows.shape
    n = n1 + m
    A = sp.csr_matrix((A_vals.ravel(), A_rows.ravel(), np.arange(0, m * k + 1, k)),
                      shape=(m, n1))
    K = sp.bmat([[sp.csc_matrix(H), A.T.tocsc()],
                 [A.tocsc(), -delta * sp.identity(m, format="csc")]], format="csc")
    Ap, Ai, Ax = upper_csc(K)
    if nrhs == 1:
        x_true = rng.uniform(-1.0, 1.0, size=n)
        b = symmetric_matvec(n, Ap, Ai, Ax, x_true)
    else:
        x_true = rng.uniform(-1.0, 1.0, size=(nrhs, n))
        b = np.stack([symmetric_matvec(n, Ap, Ai, Ax, xt) for xt in x_true])
    return KKT(n, Ap, Ai, Ax, n1, m, x_true, b, dict(meta or {}, delta=delta))


def make(grid: int, dim: int, m: int, per_row: int, delta: float, shift: float = 1e-2,
         seed: int = 0, scaled_range=None, diag_range=None, nrhs: int = 1) -> KKT:
    """General generator.  ``scaled_range=(lo, hi)`` gives H = D L D + shift I
    with D log-uniform in [lo, hi]; ``diag_range`` gives H = L + diag(s) with s
    log-uniform (the shift is then not added)."""
    rng = np.random.default_rng(seed)
    L = laplacian(grid, dim)
    n1 = L.shape[0]
    if scaled_range is not None:
        d = np.exp(rng.uniform(np.log(scaled_range[0]), np.log(scaled_range[1]), size=n1))
        Dm = sp.diags(d)
        H = Dm @ L @ Dm + shift * sp.identity(n1)
    elif diag_range is not None:
        s = np.exp(rng.uniform(np.log(diag_range[0]), np.log(diag_range[1]), size=n1))
        H = L + sp.diags(s)
    else:
        H = L + shift * sp.identity(n1)
    rows = random_rows(rng, m, n1, per_row)
    vals = rng.standard_normal(size=(m, per_row))
    return assemble(H, rows, vals, delta, rng, nrhs=nrhs,
                    meta=dict(grid=grid, dim=dim, m=m, per_row=per_row, seed=seed))


# Named workloads --------------------------------------------------------------

def small2d(seed: int = 0) -> KKT:
    """n = 1280: 32x32 5-point Laplacian + 1e-2 I, m = 256, 4 per row, delta 1e-4."""
    return make(32, 2, 256, 4, 1e-4, shift=1e-2, seed=seed)


def grid3d(seed: int = 0, grid: int = 48) -> KKT:
    """n = 138,240 at grid=48: 7-point Laplacian + 1e-2 I, m = grid^3/4, 6 per
    row, delta 1e-6.  Smaller ``grid`` keeps the same proportions."""
    return make(grid, 3, grid ** 3 // 4, 6, 1e-6, shift=1e-2, seed=seed)


def illcond3d(seed: int = 0, grid: int = 64) -> KKT:
    """D L3D D + 1e-8 I, D log-uniform in [1e-3, 1e3], m = grid^3/4, 8 per row,
    delta 1e-8."""
    return make(grid, 3, grid ** 3 // 4, 8, 1e-8, shift=1e-8, seed=seed,
                scaled_range=(1e-3, 1e3))


def batch2d(instances: int = 64, grid: int = 256, nrhs: int = 16, seed: int = 0):
    """Same-pattern batch: one pattern, per-instance H = L2D + diag(s) with s
    log-uniform in [1e-6, 1e2], m = grid^2/4 rows with 4 per row, delta 1e-8.
    Returns a list of KKT (shared Ap/Ai arrays, own Ax, x_true, b)."""
    rng = np.random.default_rng(seed)
    L = laplacian(grid, 2)
    n1 = L.shape[0]
    m = n1 // 4
    rows = random_rows(rng, m, n1, 4)
    vals = rng.standard_normal(size=(m, 4))
    out = []
    base = None
    for i in range(instances):
        s = np.exp(rng.uniform(np.log(1e-6), np.log(1e2), size=n1))
        H = L + sp.diags(s)
        sys_i = assemble(H, rows, vals, 1e-8, rng, nrhs=nrhs,
                         meta=dict(grid=grid, dim=2, m=m, per_row=4, seed=seed, instance=i))
        if base is None:
            base = sys_i
        else:
            assert np.array_equal(base.Ap, sys_i.Ap) and np.array_equal(base.Ai, sys_i.Ai)
            sys_i.Ap, sys_i.Ai = base.Ap, base.Ai
        out.append(sys_i)
    return out


def backward_error(n, Ap, Ai, Ax, x, b) -> float:
    """Normwise backward error ||b - Kx||_inf / (||K||_inf ||x||_inf + ||b||_inf)."""
    r = b - symmetric_matvec(n, Ap, Ai, Ax, x)
    absK = symmetric_matvec(n, Ap, Ai, np.abs(Ax), np.ones(n))
    return float(np.max(np.abs(r)) / (np.max(absK) * np.max(np.abs(x)) + np.max(np.abs(b))))


def forward_error(x, x_true) -> float:
    return float(np.max(np.abs(x - x_true)) / np.max(np.abs(x_true)))
