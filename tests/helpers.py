"""Shared helpers for the tests: permuted matrices and comparisons."""
import numpy as np
import scipy.sparse as sp


def full_csc(n, Ap, Ai, Ax):
    cols = np.repeat(np.arange(n), np.diff(Ap))
    K = sp.coo_matrix((Ax, (Ai, cols)), shape=(n, n)).tocsc()
    return K + sp.triu(K, 1).T


def permuted_upper(n, Ap, Ai, Ax, perm):
    """Upper CSC of P K P^T with perm[new] = old, rows sorted."""
    K = full_csc(n, Ap, Ai, Ax).tocsr()
    Kp = K[perm][:, perm]
    U = sp.triu(Kp, format="csc")
    U.sort_indices()
    return U.indptr.astype(np.int64), U.indices.astype(np.int64), U.data.astype(np.float64)


def diag_signs(n, Ap, Ai, Ax):
    cols = np.repeat(np.arange(n), np.diff(Ap))
    d = np.zeros(n)
    m = Ai == cols
    d[cols[m]] = Ax[m]
    return d


def rel_norm_diff(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
