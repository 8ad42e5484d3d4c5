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


def exact_residual(n, Ap, Ai, Ax, x, b):
    """r = b - K x in exact rational arithmetic (K symmetric, given by its
    upper triangle in CSC), with m_i = |b_i| + sum_j |k_ij x_j|, both as
    Fractions per row: the yardstick for residuals computed in float64 or
    double-double."""
    from fractions import Fraction
    r = [Fraction(float(v)) for v in b]
    m = [abs(v) for v in r]
    xf = [Fraction(float(v)) for v in x]
    for c in range(n):
        for p in range(int(Ap[c]), int(Ap[c + 1])):
            i = int(Ai[p])
            a = Fraction(float(Ax[p]))
            t = a * xf[i]
            r[c] -= t
            m[c] += abs(t)
            if i != c:
                t = a * xf[c]
                r[i] -= t
                m[i] += abs(t)
    return r, m


def residual_error_ratios(r, exact, mag):
    """Per row |r_i - exact_i| / m_i, with an exact difference to a float64 r_i
    that first loses half an ulp of exact_i (the final rounding to float64,
    which no residual arithmetic avoids)."""
    import math
    from fractions import Fraction
    out = np.zeros(len(exact))
    for i, (ri, ei, mi) in enumerate(zip(r, exact, mag)):
        d = abs(Fraction(float(ri)) - ei)
        d = max(d - Fraction(math.ulp(float(ei))) / 2, Fraction(0))
        out[i] = float(d / mi) if mi > 0 else float(d)
    return out
