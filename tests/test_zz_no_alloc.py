"""QDLDL_solve for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: processes whose device memory is reserved
up front and owned entirely by their own pooling allocator, and loops that
cannot take cudaMalloc's implicit device-wide synchronisation.  mpir_qdldl_solve_noalloc
serves them from a fixed array the library holds on every GPU.  This file
checks it through the C ABI against the allocating mpir_qdldl_solve on two
calls in a row, and that out-of-limit factors are refused cleanly.  It is
named to be collected last."""
import numpy as np
import pytest
import scipy.sparse as sp

import mpir_b200 as mp
from helpers import rel_norm_diff

pytestmark = pytest.mark.gpu


def strip_factor(oracle_lib, width=8, length=400, seed=0):
    """float32 LDL^T of a shifted 5-point Laplacian on a width x length strip
    in natural order (bandwidth `width`, so every supernodal front is small)."""
    def lap1(k):
        return sp.diags([-np.ones(k - 1), 2 * np.ones(k), -np.ones(k - 1)], [-1, 0, 1])
    K = (sp.kron(sp.identity(length), lap1(width)) + sp.kron(lap1(length), sp.identity(width))
         + 1e-2 * sp.identity(width * length))
    U = sp.triu(K, format="csc")
    U.sort_indices()
    n = U.shape[0]
    st, Lp, Li, Lx, D, Dinv = oracle_lib.factor(n, U.indptr, U.indices, U.data, np.float32)
    assert st == n
    rng = np.random.default_rng(seed)
    return n, Lp, Li, Lx, Dinv, rng


def test_noalloc_matches_allocating_solve_twice(oracle_lib):
    n, Lp, Li, Lx, Dinv, rng = strip_factor(oracle_lib)
    for _ in range(2):  # two calls in a row share the scratch array
        b = rng.standard_normal(n)
        x_ref = b.copy()
        mp.QDLDL_solve(n, Lp, Li, Lx, Dinv, x_ref)
        x = b.copy()
        mp.QDLDL_solve_noalloc(n, Lp, Li, Lx, Dinv, x)
        assert rel_norm_diff(x, x_ref) <= 1e-10
        x_or = oracle_lib.solve(n, Lp, Li, Lx, Dinv, b)
        assert rel_norm_diff(x, x_or) <= 1e-10
    # a warmed-up call takes no device memory: the free bytes cudaMemGetInfo
    # reports are the same before and after it
    import torch
    x = rng.standard_normal(n)
    free0 = torch.cuda.mem_get_info(0)[0]
    mp.QDLDL_solve_noalloc(n, Lp, Li, Lx, Dinv, x)
    assert torch.cuda.mem_get_info(0)[0] == free0


def test_noalloc_refuses_out_of_limit_factors(oracle_lib):
    from mpir_b200 import kkt
    s = kkt.small2d()  # natural order: dense trailing fronts of ~290 rows
    st, Lp, Li, Lx, D, Dinv = oracle_lib.factor(s.n, s.Ap, s.Ai, s.Ax, np.float32)
    x = s.b.copy()
    with pytest.raises(mp.MpirError) as e:
        mp.QDLDL_solve_noalloc(s.n, Lp, Li, Lx, Dinv, x)
    assert e.value.code == -7
    assert np.array_equal(x, s.b)  # untouched
    # and the entry point still works afterwards
    n, Lp, Li, Lx, Dinv, rng = strip_factor(oracle_lib, width=6, length=100, seed=1)
    b = rng.standard_normal(n)
    x = b.copy()
    mp.QDLDL_solve_noalloc(n, Lp, Li, Lx, Dinv, x)
    x_ref = b.copy()
    mp.QDLDL_solve(n, Lp, Li, Lx, Dinv, x_ref)
    assert rel_norm_diff(x, x_ref) <= 1e-10
