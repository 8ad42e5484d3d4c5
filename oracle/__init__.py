"""Oracle loaders: ctypes bindings for the two CPU checkers.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this package, and only as the checker.

* ``Oracle`` wraps ``oracle/liboracle.so``: the plain-C restatement of the
  reference path (``oracle/oracle.c``; each function cites the reference
  file:line it restates).
* ``Reference`` wraps ``oracle/_ref/libmpir_ref.so``: the reference's own
  headers (``include/MPIR/qdldl.hpp``, ``ops.hpp``, ``gmres_ir.hpp``) compiled
  unmodified by ``oracle/Makefile``.  It exists where the reference tree was
  present at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmpir_ref.so")

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_i64 = C.c_int64
FLT_EPS = float(np.finfo(np.float32).eps)


def build(ref_root: str | None = None) -> None:
    """Compile the oracle (and the reference harness when its tree exists)."""
    env = dict(os.environ)
    if ref_root:
        env["REF"] = ref_root
    args = ["make", "-s", "-C", HERE]
    if ref_root:
        args.append(f"REF={ref_root}")
    subprocess.run(args, check=True, env=env)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Common:
    prefix = ""

    def __init__(self, path):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        p = self.prefix
        L = self.lib
        f = getattr(L, f"{p}_etree")
        f.restype = _i64
        f.argtypes = [_i64, _i64p, _i64p, _i64p, _i64p, _i64p]
        for t, fp in (("f64", _f64p), ("f32", _f32p)):
            f = getattr(L, f"{p}_factor_{t}")
            f.restype = _i64
            f.argtypes = [_i64, _i64p, _i64p, _f64p, _i64p, _i64p, fp, fp, fp, _i64p, _i64p]
        for name, fp, xp in (("f64_f64", _f64p, _f64p), ("f32_f64", _f32p, _f64p),
                             ("f32_f32", _f32p, _f32p)):
            f = getattr(L, f"{p}_solve_{name}")
            f.restype = None
            f.argtypes = [_i64, _i64p, _i64p, fp, fp, xp]
        f = getattr(L, f"{p}_matmul")
        f.restype = None
        f.argtypes = [_i64, _i64p, _i64p, _f64p, _f64p, _f64p]
        for nm in ("dnrm2", "infnrm"):
            f = getattr(L, f"{p}_{nm}")
            f.restype = C.c_double
            f.argtypes = [_i64, _f64p]
        f = getattr(L, f"{p}_dot")
        f.restype = C.c_double
        f.argtypes = [_i64, _f64p, _f64p]

    # --- QDLDL -----------------------------------------------------------
    def etree(self, n, Ap, Ai):
        Ap, Ai = _i(Ap), _i(Ai)
        work = np.zeros(max(n, 1), np.int64)
        Lnz = np.zeros(max(n, 1), np.int64)
        et = np.zeros(max(n, 1), np.int64)
        s = getattr(self.lib, f"{self.prefix}_etree")(n, Ap, Ai, work, Lnz, et)
        return int(s), Lnz[:n], et[:n]

    def factor(self, n, Ap, Ai, Ax, dtype=np.float32):
        """Returns (status, Lp, Li, Lx, D, Dinv) in the factor type."""
        Ap, Ai, Ax = _i(Ap), _i(Ai), _d(Ax)
        s, Lnz, et = self.etree(n, Ap, Ai)
        if s < 0:
            return s, None, None, None, None, None
        Lp = np.zeros(n + 1, np.int64)
        Li = np.zeros(max(s, 1), np.int64)
        Lx = np.zeros(max(s, 1), dtype)
        D = np.zeros(max(n, 1), dtype)
        Dinv = np.zeros(max(n, 1), dtype)
        t = "f64" if dtype == np.float64 else "f32"
        r = getattr(self.lib, f"{self.prefix}_factor_{t}")(
            n, Ap, Ai, Ax, Lp, Li, Lx, D, Dinv, np.ascontiguousarray(Lnz), np.ascontiguousarray(et))
        return int(r), Lp, Li[:s], Lx[:s], D[:n], Dinv[:n]

    def solve(self, n, Lp, Li, Lx, Dinv, b, xdtype=np.float64):
        x = np.array(b, dtype=xdtype, copy=True)
        fd = "f64" if Lx.dtype == np.float64 else "f32"
        xd = "f64" if xdtype == np.float64 else "f32"
        getattr(self.lib, f"{self.prefix}_solve_{fd}_{xd}")(
            n, _i(Lp), _i(Li), np.ascontiguousarray(Lx), np.ascontiguousarray(Dinv), x)
        return x

    # --- ops ---------------------------------------------------------------
    def matmul(self, n, Ap, Ai, Ax, x):
        y = np.zeros(n, np.float64)
        getattr(self.lib, f"{self.prefix}_matmul")(n, _i(Ap), _i(Ai), _d(Ax), _d(x), y)
        return y

    def dnrm2(self, x):
        x = _d(x)
        return getattr(self.lib, f"{self.prefix}_dnrm2")(x.size, x)

    def infnrm(self, x):
        x = _d(x)
        return getattr(self.lib, f"{self.prefix}_infnrm")(x.size, x)

    def dot(self, a, b):
        a, b = _d(a), _d(b)
        return getattr(self.lib, f"{self.prefix}_dot")(a.size, a, b)


class Oracle(_Common):
    """The C restatement (oracle/oracle.c)."""

    prefix = "oracle"

    def __init__(self, path=ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.oracle_row_work.restype = _i64
        L.oracle_row_work.argtypes = [_i64, _i64p, _i64p, _f64p]
        L.oracle_scale.restype = None
        L.oracle_scale.argtypes = [_i64, _i64p, _i64p, _f64p, C.c_double, _f64p, _f64p]
        L.oracle_gmres_ir.restype = C.c_int
        L.oracle_gmres_ir.argtypes = [
            _i64, _i64p, _i64p, _f64p, _f64p, _i64p, _i64p, _f64p, _f64p, _f64p,
            C.c_int, C.c_int, _f64p, _f64p, _i64, _i64, C.c_double, _f64p]

    def row_work(self, n, Ap, Ai):
        """Multiply-subtract updates QDLDL_factor spends on each row of L."""
        w = np.zeros(max(n, 1), np.float64)
        r = self.lib.oracle_row_work(n, _i(Ap), _i(Ai), w)
        if r < 0:
            raise ValueError("not upper triangular")
        return w[:n]

    def scale(self, n, Ap, Ai, Ax, eps_uf=FLT_EPS):
        AD = np.zeros(n, np.float64)
        Axs = np.zeros(len(Ax), np.float64)
        self.lib.oracle_scale(n, _i(Ap), _i(Ai), _d(Ax), eps_uf, AD, Axs)
        return AD, Axs

    def luir(self, n, Ap, Ai, Ax, b, maxiter=10):
        """LUIR_QDLDL<float,double,double,double> restated: returns (x, info)
        with info = {steps, relres, nnzL}."""
        L = self.lib
        L.oracle_luir_f32.restype = C.c_int
        L.oracle_luir_f32.argtypes = [_i64, _i64p, _i64p, _f64p, _f64p, _f64p, C.c_int, _f64p]
        x = np.zeros(n, np.float64)
        info = np.zeros(3, np.float64)
        if L.oracle_luir_f32(n, _i(Ap), _i(Ai), _d(Ax), _d(b), x, int(maxiter), info) != 0:
            raise RuntimeError("oracle luir failed")
        return x, dict(zip(("steps", "relres", "nnzL"), info.tolist()))

    def gmres_ir(self, n, Ap, Ai, Ax, b, uf=np.float32, form=0, ir_iter=10,
                 gmres_iter=10, tol=1e-10):
        """Full GMRES-IR: scaling, QDLDL factor in ``uf``, then Solve.

        Returns (x, stats) with stats = {ir_steps, gmres_steps, reorth,
        precond_applies, spmv}."""
        eps = FLT_EPS if uf == np.float32 else float(np.finfo(np.float64).eps)
        AD, Axs = self.scale(n, Ap, Ai, Ax, eps)
        st, Lp, Li, Lx, D, Dinv = self.factor(n, Ap, Ai, Axs, dtype=uf)
        if st < 0:
            raise RuntimeError(f"oracle factor failed: {st}")
        x = np.zeros(n, np.float64)
        stats = np.zeros(5, np.float64)
        Lpad = Lx if Lx.size else np.zeros(1, uf)
        Lipad = Li if Li.size else np.zeros(1, np.int64)
        r = self.lib.oracle_gmres_ir(
            n, _i(Ap), _i(Ai), Axs, AD, _i(Lp), _i(Lipad), _d(Lpad.astype(np.float64)),
            _d(D.astype(np.float64)), _d(Dinv.astype(np.float64)), int(form),
            1 if uf == np.float32 else 0, _d(b), x, int(ir_iter), int(gmres_iter),
            float(tol), stats)
        if r != 0:
            raise RuntimeError("oracle gmres_ir failed")
        keys = ("ir_steps", "gmres_steps", "reorth", "precond_applies", "spmv")
        return x, dict(zip(keys, stats.tolist()))


class Reference(_Common):
    """The reference's own headers, compiled by oracle/Makefile."""

    prefix = "ref_qdldl"

    def __init__(self, path=REF_SO):
        # the reference exports ref_qdldl_* for QDLDL and ref_* for ops
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_qdldl_etree.restype = _i64
        L.ref_qdldl_etree.argtypes = [_i64, _i64p, _i64p, _i64p, _i64p, _i64p]
        for t, fp in (("f64", _f64p), ("f32", _f32p), ("bf16", _u16p), ("f16", _u16p)):
            f = getattr(L, f"ref_qdldl_factor_{t}")
            f.restype = _i64
            f.argtypes = [_i64, _i64p, _i64p, _f64p, _i64p, _i64p, fp, fp, fp, _i64p, _i64p]
        for name, fp, xp in (("f64_f64", _f64p, _f64p), ("f32_f64", _f32p, _f64p),
                             ("f32_f32", _f32p, _f32p), ("bf16_f32", _u16p, _f32p),
                             ("f16_f32", _u16p, _f32p)):
            f = getattr(L, f"ref_qdldl_solve_{name}")
            f.restype = None
            f.argtypes = [_i64, _i64p, _i64p, fp, fp, xp]
        L.ref_matmul.restype = None
        L.ref_matmul.argtypes = [_i64, _i64p, _i64p, _f64p, _f64p, _f64p]
        for nm in ("ref_dnrm2", "ref_infnrm"):
            getattr(L, nm).restype = C.c_double
            getattr(L, nm).argtypes = [_i64, _f64p]
        L.ref_dot.restype = C.c_double
        L.ref_dot.argtypes = [_i64, _f64p, _f64p]
        L.ref_dot_f32.restype = C.c_float
        L.ref_dot_f32.argtypes = [_i64, _f32p, _f32p]
        L.ref_vector_op.restype = None
        L.ref_vector_op.argtypes = [C.c_int, _i64, _f64p, _f64p, _f64p]
        L.ref_time_factor_leading_f32.restype = C.c_double
        L.ref_time_factor_leading_f32.argtypes = [_i64, _i64p, _i64p, _f64p]
        for t in ("f32", "f64"):
            f = getattr(L, f"ref_gmres_ir_{t}")
            f.restype = C.c_int
            f.argtypes = [_i64, _i64p, _i64p, _f64p, _f64p, _f64p, _i64, _i64, C.c_double,
                          _f64p, _f64p]
        L.ref_gmres_ir_f32_ex.restype = C.c_int
        L.ref_gmres_ir_f32_ex.argtypes = [_i64, _i64p, _i64p, _f64p, _f64p, _f64p, _i64, _i64,
                                          C.c_double, _f64p, _f64p, _f32p, _f32p]

    def etree(self, n, Ap, Ai):
        Ap, Ai = _i(Ap), _i(Ai)
        work = np.zeros(max(n, 1), np.int64)
        Lnz = np.zeros(max(n, 1), np.int64)
        et = np.zeros(max(n, 1), np.int64)
        s = self.lib.ref_qdldl_etree(n, Ap, Ai, work, Lnz, et)
        return int(s), Lnz[:n], et[:n]

    def factor(self, n, Ap, Ai, Ax, dtype=np.float32):
        Ap, Ai, Ax = _i(Ap), _i(Ai), _d(Ax)
        s, Lnz, et = self.etree(n, Ap, Ai)
        if s < 0:
            return s, None, None, None, None, None
        store = {np.float64: np.float64, np.float32: np.float32}.get(dtype, np.uint16)
        tag = {np.float64: "f64", np.float32: "f32"}.get(dtype)
        if tag is None:
            tag = "bf16" if dtype == "bf16" else "f16"
        Lp = np.zeros(n + 1, np.int64)
        Li = np.zeros(max(s, 1), np.int64)
        Lx = np.zeros(max(s, 1), store)
        D = np.zeros(max(n, 1), store)
        Dinv = np.zeros(max(n, 1), store)
        r = getattr(self.lib, f"ref_qdldl_factor_{tag}")(
            n, Ap, Ai, Ax, Lp, Li, Lx, D, Dinv, np.ascontiguousarray(Lnz), np.ascontiguousarray(et))
        return int(r), Lp, Li[:s], Lx[:s], D[:n], Dinv[:n]

    def solve(self, n, Lp, Li, Lx, Dinv, b, xdtype=np.float64, ftag=None):
        x = np.array(b, dtype=xdtype, copy=True)
        if ftag is None:
            ftag = "f64" if Lx.dtype == np.float64 else "f32"
        xd = "f64" if xdtype == np.float64 else "f32"
        getattr(self.lib, f"ref_qdldl_solve_{ftag}_{xd}")(
            n, _i(Lp), _i(Li), np.ascontiguousarray(Lx), np.ascontiguousarray(Dinv), x)
        return x

    def matmul(self, n, Ap, Ai, Ax, x):
        y = np.zeros(n, np.float64)
        self.lib.ref_matmul(n, _i(Ap), _i(Ai), _d(Ax), _d(x), y)
        return y

    def dnrm2(self, x):
        x = _d(x)
        return self.lib.ref_dnrm2(x.size, x)

    def infnrm(self, x):
        x = _d(x)
        return self.lib.ref_infnrm(x.size, x)

    def dot(self, a, b):
        a, b = _d(a), _d(b)
        return self.lib.ref_dot(a.size, a, b)

    def vector_op(self, op, a, b):
        a = _d(a)
        b = _d(np.atleast_1d(b))
        c = np.zeros(a.size, np.float64)
        self.lib.ref_vector_op(op, a.size, a, b, c)
        return c

    def luir(self, n, Ap, Ai, Ax, b, maxiter=10):
        """The reference's LUIR_QDLDL<float,double,double,double>: returns
        (x, info) with info = {steps, relres, nnzL}."""
        L = self.lib
        L.ref_luir_qdldl_f32.restype = C.c_int
        L.ref_luir_qdldl_f32.argtypes = [_i64, _i64p, _i64p, _f64p, _f64p, _f64p, C.c_int,
                                         _f64p]
        x = np.zeros(n, np.float64)
        info = np.zeros(3, np.float64)
        L.ref_luir_qdldl_f32(n, _i(Ap), _i(Ai), _d(Ax), _d(b), x, int(maxiter), info)
        return x, dict(zip(("steps", "relres", "nnzL"), info.tolist()))

    def gmres_ir(self, n, Ap, Ai, Ax, b, uf=np.float32, ir_iter=10, gmres_iter=10, tol=1e-10):
        """GmresLDLIR<UF,double,double>::Solve preconditioned by QDLDL<UF>.

        Returns (x, AD, info) with info = {factor_s, solve_s, ir_steps,
        reorth, nnzL, npos}."""
        x = np.zeros(n, np.float64)
        AD = np.zeros(n, np.float64)
        info = np.zeros(6, np.float64)
        tag = "f32" if uf == np.float32 else "f64"
        r = getattr(self.lib, f"ref_gmres_ir_{tag}")(
            n, _i(Ap), _i(Ai), _d(Ax), _d(b), x, int(ir_iter), int(gmres_iter), float(tol), AD, info)
        if r != 0:
            raise RuntimeError(f"reference gmres_ir failed: {r}")
        keys = ("factor_s", "solve_s", "ir_steps", "reorth", "nnzL", "npos")
        return x, AD, dict(zip(keys, info.tolist()))

    def gmres_ir_with_factor(self, n, Ap, Ai, Ax, b, ir_iter=10, gmres_iter=10, tol=1e-10):
        """As gmres_ir with UF = float, also returning the reference's float32
        QDLDL factor of the scaled matrix it preconditions with.

        Returns (x, AD, info, Lx, D): info adds etree_s (QDLDL_etree) and
        compute_s (the shipped Compute, run only for the diagonal scaling);
        Lx is in QDLDL's CSC order for the pattern of QDLDL_etree on (Ap, Ai)."""
        s, Lnz, _ = self.etree(n, Ap, Ai)
        if s < 0:
            raise RuntimeError(f"reference etree failed: {s}")
        x = np.zeros(n, np.float64)
        AD = np.zeros(n, np.float64)
        info = np.zeros(8, np.float64)
        Lx = np.zeros(max(s, 1), np.float32)
        D = np.zeros(max(n, 1), np.float32)
        r = self.lib.ref_gmres_ir_f32_ex(n, _i(Ap), _i(Ai), _d(Ax), _d(b), x, int(ir_iter),
                                         int(gmres_iter), float(tol), AD, info, Lx, D)
        if r != 0:
            raise RuntimeError(f"reference gmres_ir failed: {r}")
        keys = ("factor_s", "solve_s", "ir_steps", "reorth", "nnzL", "npos", "etree_s",
                "compute_s")
        return x, AD, dict(zip(keys, info.tolist())), Lx[:s], D[:n]

    def time_factor_leading(self, k, Ap, Ai, Ax):
        return self.lib.ref_time_factor_leading_f32(int(k), _i(Ap), _i(Ai), _d(Ax))


def permuted_scaled_upper(O, n, Ap, Ai, Ax, perm, eps_uf=FLT_EPS):
    """Upper CSC of P (AD K AD) P^T (perm[new] = old), scaled by the oracle's
    restatement of the reference's diagonal scaling: the matrix the
    reference's QDLDL_factor gets inside GMRES-IR on the same ordering."""
    import scipy.sparse as sp
    AD, Axs = O.scale(n, Ap, Ai, Ax, eps_uf)
    cols = np.repeat(np.arange(n), np.diff(np.asarray(Ap)))
    K = sp.coo_matrix((Axs, (np.asarray(Ai), cols)), shape=(n, n)).tocsc()
    K = (K + sp.triu(K, 1).T).tocsr()
    U = sp.triu(K[perm][:, perm], format="csc")
    U.sort_indices()
    return U.indptr.astype(np.int64), U.indices.astype(np.int64), U.data.astype(np.float64)


def have_reference() -> bool:
    return os.path.exists(REF_SO)
