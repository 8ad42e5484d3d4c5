"""mpir_b200: GMRES-IR with a supernodal LDL^T preconditioner on the NVIDIA B200.

The compute path is the in-tree CUDA library ``libmpir_b200.so`` (built for
sm_100a by ``mpir_b200/build.py``) behind the C ABI of
``include/mpir_b200.h``.  This module binds that ABI with ctypes and mirrors
the reference's interface for the path:

* :class:`GmresLDLIR` - ``GmresLDLIR<UF,UW,UR>`` of include/MPIR/gmres_ir.hpp
  (``Compute``, ``Solve``, ``SetMaxIRIterations``, ``SetMaxGmresIterations``,
  ``SetTolerance``), with ``Solve`` returning an empty array on a size
  mismatch as the reference does (gmres_ir.hpp:639-642);
* :func:`QDLDL_etree`, :func:`QDLDL_factor`, :func:`QDLDL_solve` - the QDLDL
  functions of include/MPIR/qdldl.hpp with their return codes.

There is no CPU fallback: importing succeeds without a GPU (analysis and
QDLDL_etree run on the host), but every numeric call needs the CUDA library
and a device, and raises if either is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import kkt  # noqa: F401  (synthetic systems)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpir_b200.so")

F64, F32, BF16, F16, DD = 0, 1, 2, 3, 4
ORDER_NATURAL, ORDER_AUTO = 0, 1
_PREC = {"f64": F64, "double": F64, np.float64: F64, "f32": F32, "float": F32,
         np.float32: F32, "bf16": BF16, "bfloat16": BF16, "f16": F16, "half": F16,
         np.float16: F16, "dd": DD, "dd_real": DD}
UPDATE = {"default": 0, "tf32x3": 1, "bf16x3": 2}
STATUS = {0: "ok", -1: "input", -2: "overflow", -3: "cuda", -4: "nomem", -5: "timeout",
          -6: "argument", -7: "unsupported", -8: "state"}


class MpirError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mpir status {code} ({STATUS.get(code, '?')}): {msg}")
        self.code = code


class Report(C.Structure):
    _fields_ = [("status", C.c_int32), ("ir_iterations", C.c_int32),
                ("gmres_iterations", C.c_int32), ("precond_applies", C.c_int32),
                ("spmv_count", C.c_int32), ("reorth_count", C.c_int32),
                ("stop_reason", C.c_int32), ("factor_prec", C.c_int32),
                ("residual_norm", C.c_double), ("backward_error", C.c_double),
                ("factor_ms", C.c_double), ("solve_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Info(C.Structure):
    _fields_ = [("n", C.c_int64), ("nnz_upper", C.c_int64), ("nnz_L", C.c_int64),
                ("supernodes", C.c_int64), ("levels", C.c_int64), ("panel_bytes", C.c_int64),
                ("update_bytes", C.c_int64), ("max_front", C.c_int64),
                ("factor_flops", C.c_double), ("solve_bytes", C.c_double),
                ("update_flops", C.c_double), ("trsm_flops", C.c_double),
                ("panel_read_bytes", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("uf", C.c_int32), ("ur", C.c_int32),
                ("workers", C.c_int32), ("max_batch", C.c_int32), ("update", C.c_int32),
                ("budget_bytes", C.c_int64), ("max_ir_iterations", C.c_int64),
                ("max_gmres_iterations", C.c_int64), ("tolerance", C.c_double)]


class ServerRequest(C.Structure):
    _fields_ = [("pattern_key", C.c_uint64), ("values_key", C.c_uint64), ("n", C.c_int64),
                ("Ap", C.c_void_p), ("Ai", C.c_void_p), ("Ax", C.c_void_p), ("b", C.c_void_p),
                ("x", C.c_void_p)]


class ServerResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int32), ("path", C.c_int32),
                ("batch", C.c_int32), ("pad", C.c_int32), ("latency_ms", C.c_double),
                ("queue_ms", C.c_double), ("service_ms", C.c_double), ("report", Report)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_int64) for k in (
        "submitted", "completed", "failed", "refused", "analyses", "factorizations", "solves",
        "batched_solves", "batched_rhs", "evictions", "resident_factors", "resident_patterns",
        "queued", "bytes_in_use", "peak_bytes", "analysis_reuses", "plan_uploads")] + [
        (k, C.c_double) for k in ("analysis_ms", "plan_ms", "factor_ms", "solve_ms",
                                  "factor_device_ms", "solve_device_ms", "setup_ms",
                                  "trim_ms", "plan_upload_ms")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise MpirError(-3, f"{LIB_PATH} is missing; run mpir_b200/build.py (no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, dbl = C.c_void_p, C.c_int64, C.c_int, C.c_double
    sig = {
        "mpir_version": (i32, []),
        "mpir_last_error": (C.c_char_p, []),
        "mpir_device_count": (i32, [vp]),
        "mpir_qdldl_etree": (i64, [i64, vp, vp, vp, vp, vp]),
        "mpir_qdldl_factor": (i64, [i64, vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, i32]),
        "mpir_qdldl_solve": (i32, [i64, vp, vp, vp, vp, i32, vp, i32, i32]),
        "mpir_qdldl_solve_noalloc": (i32, [i64, vp, vp, vp, vp, vp, i32]),
        "mpir_solver_create": (i32, [vp, i32, i32, i32, i32]),
        "mpir_solver_destroy": (i32, [vp]),
        "mpir_solver_set_max_ir_iterations": (i32, [vp, i64]),
        "mpir_solver_set_max_gmres_iterations": (i32, [vp, i64]),
        "mpir_solver_set_tolerance": (i32, [vp, dbl]),
        "mpir_solver_compute": (i32, [vp, i64, vp, vp, vp]),
        "mpir_solver_analyze": (i32, [vp, i64, vp, vp, vp, i32]),
        "mpir_solver_factor": (i32, [vp, vp]),
        "mpir_solver_factor_device": (i32, [vp, vp]),
        "mpir_solver_solve": (i32, [vp, vp, vp, vp]),
        "mpir_solver_solve_device": (i32, [vp, vp, vp, vp]),
        "mpir_solver_set_stream": (i32, [vp, vp]),
        "mpir_solver_set_update": (i32, [vp, i32]),
        "mpir_solver_solve_many": (i32, [vp, i64, vp, vp, vp]),
        "mpir_solver_solve_batch": (i32, [vp, i32, vp, vp, vp]),
        "mpir_solver_solve_batch_device": (i32, [vp, i32, vp, vp, vp]),
        "mpir_solver_apply_factor": (i32, [vp, i32, vp]),
        "mpir_solver_set_wait_controls": (i32, [vp, i32, i32]),
        "mpir_qdldl_lsolve": (i32, [i64, vp, vp, vp, i32, vp, i32, i32]),
        "mpir_qdldl_ltsolve": (i32, [i64, vp, vp, vp, i32, vp, i32, i32]),
        "mpir_solver_dump_log": (i32, [vp, vp, i64, vp]),
        "mpir_solver_luir": (i32, [vp, vp, vp, i32, vp]),
        "mpir_solver_residual": (i32, [vp, vp, vp, vp, i32, vp]),
        "mpir_solver_luir_device": (i32, [vp, vp, vp, i32, vp]),
        "mpir_luir_qdldl": (i32, [i64, vp, vp, vp, vp, vp, i32, i32, vp, i32]),
        "mpir_solver_info": (i32, [vp, vp]),
        "mpir_solver_symbolic": (i32, [vp, vp, vp, vp, vp, vp, vp]),
        "mpir_solver_export_factor": (i32, [vp, vp, vp, vp, vp, vp]),
        "mpir_solver_export_factor_leading": (i32, [vp, i64, vp, vp, vp, vp, vp]),
        "mpir_solver_supernodes": (i32, [vp, vp, vp, vp, vp]),
        "mpir_analyze_host": (i32, [i64, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp]),
        "mpir_group_create": (i32, [vp, vp, i32]),
        "mpir_group_factor": (i32, [vp, vp, vp]),
        "mpir_group_solve": (i32, [vp, i32, vp, vp, vp]),
        "mpir_group_solve_batch": (i32, [vp, i32, i32, vp, vp, vp]),
        "mpir_group_destroy": (i32, [vp]),
        "mpir_server_create": (i32, [vp, vp]),
        "mpir_server_submit": (i32, [vp, vp, vp]),
        "mpir_server_wait": (i32, [vp, i64, vp]),
        "mpir_server_drain": (i32, [vp]),
        "mpir_server_get_stats": (i32, [vp, vp]),
        "mpir_server_destroy": (i32, [vp]),
        "mpir_kernel_timer_enable": (i32, [i32]),
        "mpir_launch_count": (i64, []),
        "mpir_kernel_timer_collect": (i32, [vp, vp, i32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return lib().mpir_last_error().decode(errors="replace")


def _check(code):
    if code < 0:
        raise MpirError(int(code), last_error())
    return code


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def device_count() -> int:
    c = C.c_int(0)
    _check(lib().mpir_device_count(C.byref(c)))
    return c.value


# ----------------------------------------------------------------------------
# QDLDL (include/MPIR/qdldl.hpp)

def QDLDL_etree(n, Ap, Ai):
    """QDLDL_etree (qdldl.hpp:48-105): returns (sumLnz or -1/-2, Lnz, etree)."""
    Ap, Ai = _i64(Ap), _i64(Ai)
    work = np.zeros(max(n, 1), np.int64)
    Lnz = np.zeros(max(n, 1), np.int64)
    et = np.zeros(max(n, 1), np.int64)
    r = lib().mpir_qdldl_etree(n, _p(Ap), _p(Ai), _p(work), _p(Lnz), _p(et))
    if r < -2:
        raise MpirError(int(r), last_error())
    return int(r), Lnz[:n], et[:n]


def QDLDL_factor(n, Ap, Ai, Ax, Lnz, etree, fact_prec="f32", device=0):
    """QDLDL_factor (qdldl.hpp:172-345) on the GPU, natural order.

    Returns (status, Lp, Li, Lx, D, Dinv); status is the number of positive
    D entries or -1 on a zero pivot.  16-bit factors come back as uint16 bit
    patterns."""
    prec = _PREC[fact_prec]
    Ap, Ai, Ax = _i64(Ap), _i64(Ai), _f64(Ax)
    Lnz, etree = _i64(Lnz), _i64(etree)
    nl = int(Lnz.sum())
    dt = np.float32 if prec == F32 else np.uint16
    Lp = np.zeros(n + 1, np.int64)
    Li = np.zeros(max(nl, 1), np.int64)
    Lx = np.zeros(max(nl, 1), dt)
    D = np.zeros(max(n, 1), dt)
    Dinv = np.zeros(max(n, 1), dt)
    r = lib().mpir_qdldl_factor(n, _p(Ap), _p(Ai), _p(Ax), _p(Lp), _p(Li), _p(Lx), _p(D),
                                _p(Dinv), prec, _p(Lnz), _p(etree), device)
    if r < -1:
        raise MpirError(int(r), last_error())
    return int(r), Lp, Li[:nl], Lx[:nl], D[:n], Dinv[:n]


def QDLDL_solve(n, Lp, Li, Lx, Dinv, x, fact_prec="f32", device=0):
    """QDLDL_solve (qdldl.hpp:417-432) on the GPU: x <- (L D L^T)^{-1} x in
    place (x float64 or float32)."""
    prec = _PREC[fact_prec]
    xp = F64 if x.dtype == np.float64 else F32
    if not x.flags["C_CONTIGUOUS"]:
        raise ValueError("x must be contiguous")
    Lx = np.ascontiguousarray(Lx)
    Dinv = np.ascontiguousarray(Dinv)
    _check(lib().mpir_qdldl_solve(n, _p(_i64(Lp)), _p(_i64(Li)), _p(Lx), _p(Dinv), prec,
                                  _p(x), xp, device))
    return x


def _lsolve_common(fn, n, Lp, Li, Lx, x, fact_prec, device):
    prec = _PREC[fact_prec]
    xp = F64 if x.dtype == np.float64 else F32
    if not x.flags["C_CONTIGUOUS"]:
        raise ValueError("x must be contiguous")
    Lx = np.ascontiguousarray(Lx)
    _check(fn(n, _p(_i64(Lp)), _p(_i64(Li)), _p(Lx), prec, _p(x), xp, device))
    return x


def QDLDL_Lsolve(n, Lp, Li, Lx, x, fact_prec="f32", device=0):
    """QDLDL_Lsolve (qdldl.hpp:362-372) on the GPU: x <- (L + I)^{-1} x in place."""
    return _lsolve_common(lib().mpir_qdldl_lsolve, n, Lp, Li, Lx, x, fact_prec, device)


def QDLDL_Ltsolve(n, Lp, Li, Lx, x, fact_prec="f32", device=0):
    """QDLDL_Ltsolve (qdldl.hpp:389-400) on the GPU: x <- (L + I)^{-T} x in place."""
    return _lsolve_common(lib().mpir_qdldl_ltsolve, n, Lp, Li, Lx, x, fact_prec, device)


def LUIR_QDLDL(n, Ap, Ai, Ax, b, fact_prec="f32", maxiter=10, device=0):
    """LUIR_QDLDL<FACTPREC, double, double, double> (qdldl-luir/luir.hpp):
    factor A (upper CSC) in ``fact_prec`` and refine, all on the GPU.
    Returns (x, stats) with the reference's Stats fields
    num_refinement_steps_, relative_residual_ and Lnz_, plus the report."""
    Ap, Ai, Ax, b = _i64(Ap), _i64(Ai), _f64(Ax), _f64(b)
    x = np.zeros(n, np.float64)
    rep = Report()
    _check(lib().mpir_luir_qdldl(n, _p(Ap), _p(Ai), _p(Ax), _p(b), _p(x), _PREC[fact_prec],
                                 int(maxiter), C.byref(rep), device))
    r = rep.as_dict()
    stats = {"num_refinement_steps_": r["ir_iterations"],
             "relative_residual_": r["residual_norm"], "report": r}
    return x, stats


def QDLDL_solve_noalloc(n, Lp, Li, Lx, Dinv, x, device=0):
    """QDLDL_solve for callers that cannot allocate device memory (device
    memory reserved by a process-wide pooling allocator): float32
    factor, float64 x in place; all device data lives in the library's fixed
    32 MiB array.  Fronts of at most 64 rows; raises MpirError beyond the
    limits.  Calls overlapping on the GPU share that array and race."""
    if x.dtype != np.float64 or not x.flags["C_CONTIGUOUS"]:
        raise ValueError("x must be contiguous float64")
    Lx = np.ascontiguousarray(Lx, dtype=np.float32)
    Dinv = np.ascontiguousarray(Dinv, dtype=np.float32)
    _check(lib().mpir_qdldl_solve_noalloc(n, _p(_i64(Lp)), _p(_i64(Li)), _p(Lx), _p(Dinv),
                                          _p(x), device))
    return x


# ----------------------------------------------------------------------------
# GmresLDLIR (include/MPIR/gmres_ir.hpp:90-315)

class GmresLDLIR:
    """GMRES-IR with an LDL^T preconditioner, ``GmresLDLIR<UF,UW,UR>``.

    ``uf``/``uw``/``ur`` are the factor, working and residual precisions
    ("f32", "f64", "dd").  Defaults follow gmres_ir.hpp:113-117: 10
    refinement steps, 10 GMRES steps, tolerance 1e-10."""

    def __init__(self, uf="f32", uw="f64", ur="f64", device=0):
        self._h = C.c_void_p()
        _check(lib().mpir_solver_create(C.byref(self._h), _PREC[uf], _PREC[uw], _PREC[ur],
                                        device))
        self.n = 0
        self.last_report = None

    def close(self):
        if self._h:
            lib().mpir_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # setters (gmres_ir.hpp:291-303)
    def SetMaxIRIterations(self, n):
        _check(lib().mpir_solver_set_max_ir_iterations(self._h, int(n)))

    def SetMaxGmresIterations(self, n):
        _check(lib().mpir_solver_set_max_gmres_iterations(self._h, int(n)))

    def SetTolerance(self, tol):
        _check(lib().mpir_solver_set_tolerance(self._h, float(tol)))

    def Compute(self, Ap, Ai, Ax, ILU_k=0):
        """Analyse (fill-reducing order) and factor.  ``ILU_k`` is accepted for
        signature parity; the complete LDL^T factor has no ILU level."""
        Ap, Ai, Ax = _i64(Ap), _i64(Ai), _f64(Ax)
        self.n = len(Ap) - 1
        self._keep = (Ap, Ai)
        _check(lib().mpir_solver_compute(self._h, self.n, _p(Ap), _p(Ai), _p(Ax)))

    def analyze(self, Ap, Ai, Ax=None, ordering=ORDER_AUTO):
        Ap, Ai = _i64(Ap), _i64(Ai)
        self.n = len(Ap) - 1
        Axp = None if Ax is None else _f64(Ax)
        _check(lib().mpir_solver_analyze(self._h, self.n, _p(Ap), _p(Ai), _p(Axp), ordering))

    def factor(self, Ax):
        """New values on the analysed pattern; returns the status (0, or -1 on a
        zero pivot, which the caller may treat as QDLDL_factor's -1)."""
        Ax = _f64(Ax)
        r = lib().mpir_solver_factor(self._h, _p(Ax))
        if r < -1:
            raise MpirError(int(r), last_error())
        return int(r)

    def Solve(self, b):
        b = _f64(b)
        if b.shape != (self.n,):
            return np.zeros(0, np.float64)
        x = np.zeros(self.n, np.float64)
        rep = Report()
        _check(lib().mpir_solver_solve(self._h, _p(b), _p(x), C.byref(rep)))
        self.last_report = rep.as_dict()
        return x

    def DumpLog(self):
        """The log of the solves since the last call (the reference's
        GmresLDLIR::DumpLog schema under VERBOSE) as a dict; clears it."""
        import json
        n = C.c_int64(0)
        _check(lib().mpir_solver_dump_log(self._h, None, 0, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        _check(lib().mpir_solver_dump_log(self._h, buf, n.value, C.byref(n)))
        return json.loads(buf.value.decode())

    def SolveMany(self, B):
        """B: (nrhs, n) right-hand sides (one per row); returns X of the
        same shape, one GMRES-IR solve per row; reports in last_reports."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        if B.ndim != 2 or B.shape[1] != self.n:
            return np.zeros((0, self.n), np.float64)
        X = np.zeros_like(B)
        reps = (Report * max(B.shape[0], 1))()
        _check(lib().mpir_solver_solve_many(self._h, B.shape[0], _p(B), _p(X), reps))
        self.last_reports = [reps[k].as_dict() for k in range(B.shape[0])]
        return X

    def SolveBatch(self, B):
        """1 to 16 right-hand sides (rows of B) solved in lockstep, every
        preconditioner application one several-vector triangular solve;
        returns X of B's shape; reports in last_reports."""
        B = np.ascontiguousarray(B, dtype=np.float64)
        if B.ndim != 2 or B.shape[1] != self.n:
            return np.zeros((0, self.n), np.float64)
        X = np.zeros_like(B)
        reps = (Report * B.shape[0])()
        _check(lib().mpir_solver_solve_batch(self._h, B.shape[0], _p(B), _p(X), reps))
        self.last_reports = [reps[k].as_dict() for k in range(B.shape[0])]
        return X

    def apply_factor(self, X):
        """X (rows = vectors, internal permuted and scaled order) <-
        (L D L^T)^{-1} X for 1 to 16 vectors; returns a new array."""
        X = np.array(X, dtype=np.float64, order="C", copy=True)
        _check(lib().mpir_solver_apply_factor(self._h, X.shape[0], _p(X)))
        return X

    def set_wait_controls(self, poll_log2=0, withhold_item=-1):
        """Failure-test controls of the bounded device waits (see
        mpir_solver_set_wait_controls)."""
        _check(lib().mpir_solver_set_wait_controls(self._h, int(poll_log2), int(withhold_item)))

    def luir(self, b, maxiter=10):
        """Plain iterative refinement with the current factor (LUIR_QDLDL's
        loop, qdldl-luir/luir.hpp:182-232); the report's ir_iterations and
        residual_norm are the reference's num_refinement_steps_ and
        relative_residual_."""
        b = _f64(b)
        x = np.zeros(self.n, np.float64)
        rep = Report()
        _check(lib().mpir_solver_luir(self._h, _p(b), _p(x), int(maxiter), C.byref(rep)))
        self.last_report = rep.as_dict()
        return x

    def residual(self, b, x, prec="dd"):
        """r = b - A x on the device for the current values (the residual
        step of GmresLDLIR::Solve, gmres_ir.hpp:550-551) in float64 ("f64")
        or double-double ("dd") arithmetic; returns r rounded to float64."""
        b = _f64(b)
        x = _f64(x)
        r = np.zeros(self.n, np.float64)
        rinf = C.c_double(0.0)
        _check(lib().mpir_solver_residual(self._h, _p(b), _p(x), _p(r), _PREC[prec],
                                          C.byref(rinf)))
        return r

    def solve_device(self, d_b: int, d_x: int):
        """Device pointers (ints) in the caller's order."""
        rep = Report()
        _check(lib().mpir_solver_solve_device(self._h, C.c_void_p(d_b), C.c_void_p(d_x),
                                              C.byref(rep)))
        self.last_report = rep.as_dict()
        return self.last_report

    def factor_device(self, d_Ax: int):
        r = lib().mpir_solver_factor_device(self._h, C.c_void_p(d_Ax))
        if r < -1:
            raise MpirError(int(r), last_error())
        return int(r)

    def set_update(self, engine):
        """Trailing-update engine of a float32 factor: "tf32x3" (default) or
        "bf16x3" (from the next factorization)."""
        _check(lib().mpir_solver_set_update(self._h, UPDATE[engine]))

    def set_stream(self, stream_handle: int):
        _check(lib().mpir_solver_set_stream(self._h, C.c_void_p(stream_handle)))

    def info(self):
        inf = Info()
        _check(lib().mpir_solver_info(self._h, C.byref(inf)))
        return inf.as_dict()

    def symbolic(self):
        inf = self.info()
        n, nnz = inf["n"], inf["nnz_upper"]
        perm = np.zeros(n, np.int64)
        et = np.zeros(n, np.int64)
        Lnz = np.zeros(n, np.int64)
        Cp = np.zeros(n + 1, np.int64)
        Ci = np.zeros(nnz, np.int64)
        Cs = np.zeros(nnz, np.int64)
        _check(lib().mpir_solver_symbolic(self._h, _p(perm), _p(et), _p(Lnz), _p(Cp), _p(Ci),
                                          _p(Cs)))
        return dict(perm=perm, etree=et, Lnz=Lnz, Cp=Cp, Ci=Ci, Csrc=Cs)

    def supernodes(self):
        """(sfirst, srowptr, srows) of the analysed pattern."""
        inf = self.info()
        ns = inf["supernodes"]
        nrows = C.c_int64(0)
        _check(lib().mpir_solver_supernodes(self._h, None, None, None, C.byref(nrows)))
        sfirst = np.zeros(ns + 1, np.int64)
        srowptr = np.zeros(ns + 1, np.int64)
        srows = np.zeros(max(nrows.value, 1), np.int32)
        _check(lib().mpir_solver_supernodes(self._h, _p(sfirst), _p(srowptr), _p(srows),
                                            C.byref(nrows)))
        return sfirst, srowptr, srows[:nrows.value]

    def export_factor(self):
        inf = self.info()
        n, nl = inf["n"], inf["nnz_L"]
        Lp = np.zeros(n + 1, np.int64)
        Li = np.zeros(max(nl, 1), np.int64)
        Lx = np.zeros(max(nl, 1), np.float32)
        D = np.zeros(max(n, 1), np.float32)
        Dinv = np.zeros(max(n, 1), np.float32)
        _check(lib().mpir_solver_export_factor(self._h, _p(Lp), _p(Li), _p(Lx), _p(D), _p(Dinv)))
        return Lp, Li[:nl], Lx[:nl], D[:n], Dinv[:n]


class FactorGroup:
    """k value sets on the pattern a GmresLDLIR has analysed, refactorized by
    one CUDA graph launch (mpir_group_* in include/mpir_b200.h); each member
    is then solved like a solver of its own."""

    def __init__(self, solver, k):
        self.k = int(k)
        self.n = solver.n
        self._h = C.c_void_p()
        _check(lib().mpir_group_create(C.byref(self._h), solver._h, self.k))

    def factor(self, Axs):
        """Axs: k value arrays (rows).  Returns the positive-pivot counts."""
        A = np.ascontiguousarray(np.stack([_f64(a) for a in Axs]))
        npos = np.zeros(self.k, np.int64)
        r = lib().mpir_group_factor(self._h, _p(A), _p(npos))
        if r < -1:
            raise MpirError(int(r), last_error())
        self.last_status = int(r)
        return npos

    def Solve(self, member, b):
        b = _f64(b)
        x = np.zeros(self.n, np.float64)
        rep = Report()
        _check(lib().mpir_group_solve(self._h, int(member), _p(b), _p(x), C.byref(rep)))
        self.last_report = rep.as_dict()
        return x

    def SolveBatch(self, member, B):
        B = np.ascontiguousarray(B, dtype=np.float64)
        X = np.zeros_like(B)
        reps = (Report * B.shape[0])()
        _check(lib().mpir_group_solve_batch(self._h, int(member), B.shape[0], _p(B), _p(X), reps))
        self.last_reports = [reps[k].as_dict() for k in range(B.shape[0])]
        return X

    def close(self):
        if self._h:
            lib().mpir_group_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The serving engine (mpir_server_* in include/mpir_b200.h): GMRES-IR
    requests of mixed sizes and kinds on one GPU, with resident patterns and
    factors under a device-memory budget, lockstep batches of the queued
    right-hand sides on one factor, and concurrent work on different factors.

    ``submit`` takes one request (the system in upper CSC, its values, its
    right-hand side, and the keys naming its pattern and its values) and
    returns an id at once; ``wait`` returns that request's solution and
    result.  Arrays are kept referenced until the request is done."""

    def __init__(self, uf="f32", ur="f64", workers=4, max_batch=16, budget_bytes=150 * 10 ** 9,
                 ir_iter=10, gmres_iter=10, tol=1e-10, device=0, update="default"):
        cfg = ServerConfig(device=device, uf=_PREC[uf], ur=_PREC[ur], workers=workers,
                           max_batch=max_batch, update=UPDATE[update],
                           budget_bytes=int(budget_bytes),
                           max_ir_iterations=ir_iter, max_gmres_iterations=gmres_iter,
                           tolerance=tol)
        self._h = C.c_void_p()
        _check(lib().mpir_server_create(C.byref(self._h), C.byref(cfg)))
        self._live = {}

    def submit(self, pattern_key, values_key, Ap, Ai, Ax, b):
        Ap, Ai, Ax, b = _i64(Ap), _i64(Ai), _f64(Ax), _f64(b)
        n = len(Ap) - 1
        x = np.zeros(n, np.float64)
        req = ServerRequest(pattern_key, values_key, n, Ap.ctypes.data, Ai.ctypes.data,
                            Ax.ctypes.data, b.ctypes.data, x.ctypes.data)
        rid = C.c_int64(0)
        _check(lib().mpir_server_submit(self._h, C.byref(req), C.byref(rid)))
        self._live[rid.value] = (Ap, Ai, Ax, b, x)
        return rid.value

    def wait(self, rid):
        """(x, result dict) of request rid; result["status"] < 0 on failure
        (result["message"] says why)."""
        res = ServerResult()
        _check(lib().mpir_server_wait(self._h, int(rid), C.byref(res)))
        arrays = self._live.pop(rid)
        out = {k: getattr(res, k) for k, _ in res._fields_ if k not in ("pad", "report")}
        out["report"] = res.report.as_dict()
        out["message"] = last_error() if res.status != 0 else ""
        return arrays[4], out

    def drain(self):
        _check(lib().mpir_server_drain(self._h))

    def stats(self):
        st = ServerStats()
        _check(lib().mpir_server_get_stats(self._h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if self._h:
            lib().mpir_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def export_factor_leading(solver, k):
    """(Lp, Li, Lx, D) of the leading k x k block of a GmresLDLIR's factor
    (permuted order, QDLDL's CSC form)."""
    nnz = C.c_int64(0)
    Lp = np.zeros(k + 1, np.int64)
    _check(lib().mpir_solver_export_factor_leading(solver._h, k, _p(Lp), None, None, None,
                                                   C.byref(nnz)))
    Li = np.zeros(max(nnz.value, 1), np.int64)
    Lx = np.zeros(max(nnz.value, 1), np.float32)
    D = np.zeros(max(k, 1), np.float32)
    _check(lib().mpir_solver_export_factor_leading(solver._h, k, _p(Lp), _p(Li), _p(Lx), _p(D),
                                                   C.byref(nnz)))
    return Lp, Li[:nnz.value], Lx[:nnz.value], D[:k]


def analyze_host(Ap, Ai, Ax=None, ordering=ORDER_AUTO, pattern=False):
    """Host-only symbolic analysis: permutation, etree, Lnz, permuted upper CSC
    and (pattern=True) the exact L pattern of QDLDL_factor on P K P^T."""
    Ap, Ai = _i64(Ap), _i64(Ai)
    n = len(Ap) - 1
    Axp = None if Ax is None else _f64(Ax)
    inf = Info()
    _check(lib().mpir_analyze_host(n, _p(Ap), _p(Ai), _p(Axp), ordering, None, None, None, None,
                                   None, None, None, C.byref(inf)))
    nnz, nl = int(Ap[-1]) if n else 0, inf.nnz_L
    out = dict(perm=np.zeros(n, np.int64), etree=np.zeros(n, np.int64),
               Lnz=np.zeros(n, np.int64), Cp=np.zeros(n + 1, np.int64),
               Ci=np.zeros(max(nnz, 1), np.int64))
    Lp = np.zeros(n + 1, np.int64) if pattern else None
    Li = np.zeros(max(nl, 1), np.int64) if pattern else None
    _check(lib().mpir_analyze_host(n, _p(Ap), _p(Ai), _p(Axp), ordering, _p(out["perm"]),
                                   _p(out["etree"]), _p(out["Lnz"]), _p(out["Cp"]),
                                   _p(out["Ci"]), _p(Lp), _p(Li), C.byref(inf)))
    out["Ci"] = out["Ci"][:nnz]
    if pattern:
        out["Lp"], out["Li"] = Lp, Li[:nl]
    out["info"] = inf.as_dict()
    return out


KERNEL_CLASSES = ["small_front", "diag_block", "panel_solve", "trailing_update", "extend_add",
                  "zero_fill", "scatter", "solve_forward", "solve_backward", "spmv", "vector",
                  "split_reduce"]


def launch_count() -> int:
    """Kernel launches issued by the library so far in this process."""
    return int(lib().mpir_launch_count())


def kernel_timer(enable: bool):
    _check(lib().mpir_kernel_timer_enable(1 if enable else 0))


def kernel_times():
    n = len(KERNEL_CLASSES)
    ms = np.zeros(n, np.float64)
    cnt = np.zeros(n, np.int64)
    _check(lib().mpir_kernel_timer_collect(_p(ms), _p(cnt), n))
    return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(KERNEL_CLASSES)}
