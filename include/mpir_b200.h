/* mpir_b200 C ABI: GMRES-IR for sparse quasidefinite systems preconditioned
 * by a supernodal LDL^T factor, on one NVIDIA B200 (sm_100a).
 *
 * The entry points replace the CPU hot path of the reference library (MPIR,
 * header-only C++): QDLDL_etree / QDLDL_factor / QDLDL_solve in
 * include/MPIR/qdldl.hpp and the GmresLDLIR<UF,UW,UR> solver in
 * include/MPIR/gmres_ir.hpp.  The C++ headers include/MPIR/qdldl.hpp and
 * include/MPIR/gmres_ir.hpp of this project keep the reference's template
 * signatures and forward to these functions.
 *
 * Conventions: plain host pointers and sizes; all matrices are the upper
 * triangle of a symmetric matrix in CSC with int64 column pointers and row
 * indices, no duplicates.  Status codes are 0 on success and negative on
 * failure; mpir_last_error() returns the calling thread's last message.
 */
#ifndef MPIR_B200_H
#define MPIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  -1 and -2 mean what they mean for QDLDL_etree /
 * QDLDL_factor (qdldl.hpp:43-45, :135-138). */
enum {
  MPIR_OK              = 0,
  MPIR_ERR_INPUT       = -1, /* not upper triangular, empty column, zero pivot */
  MPIR_ERR_OVERFLOW    = -2, /* nonzero count of L overflows */
  MPIR_ERR_CUDA        = -3, /* CUDA runtime error (message has details) */
  MPIR_ERR_NOMEM       = -4, /* device or host allocation failed */
  MPIR_ERR_TIMEOUT     = -5, /* a bounded device wait ran out */
  MPIR_ERR_ARGUMENT    = -6, /* invalid argument */
  MPIR_ERR_UNSUPPORTED = -7, /* precision combination not provided */
  MPIR_ERR_STATE       = -8  /* call out of order (solve before factor, ...) */
};

/* Floating-point types of the factor (UF), working (UW) and residual (UR)
 * precisions, as the reference's template parameters. */
enum {
  MPIR_F64  = 0,
  MPIR_F32  = 1,
  MPIR_BF16 = 2,
  MPIR_F16  = 3,
  MPIR_DD   = 4 /* double-double, the reference's dd_real residual type */
};

/* Orderings for mpir_solver_analyze. */
enum { MPIR_ORDER_NATURAL = 0, MPIR_ORDER_AUTO = 1 };

/* Outcome of one GMRES-IR solve. */
typedef struct mpir_report {
  int32_t status;
  int32_t ir_iterations;    /* refinement steps (gmres_ir.hpp:561) */
  int32_t gmres_iterations; /* inner Arnoldi steps over all PrecondGmres calls */
  int32_t precond_applies;  /* L D L^T solves */
  int32_t spmv_count;       /* products with K */
  int32_t reorth_count;     /* Brown/Hindmarsh re-orthogonalisations */
  int32_t stop_reason;      /* 0 iteration cap, 1 small update, 2 stagnation,
                               3 zero residual, 4 non-finite residual or
                               factor (a pivot beyond the factor type's
                               range; x is then the first solve's) */
  int32_t factor_prec;      /* MPIR_F32 / MPIR_BF16 / MPIR_F16: the type the
                               factor was computed and applied in (MPIR_F32
                               for a solver created with UF = MPIR_F64) */
  double residual_norm;  /* ||r||_inf / ||b_scaled||_inf at exit (gmres_ir.hpp:580) */
  double backward_error; /* ||b - Kx||_inf / (||K||_inf ||x||_inf + ||b||_inf) */
  double factor_ms;      /* device time of the last numeric factorization */
  double solve_ms;       /* device time of this solve */
} mpir_report;

/* Facts about an analysed pattern. */
typedef struct mpir_info {
  int64_t n, nnz_upper, nnz_L;   /* nnz_L = sum of QDLDL_etree's Lnz */
  int64_t supernodes, levels;
  int64_t panel_bytes;           /* factor storage */
  int64_t update_bytes;          /* update-matrix arena */
  int64_t max_front;             /* largest front height */
  double  factor_flops;          /* sum_j Lnz_j^2: multiply-adds x 2 of the
                                    exact elimination */
  double  solve_bytes;           /* bytes one L D L^T solve must move: float32
                                    L twice, Dinv, four float64 vectors */
  double  update_flops;          /* flops of the trailing-update launches */
  double  trsm_flops;            /* flops of the panel-solve launches */
  double  panel_read_bytes;      /* panel bytes one forward (or backward)
                                    sweep reads, padding included */
} mpir_info;

typedef struct mpir_solver_s *mpir_solver;

int         mpir_version(void);
const char *mpir_last_error(void);
int         mpir_device_count(int *count);

/* ---- QDLDL drop-in ------------------------------------------------------ */

/* Replaces QDLDL_etree (include/MPIR/qdldl.hpp:48-105).  Host computation;
 * Lnz and etree are equal element for element to the reference's.  `work`
 * (n entries) is scratch, as in the reference.  Returns sum(Lnz), -1 or -2. */
int64_t mpir_qdldl_etree(int64_t n, const int64_t *Ap, const int64_t *Ai,
                         int64_t *work, int64_t *Lnz, int64_t *etree);

/* Replaces QDLDL_factor (include/MPIR/qdldl.hpp:172-345) in natural order on
 * device `device`.  Ax is float64 (the caller's values); the factor is
 * computed in float32 and written to the caller's arrays (Lp: n+1, Li/Lx:
 * sum(Lnz), D/Dinv: n) in fact_prec (MPIR_F32, or MPIR_BF16 / MPIR_F16 as
 * raw 16-bit patterns rounded from float32).  Lnz and etree must be
 * QDLDL_etree's output.  Li comes out in QDLDL's order (rows ascending in each
 * column).  Returns the number of positive entries of D, or -1 on a zero
 * pivot, or another negative status. */
int64_t mpir_qdldl_factor(int64_t n, const int64_t *Ap, const int64_t *Ai,
                          const double *Ax, int64_t *Lp, int64_t *Li, void *Lx,
                          void *D, void *Dinv, int fact_prec,
                          const int64_t *Lnz, const int64_t *etree, int device);

/* Replaces QDLDL_solve (include/MPIR/qdldl.hpp:417-432): x <- (L D L^T)^{-1} x
 * on device `device`, with L (CSC, strictly lower, rows ascending) and Dinv
 * in fact_prec (MPIR_F32 / MPIR_BF16 / MPIR_F16) and x in x_prec (MPIR_F64 or
 * MPIR_F32).  Accumulates in float64.  Returns a status. */
int mpir_qdldl_solve(int64_t n, const int64_t *Lp, const int64_t *Li,
                     const void *Lx, const void *Dinv, int fact_prec, void *x,
                     int x_prec, int device);

/* Replace QDLDL_Lsolve (qdldl.hpp:362-372, x <- (L+I)^{-1} x) and
 * QDLDL_Ltsolve (qdldl.hpp:389-400, x <- (L+I)^{-T} x); arguments as
 * mpir_qdldl_solve without Dinv. */
int mpir_qdldl_lsolve(int64_t n, const int64_t *Lp, const int64_t *Li,
                      const void *Lx, int fact_prec, void *x, int x_prec,
                      int device);
int mpir_qdldl_ltsolve(int64_t n, const int64_t *Lp, const int64_t *Li,
                       const void *Lx, int fact_prec, void *x, int x_prec,
                       int device);

/* QDLDL_solve without device allocation (no counterpart in the reference).
 * For callers that cannot call cudaMalloc: processes whose device memory is
 * reserved up front and handed out entirely by their own pooling allocator
 * (nothing is left for the library to allocate), and loops that must not
 * take cudaMalloc's implicit device-wide synchronisation.  Same
 * arithmetic as mpir_qdldl_solve (float32 L and Dinv, float64 x, host
 * arrays), but every device buffer it needs is carved out of one fixed 32 MiB
 * array that each GPU holds for as long as the library is loaded.  Limits:
 * every supernodal front of L has at most 64 rows, and the packed layout of
 * L, Dinv, x and the fronts' update vectors fits 32 MiB; otherwise it
 * returns MPIR_ERR_UNSUPPORTED or MPIR_ERR_ARGUMENT with a message and
 * touches no device memory.  The first call on a device looks up the array's
 * device address, so make it before any stream capture.  All calls share the
 * array: calls that overlap on the GPU (other host threads, other streams)
 * race and must be serialised by the caller.  Runs on the calling thread's
 * per-thread default stream and returns when x is back on the host; the
 * calling thread's current device is the same on return as before. */
int mpir_qdldl_solve_noalloc(int64_t n, const int64_t *Lp, const int64_t *Li,
                             const float *Lx, const float *Dinv, double *x,
                             int device);

/* ---- GMRES-IR solver (replaces GmresLDLIR, gmres_ir.hpp:90-315) --------- */

/* uf/uw/ur as MPIR_F* above.  Provided: uf = MPIR_F32 (float32 factor),
 * MPIR_BF16 or MPIR_F16 (factor whose trailing updates run on the tensor
 * cores with 16-bit operands and float32 accumulation; panels, diagonal
 * blocks and panel solves stay float32), or MPIR_F64, the reference
 * example's GmresLDLIR<double, double, dd_real> (examples/example.cpp:78-80):
 * the diagonal scaling uses eps(double) as the reference's Compute does
 * (gmres_ir.hpp:352) and the factor is the float32 one (refinement brings
 * the solution to the same backward error; rep.factor_prec says MPIR_F32);
 * uw = MPIR_F64; ur = MPIR_F64 or MPIR_DD. */
int mpir_solver_create(mpir_solver *out, int uf, int uw, int ur, int device);
int mpir_solver_destroy(mpir_solver s);

/* Setters of gmres_ir.hpp:291-303 (defaults 10, 10, 1e-10). */
int mpir_solver_set_max_ir_iterations(mpir_solver s, int64_t n);
int mpir_solver_set_max_gmres_iterations(mpir_solver s, int64_t n);
int mpir_solver_set_tolerance(mpir_solver s, double tol);

/* Compute (gmres_ir.hpp:271-278, 323-532): analyse with MPIR_ORDER_AUTO and
 * factor.  The reference's FGPILU ILU_k pattern level has no meaning for the
 * complete LDL^T factor and is not an argument. */
int mpir_solver_compute(mpir_solver s, int64_t n, const int64_t *Ap,
                        const int64_t *Ai, const double *Ax);
/* Symbolic analysis only.  Ax (may be NULL) only supplies the signs of the
 * diagonal, which split the ordering into the positive and the other block. */
int mpir_solver_analyze(mpir_solver s, int64_t n, const int64_t *Ap,
                        const int64_t *Ai, const double *Ax, int ordering);
/* New values on the analysed pattern (host / device pointer). */
int mpir_solver_factor(mpir_solver s, const double *Ax);
int mpir_solver_factor_device(mpir_solver s, const double *d_Ax);

/* Solve (gmres_ir.hpp:536-634): host / device vectors in the caller's
 * order.  rep may be NULL. */
int mpir_solver_solve(mpir_solver s, const double *b, double *x,
                      mpir_report *rep);
int mpir_solver_solve_device(mpir_solver s, const double *d_b, double *d_x,
                             mpir_report *rep);

/* The solver's log of the GMRES-IR solves since the previous dump, as JSON
 * text with the schema of the reference's GmresLDLIR::DumpLog under VERBOSE
 * (gmres_ir.hpp:305-313; one "gmres_ir" event per solve with
 * initial_residual, per refinement step {iteration, residual, d_norm,
 * timestamp_ms, inner_time_ms}, stop_reason, stop_reason_detail,
 * total_iterations, total_time_ms; then max_outer_iterations,
 * max_inner_iterations, tolerance).  *len receives the size including the
 * terminating NUL; when buf is NULL or cap < *len nothing is copied (call
 * again with a large enough buffer); a completed copy clears the log. */
int mpir_solver_dump_log(mpir_solver s, char *buf, int64_t cap, int64_t *len);

/* nrhs right-hand sides with the current factor: B and X hold nrhs
 * contiguous vectors of length n (column-major n x nrhs, host memory); one
 * GMRES-IR solve per column; reps (NULL, or nrhs reports) receives each
 * solve's report.  Stops at the first error.  The reference solves one
 * right-hand side per GmresLDLIR::Solve call (gmres_ir.hpp:534); this entry
 * point runs those solves in groups of up to 16 through
 * mpir_solver_solve_batch (a group of one through mpir_solver_solve). */
int mpir_solver_solve_many(mpir_solver s, int64_t nrhs, const double *B,
                           double *X, mpir_report *reps);

/* 1 <= nrhs <= 16 GMRES-IR solves with the current factor in lockstep: each
 * right-hand side follows GmresLDLIR::Solve (gmres_ir.hpp:534-634) with its
 * own Krylov basis, iteration counts and stop tests, while every
 * preconditioner application (QDLDL_solve, qdldl.hpp:417-432, applied once
 * per vector by the reference) is one several-vector triangular solve that
 * reads the factor once for all of them.  Results agree with one-at-a-time
 * mpir_solver_solve calls to rounding (each at backward error <= 1e-14 where
 * the single solve reaches it).  B and X column-major n x nrhs in the
 * caller's order, host (_batch) or device (_batch_device) memory; reps:
 * NULL or nrhs reports (solve_ms is the whole batch's time). */
int mpir_solver_solve_batch(mpir_solver s, int nrhs, const double *B,
                            double *X, mpir_report *reps);
int mpir_solver_solve_batch_device(mpir_solver s, int nrhs, const double *d_B,
                                   double *d_X, mpir_report *reps);

/* X <- (L D L^T)^{-1} X for 1 <= nrhs <= 16 vectors (n x nrhs column-major,
 * host memory) in the solver's internal order: the permuted, diagonally
 * scaled matrix the factor belongs to (mpir_solver_symbolic's perm).  The
 * preconditioner application of QDLDL_solve (qdldl.hpp:417-432); one vector
 * runs the single-vector kernels, several the several-vector kernels. */
int mpir_solver_apply_factor(mpir_solver s, int nrhs, double *X);

/* Failure-test controls of the bounded device waits of the triangular
 * solves: each wait gives up after 2^poll_log2 polls (0 restores the default
 * of about a second), and the forward work item withhold_item (-1: none)
 * never publishes its block result, so the waits on it run out and the
 * solve returns MPIR_ERR_TIMEOUT.  For tests of the timeout path only. */
int mpir_solver_set_wait_controls(mpir_solver s, int poll_log2, int withhold_item);

/* Plain iterative refinement with the LDL^T factor, LUIR_QDLDL
 * (qdldl-luir/luir.hpp:33-241) with float64 residual, working and solution
 * vectors: x0 = solve(b); r = b - A x; d = solve(r / |r|) |r|; x += d, until
 * |d| / |x_old| <= 10 eps(float64) or |d| / |d_prev| >= 1/2 (at most
 * maxiter steps; maxiter = 0: the single solve).  The right-hand side and
 * result of each solve are rounded to the factor's type, as the reference
 * keeps them in FACTPREC.  rep->ir_iterations = the reference's
 * num_refinement_steps_, rep->residual_norm = its relative_residual_
 * (|b - A x|_inf / |b|_inf), rep->precond_applies = solves.
 * mpir_solver_luir[_device] use the solver's current factor;
 * mpir_luir_qdldl analyses and factors A (upper CSC, caller order) first,
 * as the reference does, with fact_prec MPIR_F32, MPIR_BF16 or MPIR_F16. */
int mpir_solver_luir(mpir_solver s, const double *b, double *x, int maxiter,
                     mpir_report *rep);
int mpir_solver_luir_device(mpir_solver s, const double *d_b, double *d_x,
                            int maxiter, mpir_report *rep);

/* r = b - A x for the solver's current values (original, unscaled matrix;
 * b, x, r host arrays in caller order), the residual step of
 * GmresLDLIR::Solve (gmres_ir.hpp:550-551: MatrixMultiply<UR> then
 * VectorSubtract<UR>, ops.hpp:25-45 and :88-96) on the device: res_prec
 * MPIR_F64 in float64, MPIR_DD in double-double arithmetic (each product
 * exact, the sums in double-double) rounded to float64 at the end.
 * *rinf (may be NULL) = max|r|.  Needs a successful factorization (the
 * values are those it uploaded); MPIR_ERR_STATE before one. */
int mpir_solver_residual(mpir_solver s, const double *b, const double *x, double *r,
                         int res_prec, double *rinf);
int mpir_luir_qdldl(int64_t n, const int64_t *Ap, const int64_t *Ai,
                    const double *Ax, const double *b, double *x,
                    int fact_prec, int maxiter, mpir_report *rep, int device);

/* Trailing-update engine of a float32 factor (from the next factorization):
 * MPIR_UPDATE_TF32X3 (the default: three tf32 tensor-core products per
 * update, float32-level accuracy) or MPIR_UPDATE_BF16X3 (three bfloat16
 * products of high and low parts: about 16 significant bits, twice the
 * rate; a preconditioner for GMRES-IR, not a float32-accurate factor).
 * 16-bit factor types ignore it. */
enum { MPIR_UPDATE_DEFAULT = 0, MPIR_UPDATE_TF32X3 = 1, MPIR_UPDATE_BF16X3 = 2 };
int mpir_solver_set_update(mpir_solver s, int engine);

/* Launch the solver's work on a caller stream (a cudaStream_t; NULL
 * restores the solver's own stream). */
int mpir_solver_set_stream(mpir_solver s, void *stream);
int mpir_solver_info(mpir_solver s, mpir_info *info);

/* Permutation (perm[new] = old) and the elimination tree / column counts of
 * the permuted matrix, each n entries; Cp (n+1), Ci and Csrc (nnz_upper)
 * describe the permuted upper CSC and the source index of each entry.  Any
 * pointer may be NULL. */
int mpir_solver_symbolic(mpir_solver s, int64_t *perm, int64_t *etree,
                         int64_t *Lnz, int64_t *Cp, int64_t *Ci, int64_t *Csrc);

/* Supernode partition of the analysed pattern: sfirst (supernodes+1) column
 * ranges, srowptr (supernodes+1) and srows (srowptr[last]) the row index set
 * of each supernode (its own columns, then the rows below, ascending).  Any
 * pointer may be NULL; *nrows receives srowptr[last]. */
int mpir_solver_supernodes(mpir_solver s, int64_t *sfirst, int64_t *srowptr,
                           int32_t *srows, int64_t *nrows);

/* Factor in QDLDL's CSC form for the permuted matrix (Lp: n+1, Li/Lx: nnz_L,
 * D/Dinv: n, float32). */
int mpir_solver_export_factor(mpir_solver s, int64_t *Lp, int64_t *Li,
                              float *Lx, float *D, float *Dinv);

/* The leading k x k block of the factor (columns < k, rows < k) in QDLDL's
 * CSC form for the permuted matrix: Lp (k+1), Li/Lx (*nnz entries), D (k).
 * QDLDL_factor computes row r of L from rows < r (qdldl.hpp:228-342), so
 * this block is the reference's factor of the leading k x k block.  Pass
 * Li = Lx = NULL first to learn *nnz. */
int mpir_solver_export_factor_leading(mpir_solver s, int64_t k, int64_t *Lp,
                                      int64_t *Li, float *Lx, float *D,
                                      int64_t *nnz);

/* Host-only symbolic analysis (no device needed): the permutation, the
 * elimination tree and column counts of P K P^T, its upper CSC (Cp: n+1, Ci:
 * nnz_upper) and the exact pattern of L in QDLDL's CSC form (Lp: n+1, Li:
 * nnz_L; pass Li = NULL to size it first from info->nnz_L).  Any output may
 * be NULL.  Returns a status (-1 / -2 as QDLDL_etree). */
int mpir_analyze_host(int64_t n, const int64_t *Ap, const int64_t *Ai,
                      const double *Ax, int ordering, int64_t *perm,
                      int64_t *etree, int64_t *Lnz, int64_t *Cp, int64_t *Ci,
                      int64_t *Lp, int64_t *Li, mpir_info *info);

/* ---- Factor groups ------------------------------------------------------- */
/* k value sets on the pattern a solver has analysed, refactorized by one CUDA
 * graph launch: the reference factors one matrix per QDLDL_factor /
 * GmresLDLIR::Compute call (qdldl.hpp:172-345, gmres_ir.hpp:323); a group
 * records every member's factorization once, joins them as parallel branches
 * of one graph and replays it for every new set of values (same-pattern
 * instances such as interior-point iterations).  Members take the solver's
 * precisions and settings at creation and share its analysis; each has its
 * own factor storage. */
typedef struct mpir_group_s *mpir_group;

int mpir_group_create(mpir_group *out, mpir_solver s, int k);
/* Ax: k value sets of the analysed pattern (k x nnz_upper, row i for member
 * i, host, caller order).  npos: NULL or k entries receiving each factor's
 * positive pivots (-1 on a zero pivot).  Returns 0, or the first member's
 * failure (-1 zero pivot, -5 timeout). */
int mpir_group_factor(mpir_group g, const double *Ax, int64_t *npos);
/* GMRES-IR with member `member`'s factor: one right-hand side, or 1 .. 16 in
 * lockstep (as mpir_solver_solve / mpir_solver_solve_batch). */
int mpir_group_solve(mpir_group g, int member, const double *b, double *x,
                     mpir_report *rep);
int mpir_group_solve_batch(mpir_group g, int member, int nrhs, const double *B,
                           double *X, mpir_report *reps);
int mpir_group_destroy(mpir_group g);

/* ---- Serving engine ------------------------------------------------------ */
/* A request stream of GMRES-IR solves (each one the reference's
 * GmresLDLIR::Compute + Solve, gmres_ir.hpp:323 and :534-634) served on one
 * GPU by worker threads with a stream each.  Requests name their pattern and
 * values by caller-chosen keys; the engine keeps analysed patterns and
 * factors resident (when a new factor does not fit the device-memory
 * budget it evicts first what no queued request names, least recently used
 * first, then what the queue needs last), solves the queued requests on one
 * factor together (up to max_batch right-hand sides in lockstep, as
 * mpir_solver_solve_batch), and runs requests on different factors
 * concurrently.  A request whose factor alone exceeds the budget, or that
 * finds no room while every other running job waits for room too, or for
 * two minutes, is refused (status MPIR_ERR_NOMEM in its result). */
typedef struct mpir_server_s *mpir_server;

typedef struct mpir_server_config {
  int32_t device;
  int32_t uf;          /* MPIR_F32, MPIR_BF16 or MPIR_F16 */
  int32_t ur;          /* MPIR_F64 or MPIR_DD */
  int32_t workers;     /* concurrent jobs (host threads, one CUDA stream each) */
  int32_t max_batch;   /* right-hand sides per lockstep solve, 1 .. 16 */
  int32_t update;      /* MPIR_UPDATE_* engine of float32 factors */
  int64_t budget_bytes;           /* device memory for plans and factors */
  int64_t max_ir_iterations;      /* GmresLDLIR setters (gmres_ir.hpp:291-303) */
  int64_t max_gmres_iterations;
  double  tolerance;
} mpir_server_config;

/* The system (upper CSC in the caller's order), its right-hand side and the
 * output vector: all host arrays, valid until the request is done.
 * pattern_key names (n, Ap, Ai) and values_key the values Ax on it: equal
 * keys must mean equal arrays. */
typedef struct mpir_server_request {
  uint64_t       pattern_key, values_key;
  int64_t        n;
  const int64_t *Ap, *Ai;
  const double  *Ax, *b;
  double        *x;
} mpir_server_request;

typedef struct mpir_server_result {
  int64_t     id;
  int32_t     status;   /* as the solver's entry points */
  int32_t     path;     /* 0 resident factor, 1 refactorization, 2 new pattern */
  int32_t     batch;    /* right-hand sides solved in the same lockstep solve */
  int32_t     pad;
  double      latency_ms, queue_ms, service_ms;  /* submit -> done, -> start */
  mpir_report report;
} mpir_server_result;

typedef struct mpir_server_stats {
  int64_t submitted, completed, failed, refused;
  int64_t analyses, factorizations, solves, batched_solves, batched_rhs;
  int64_t evictions, resident_factors, resident_patterns, queued;
  int64_t bytes_in_use, peak_bytes;
  int64_t analysis_reuses;  /* plans rebuilt from the kept host analysis of an
                               evicted pattern (the ordering is not redone) */
  int64_t plan_uploads;     /* evicted plans uploaded again from their kept
                               host tables (nothing recomputed) */
  /* worker wall time summed over workers: host analysis, plan build and
   * upload, factorizations (allocation included), solves */
  double analysis_ms, plan_ms, factor_ms, solve_ms;
  double factor_device_ms, solve_device_ms;  /* CUDA-event time of those */
  double setup_ms, trim_ms;  /* parts of factor_ms: a new factor's solver and
                                resident buffers; the release of its
                                factorization scratch afterwards */
  double plan_upload_ms;     /* part of plan_ms: plans' arrays to the device */
} mpir_server_stats;

int mpir_server_create(mpir_server *out, const mpir_server_config *cfg);
/* Queues a request and returns at once with its id. */
int mpir_server_submit(mpir_server s, const mpir_server_request *r, int64_t *id);
/* Blocks until request id is done and returns its result (once). */
int mpir_server_wait(mpir_server s, int64_t id, mpir_server_result *res);
/* Blocks until every submitted request is done. */
int mpir_server_drain(mpir_server s);
int mpir_server_get_stats(mpir_server s, mpir_server_stats *out);
/* Drains, then frees every resident plan and factor. */
int mpir_server_destroy(mpir_server s);

/* ---- Kernel timing (benchmark support) ----------------------------------- */
/* Classes: 0 small fronts, 1 diagonal blocks, 2 panel solve, 3 trailing
 * update, 4 extend-add, 5 zero fill, 6 scatter, 7 forward solve, 8 backward
 * solve, 9 SpMV, 10 vector, 11 split-K reduction of the updates. */
int mpir_kernel_timer_enable(int on);
/* Kernel launches this library has issued in this process. */
int64_t mpir_launch_count(void);
int mpir_kernel_timer_collect(double *ms, int64_t *launches, int nclass);

#ifdef __cplusplus
}
#endif
#endif
