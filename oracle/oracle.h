/* Oracle: a plain-C restatement of the reference's CPU path (QDLDL LDL^T,
 * its triangular solves, the symmetric CSC SpMV, the BLAS-like helpers and
 * the GMRES-IR driver).  TEST INFRASTRUCTURE ONLY: the tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it as the checker; nothing in
 * the product links or calls it.  Each function cites the reference
 * file:line it restates.  All indices are int64_t. */
#ifndef MPIR_ORACLE_H
#define MPIR_ORACLE_H
#include <stdint.h>

typedef int64_t oi;

/* qdldl.hpp:48-105 */
oi oracle_etree(oi n, const oi *Ap, const oi *Ai, oi *work, oi *Lnz, oi *etree);
/* Per-row multiply-subtract counts of QDLDL_factor (qdldl.hpp:291-309). */
oi oracle_row_work(oi n, const oi *Ap, const oi *Ai, double *w);
/* qdldl.hpp:145-345, factor and arithmetic in double / float */
oi oracle_factor_f64(oi n, const oi *Ap, const oi *Ai, const double *Ax, oi *Lp,
                     oi *Li, double *Lx, double *D, double *Dinv,
                     const oi *Lnz, const oi *etree);
oi oracle_factor_f32(oi n, const oi *Ap, const oi *Ai, const double *Ax, oi *Lp,
                     oi *Li, float *Lx, float *D, float *Dinv, const oi *Lnz,
                     const oi *etree);
/* qdldl.hpp:362-432 */
void oracle_solve_f64_f64(oi n, const oi *Lp, const oi *Li, const double *Lx,
                          const double *Dinv, double *x);
void oracle_solve_f32_f64(oi n, const oi *Lp, const oi *Li, const float *Lx,
                          const float *Dinv, double *x);
void oracle_solve_f32_f32(oi n, const oi *Lp, const oi *Li, const float *Lx,
                          const float *Dinv, float *x);
/* ops.hpp:25-45 */
void   oracle_matmul(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                     const double *x, double *y);
/* ops.hpp:231-255 */
double oracle_dnrm2(oi n, const double *x);
/* ops.hpp:324-329 */
double oracle_infnrm(oi n, const double *x);
/* ops.hpp:195-200 */
double oracle_dot(oi n, const double *a, const double *b);
/* gmres_ir.hpp:347-363 */
void   oracle_scale(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                    double eps_uf, double *AD, double *Axs);

/* gmres_ir.hpp:536-741 with the LDL^T factor as the preconditioner.
 * Lx and Dinv hold the factor values already rounded to the factor type.
 * form 0: apply L, Dinv, L^T as QDLDL_solve does (qdldl.hpp:417-432), with
 *         the vectors in double.
 * form 1: apply the reference's TriangularSolve (gmres_ir.hpp:746-774) with
 *         L in CSR and U = D L^T in CSC; uf32 rounds U's values to float, as
 *         a float factor stored in the solver's UF members would be.
 * stats (may be NULL): {ir_steps, gmres_steps_total, reorth_count,
 *                       precond_applies, spmv_count}. */
int oracle_gmres_ir(oi n, const oi *Ap, const oi *Ai, const double *Axs,
                    const double *AD, const oi *Lp, const oi *Li,
                    const double *Lx, const double *D, const double *Dinv,
                    int form, int uf32, const double *b, double *x,
                    oi ir_iter, oi gmres_iter, double tol, double *stats);

/* qdldl-luir/luir.hpp:33-241, FACTPREC = float */
int oracle_luir_f32(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                    const double *b, double *x, int maxiter, double *info);

#endif
