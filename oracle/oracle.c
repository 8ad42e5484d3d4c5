/* Oracle: plain-C restatement of the reference's CPU path.  TEST
 * INFRASTRUCTURE ONLY (see oracle.h).  Written to reproduce the reference's
 * order of floating-point operations, so that with contraction off it agrees
 * bit for bit with the reference compiled from its own headers. */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define UNKNOWN (-1)

/* Elimination tree and column counts of an upper-CSC quasidefinite matrix.
 * qdldl.hpp:48-105: every column visits the tree path from each of its row
 * indices until it meets a node already stamped with this column; each
 * visited node gains one entry below the diagonal. */
oi oracle_etree(oi n, const oi *Ap, const oi *Ai, oi *work, oi *Lnz,
                oi *etree) {
  for (oi i = 0; i < n; i++) {
    work[i]  = 0;
    Lnz[i]   = 0;
    etree[i] = UNKNOWN;
    if (Ap[i] == Ap[i + 1]) return -1; /* empty column */
  }
  for (oi j = 0; j < n; j++) {
    work[j] = j;
    for (oi p = Ap[j]; p < Ap[j + 1]; p++) {
      oi i = Ai[p];
      if (i > j) return -1; /* entry below the diagonal */
      while (work[i] != j) {
        if (etree[i] == UNKNOWN) etree[i] = j;
        Lnz[i]++;
        work[i] = j;
        i       = etree[i];
      }
    }
  }
  oi total = 0;
  for (oi i = 0; i < n; i++) {
    if (total > INT64_MAX - Lnz[i]) return -2;
    total += Lnz[i];
  }
  return total;
}

/* Work of the up-looking factor row by row: w[k] = number of
 * multiply-subtract updates QDLDL_factor performs while computing row k of L
 * (qdldl.hpp:291-309: each column c in row k's reach costs the entries
 * already in column c).  Same tree walk as oracle_etree.  Used only to
 * extrapolate timed samples of the reference factor. */
oi oracle_row_work(oi n, const oi *Ap, const oi *Ai, double *w) {
  oi *mark = malloc(sizeof(oi) * (size_t)(n > 0 ? n : 1));
  oi *par  = malloc(sizeof(oi) * (size_t)(n > 0 ? n : 1));
  oi *cnt  = calloc((size_t)(n > 0 ? n : 1), sizeof(oi));
  for (oi i = 0; i < n; i++) {
    mark[i] = -1;
    par[i]  = UNKNOWN;
    w[i]    = 0.0;
  }
  for (oi k = 0; k < n; k++) {
    mark[k] = k;
    double acc = 0.0;
    for (oi p = Ap[k]; p < Ap[k + 1]; p++) {
      oi i = Ai[p];
      if (i > k) {
        free(mark);
        free(par);
        free(cnt);
        return -1;
      }
      while (mark[i] != k) {
        if (par[i] == UNKNOWN) par[i] = k;
        acc += (double)cnt[i];
        cnt[i]++;
        mark[i] = k;
        i       = par[i];
      }
    }
    w[k] = acc;
  }
  free(mark);
  free(par);
  free(cnt);
  return 0;
}

/* Up-looking LDL^T, qdldl.hpp:172-345.  Row k of L solves
 * L(0:k,0:k) y = A(0:k,k); the columns y touches are the etree reach of the
 * pattern of A(:,k), visited in topological order (reverse of the buffered
 * path lists).  Row entries are appended to their columns, so each column's
 * row indices come out ascending. */
#define DEFINE_FACTOR(NAME, T)                                                 \
  oi NAME(oi n, const oi *Ap, const oi *Ai, const double *Ax, oi *Lp, oi *Li,  \
          T *Lx, T *D, T *Dinv, const oi *Lnz, const oi *etree) {              \
    if (n <= 0) return 0;                                                      \
    unsigned char *mark  = calloc((size_t)n, 1);                               \
    oi            *reach = malloc(sizeof(oi) * (size_t)n);                     \
    oi            *path  = malloc(sizeof(oi) * (size_t)n);                     \
    oi            *next  = malloc(sizeof(oi) * (size_t)n);                     \
    T             *y     = malloc(sizeof(T) * (size_t)n);                      \
    oi             pos   = 0;                                                  \
    Lp[0]                = 0;                                                  \
    for (oi i = 0; i < n; i++) {                                               \
      Lp[i + 1] = Lp[i] + Lnz[i];                                              \
      y[i]      = (T)0;                                                        \
      D[i]      = (T)0;                                                        \
      next[i]   = Lp[i];                                                       \
    }                                                                          \
    D[0] = (T)Ax[0];                                                           \
    if (D[0] == (T)0) goto fail;                                               \
    if (D[0] > (T)0) pos++;                                                    \
    Dinv[0] = (T)1 / D[0];                                                     \
    for (oi k = 1; k < n; k++) {                                               \
      oi nr = 0;                                                               \
      for (oi p = Ap[k]; p < Ap[k + 1]; p++) {                                 \
        oi b = Ai[p];                                                          \
        if (b == k) {                                                          \
          D[k] = (T)Ax[p];                                                     \
          continue;                                                            \
        }                                                                      \
        y[b] = (T)Ax[p];                                                       \
        if (mark[b]) continue;                                                 \
        oi len    = 0;                                                         \
        mark[b]   = 1;                                                         \
        path[len++] = b;                                                       \
        for (oi c = etree[b]; c != UNKNOWN && c < k && !mark[c];               \
             c    = etree[c]) {                                                \
          mark[c]     = 1;                                                     \
          path[len++] = c;                                                     \
        }                                                                      \
        while (len) reach[nr++] = path[--len];                                 \
      }                                                                        \
      for (oi t = nr; t-- > 0;) {                                              \
        const oi c  = reach[t];                                                \
        const oi e  = next[c];                                                 \
        const T  yc = y[c];                                                    \
        for (oi q = Lp[c]; q < e; q++) {                                       \
          const T prod = Lx[q] * yc;                                           \
          y[Li[q]]     = y[Li[q]] - prod;                                      \
        }                                                                      \
        Li[e] = k;                                                             \
        Lx[e] = yc * Dinv[c];                                                  \
        D[k]  = D[k] - yc * Lx[e];                                             \
        next[c]++;                                                             \
        y[c]    = (T)0;                                                        \
        mark[c] = 0;                                                           \
      }                                                                        \
      if (D[k] == (T)0) goto fail;                                             \
      if (D[k] > (T)0) pos++;                                                  \
      Dinv[k] = (T)1 / D[k];                                                   \
    }                                                                          \
    free(mark);                                                                \
    free(reach);                                                               \
    free(path);                                                                \
    free(next);                                                                \
    free(y);                                                                   \
    return pos;                                                                \
  fail:                                                                        \
    free(mark);                                                                \
    free(reach);                                                               \
    free(path);                                                                \
    free(next);                                                                \
    free(y);                                                                   \
    return -1;                                                                 \
  }

DEFINE_FACTOR(oracle_factor_f64, double)
DEFINE_FACTOR(oracle_factor_f32, float)

/* (L+I) x = b by column scatter, x *= Dinv, (L+I)^T x = y by column gather;
 * qdldl.hpp:362-432.  Factor values are widened to the vector type. */
#define DEFINE_SOLVE(NAME, TF, TX)                                             \
  void NAME(oi n, const oi *Lp, const oi *Li, const TF *Lx, const TF *Dinv,    \
            TX *x) {                                                           \
    for (oi i = 0; i < n; i++) {                                               \
      const TX v = x[i];                                                       \
      for (oi j = Lp[i]; j < Lp[i + 1]; j++)                                   \
        x[Li[j]] = x[Li[j]] - (TX)Lx[j] * v;                                   \
    }                                                                          \
    for (oi i = 0; i < n; i++) x[i] = x[i] * (TX)Dinv[i];                      \
    for (oi i = n; i-- > 0;) {                                                 \
      TX v = x[i];                                                             \
      for (oi j = Lp[i]; j < Lp[i + 1]; j++) v = v - (TX)Lx[j] * x[Li[j]];     \
      x[i] = v;                                                                \
    }                                                                          \
  }

DEFINE_SOLVE(oracle_solve_f64_f64, double, double)
DEFINE_SOLVE(oracle_solve_f32_f64, float, double)
DEFINE_SOLVE(oracle_solve_f32_f32, float, float)

/* y = K x from the upper triangle in CSC, ops.hpp:25-45: entry (r, c) adds
 * a*x[r] to y[c] and, off the diagonal, a*x[c] to y[r]. */
void oracle_matmul(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                   const double *x, double *y) {
  for (oi i = 0; i < n; i++) y[i] = 0.0;
  for (oi c = 0; c < n; c++)
    for (oi p = Ap[c]; p < Ap[c + 1]; p++) {
      const oi r = Ai[p];
      y[c]       = y[c] + Ax[p] * x[r];
      if (r < c) y[r] = y[r] + Ax[p] * x[c];
    }
}

/* Scaled sum of squares walked from the last element to the first,
 * ops.hpp:231-255. */
double oracle_dnrm2(oi n, const double *x) {
  if (n == 0) return 0.0;
  if (n == 1) return fabs(x[0]);
  double scale = 0.0, ssq = 1.0;
  for (oi i = n; i-- > 0;) {
    if (x[i] != 0.0) {
      const double a = fabs(x[i]);
      if (scale < a) {
        ssq   = 1.0 + ssq * ((scale / a) * (scale / a));
        scale = a;
      } else {
        ssq = ssq + ((a / scale) * (a / scale));
      }
    }
  }
  return scale * sqrt(ssq);
}

/* max |x_i|, ops.hpp:324-329 (an empty vector is not allowed there). */
double oracle_infnrm(oi n, const double *x) {
  double m = 0.0;
  for (oi i = 0; i < n; i++)
    if (fabs(x[i]) > m) m = fabs(x[i]);
  return m;
}

/* VectorDot, ops.hpp:195-200: std::transform_reduce as libstdc++ 13 runs it
 * for random-access ranges, which folds blocks of four as
 * acc + ((p0 + p1) + (p2 + p3)) and then the tail one by one. */
double oracle_dot(oi n, const double *a, const double *b) {
  double acc = 0.0;
  oi     i   = 0;
  for (; n - i >= 4; i += 4) {
    const double v1 = a[i] * b[i] + a[i + 1] * b[i + 1];
    const double v2 = a[i + 2] * b[i + 2] + a[i + 3] * b[i + 3];
    acc             = acc + (v1 + v2);
  }
  for (; i < n; i++) acc = acc + a[i] * b[i];
  return acc;
}

/* Symmetric diagonal scaling, gmres_ir.hpp:347-363: d_i = 1/sqrt|a_ii| when
 * |a_ii| exceeds the factor type's epsilon, else 1; a_rc *= d_r * d_c. */
void oracle_scale(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                  double eps_uf, double *AD, double *Axs) {
  for (oi i = 0; i < n; i++) AD[i] = 1.0;
  for (oi c = 0; c < n; c++)
    for (oi p = Ap[c]; p < Ap[c + 1]; p++)
      if (Ai[p] == c && fabs(Ax[p]) > eps_uf) AD[c] = 1.0 / sqrt(fabs(Ax[p]));
  for (oi c = 0; c < n; c++)
    for (oi p = Ap[c]; p < Ap[c + 1]; p++)
      Axs[p] = Ax[p] * (AD[Ai[p]] * AD[c]);
}

/* ---------------------------------------------------------------------------
 * GMRES-IR, gmres_ir.hpp:536-741. */
typedef struct {
  oi            n;
  const oi     *Ap, *Ai;
  const double *Ax;
  int           form;
  /* form 0: CSC factor */
  const oi     *Lp, *Li;
  const double *Lx, *Dinv;
  /* form 1: CSR of strictly lower L and CSC of U = D L^T (same index arrays) */
  oi           *Rp, *Rc;
  double       *Rx, *Ux;
  oi            gmres_iter;
  double        tol;
  double        stats[5];
} gmres_ctx;

static void precond(gmres_ctx *g, const double *b, double *out) {
  const oi n = g->n;
  g->stats[3] += 1;
  if (g->form == 0) {
    memcpy(out, b, sizeof(double) * (size_t)n);
    oracle_solve_f64_f64(n, g->Lp, g->Li, g->Lx, g->Dinv, out);
    return;
  }
  /* TriangularSolve, gmres_ir.hpp:746-774 */
  for (oi r = 0; r < n; r++) {
    double s = 0.0;
    for (oi q = g->Rp[r]; q < g->Rp[r + 1]; q++)
      if (g->Rc[q] < r) s = s + g->Rx[q] * out[g->Rc[q]];
    out[r] = b[r] - s;
  }
  for (oi c = n; c-- > 0;) {
    out[c] = out[c] * g->Dinv[c];
    for (oi q = g->Rp[c]; q < g->Rp[c + 1]; q++)
      if (g->Rc[q] < c) out[g->Rc[q]] = out[g->Rc[q]] - g->Ux[q] * out[c];
  }
}

static void spmv(gmres_ctx *g, const double *x, double *y) {
  g->stats[4] += 1;
  oracle_matmul(g->n, g->Ap, g->Ai, g->Ax, x, y);
}

/* PrecondGmres, gmres_ir.hpp:636-741 (writes the correction into res). */
static void precond_gmres(gmres_ctx *g, const double *b, double *res) {
  const oi n = g->n;
  if (g->gmres_iter > n) g->gmres_iter = n;
  const oi m = g->gmres_iter;
  for (oi i = 0; i < n; i++) res[i] = 0.0;
  double rho = oracle_dnrm2(n, b);
  if (rho < g->tol) return;

  double *V  = malloc(sizeof(double) * (size_t)n * (size_t)(m + 1));
  double *h  = calloc((size_t)(m + 1) * (size_t)(m > 0 ? m : 1), sizeof(double));
  double *gv = calloc((size_t)(m + 1), sizeof(double));
  double *c  = calloc((size_t)(m > 0 ? m : 1), sizeof(double));
  double *s  = calloc((size_t)(m > 0 ? m : 1), sizeof(double));
  double *y  = calloc((size_t)(m > 0 ? m : 1), sizeof(double));
#define H(i, j) h[(size_t)(i) * (size_t)(m > 0 ? m : 1) + (size_t)(j)]
#define VK(k) (V + (size_t)(k) * (size_t)n)

  precond(g, b, VK(0));
  rho = oracle_dnrm2(n, VK(0));
  {
    const double inv = 1 / rho;
    for (oi i = 0; i < n; i++) VK(0)[i] = VK(0)[i] * inv;
  }
  gv[0] = rho;

  oi k;
  for (k = 0; k < m && rho > g->tol; k++) {
    double *w = VK(k + 1);
    double *t = malloc(sizeof(double) * (size_t)n);
    spmv(g, VK(k), t);
    precond(g, t, w);
    free(t);
    const double normav = oracle_dnrm2(n, w);
    for (oi j = 0; j <= k; j++) {
      H(j, k)        = oracle_dot(n, w, VK(j));
      const double hj = H(j, k);
      for (oi i = 0; i < n; i++) w[i] = w[i] - VK(j)[i] * hj;
    }
    double normav2 = H(k + 1, k) = oracle_dnrm2(n, w);
    if (normav + 0.001 * normav2 == normav) {
      g->stats[2] += 1;
      for (oi j = 0; j <= k; j++) {
        const double hr = oracle_dot(n, w, VK(j));
        H(j, k)         = H(j, k) + hr;
        for (oi i = 0; i < n; i++) w[i] = w[i] - VK(j)[i] * hr;
      }
      H(k + 1, k) = oracle_dnrm2(n, w);
    }
    if (H(k + 1, k) != 0) {
      const double inv = 1 / H(k + 1, k);
      for (oi i = 0; i < n; i++) w[i] = w[i] * inv;
    }
    for (oi j = 0; j < k; j++) {
      const double w1 = c[j] * H(j, k) - s[j] * H(j + 1, k);
      const double w2 = s[j] * H(j, k) + c[j] * H(j + 1, k);
      H(j, k)         = w1;
      H(j + 1, k)     = w2;
    }
    const double pair[2] = {H(k, k), H(k + 1, k)};
    const double nu      = oracle_dnrm2(2, pair);
    if (nu != 0) {
      c[k]            = H(k, k) / nu;
      s[k]            = -H(k + 1, k) / nu;
      H(k, k)         = c[k] * H(k, k) - s[k] * H(k + 1, k);
      H(k + 1, k)     = 0.0;
      const double w1 = c[k] * gv[k] - s[k] * gv[k + 1];
      const double w2 = s[k] * gv[k] + c[k] * gv[k + 1];
      gv[k]           = w1;
      gv[k + 1]       = w2;
    }
    rho = fabs(gv[k + 1]);
  }
  g->stats[1] += (double)k;
  for (oi i = k; i-- > 0;) {
    y[i] = gv[i];
    for (oi j = i + 1; j < k; j++) y[i] = y[i] - H(i, j) * y[j];
    y[i] = y[i] / H(i, i);
  }
  for (oi i = 0; i < n; i++)
    for (oi j = 0; j < k; j++) res[i] = res[i] + VK(j)[i] * y[j];
#undef H
#undef VK
  free(V);
  free(h);
  free(gv);
  free(c);
  free(s);
  free(y);
}

int oracle_gmres_ir(oi n, const oi *Ap, const oi *Ai, const double *Axs,
                    const double *AD, const oi *Lp, const oi *Li,
                    const double *Lx, const double *D, const double *Dinv,
                    int form, int uf32, const double *b, double *x,
                    oi ir_iter, oi gmres_iter, double tol, double *stats) {
  gmres_ctx g;
  memset(&g, 0, sizeof g);
  g.n = n, g.Ap = Ap, g.Ai = Ai, g.Ax = Axs, g.form = form;
  g.Lp = Lp, g.Li = Li, g.Lx = Lx, g.Dinv = Dinv;
  g.gmres_iter = gmres_iter, g.tol = tol;
  const oi nl  = Lp[n];
  if (form == 1) {
    g.Rp = calloc((size_t)n + 1, sizeof(oi));
    g.Rc = malloc(sizeof(oi) * (size_t)(nl > 0 ? nl : 1));
    g.Rx = malloc(sizeof(double) * (size_t)(nl > 0 ? nl : 1));
    g.Ux = malloc(sizeof(double) * (size_t)(nl > 0 ? nl : 1));
    oi *fill = malloc(sizeof(oi) * (size_t)(n > 0 ? n : 1));
    for (oi p = 0; p < nl; p++) g.Rp[Li[p] + 1]++;
    for (oi i = 0; i < n; i++) g.Rp[i + 1] += g.Rp[i];
    for (oi i = 0; i < n; i++) fill[i] = g.Rp[i];
    for (oi j = 0; j < n; j++)
      for (oi p = Lp[j]; p < Lp[j + 1]; p++) {
        const oi q = fill[Li[p]]++;
        g.Rc[q]    = j;
        g.Rx[q]    = Lx[p];
        g.Ux[q]    = uf32 ? (double)((float)D[j] * (float)Lx[p]) : D[j] * Lx[p];
      }
    free(fill);
  }

  double *bs = malloc(sizeof(double) * (size_t)n);
  double *r  = malloc(sizeof(double) * (size_t)n);
  double *t  = malloc(sizeof(double) * (size_t)n);
  double *d  = malloc(sizeof(double) * (size_t)n);
  for (oi i = 0; i < n; i++) bs[i] = b[i] * AD[i];

  precond_gmres(&g, bs, x);
  spmv(&g, x, t);
  for (oi i = 0; i < n; i++) r[i] = bs[i] - t[i];
  double r_prev = 1.79769313486231570815e+308; /* DBL_MAX */
  oi     iter;
  for (iter = 1; iter <= ir_iter; iter++) {
    const double scale = oracle_infnrm(n, r);
    const double inv   = 1.0 / scale;
    for (oi i = 0; i < n; i++) t[i] = r[i] * inv;
    precond_gmres(&g, t, d);
    for (oi i = 0; i < n; i++) d[i] = d[i] * scale;
    const double d_norm = oracle_infnrm(n, d);
    const double x_norm = oracle_infnrm(n, x);
    for (oi i = 0; i < n; i++) x[i] = x[i] + d[i];
    spmv(&g, x, t);
    for (oi i = 0; i < n; i++) r[i] = bs[i] - t[i];
    const double r_norm = oracle_infnrm(n, r) / oracle_infnrm(n, bs);
    g.stats[0] += 1;
    if (d_norm <= x_norm * (10 * 2.220446049250313e-16)) break;
    if (fabs(r_norm - r_prev) < tol) break;
    r_prev = r_norm;
  }
  for (oi i = 0; i < n; i++) x[i] = x[i] * AD[i];
  if (stats) memcpy(stats, g.stats, sizeof g.stats);
  free(bs);
  free(r);
  free(t);
  free(d);
  free(g.Rp);
  free(g.Rc);
  free(g.Rx);
  free(g.Ux);
  return 0;
}

/* ------------------------------------------------------------------------
 * LUIR_QDLDL<float, double, double, double> (qdldl-luir/luir.hpp:33-241):
 * QDLDL factor of A in float (natural order), then plain iterative
 * refinement.  The residual (qdldl-luir/residual.hpp:15-41: the same loop as
 * MatrixMultiply, in double) is stored in float, scaled by 1/|r|, solved in
 * float and scaled back; x += d in double; stop when |d|/|x| <= 10 eps(double)
 * or |d|/|d_prev| >= 0.5.  info = {steps, |b - A x|/|b| (residual stored in
 * float, as the reference), nnz(L)}.  Returns -1 on a structural error or
 * zero pivot. */
static double inf_norm_f(oi n, const float *x) {
  float m = 0.0f;
  for (oi i = 0; i < n; i++) {
    const float a = x[i] >= 0 ? x[i] : -x[i];
    if (a > m) m = a;
  }
  return (double)m;
}

static double inf_norm_d(oi n, const double *x) {
  double m = 0.0;
  for (oi i = 0; i < n; i++) {
    const double a = x[i] >= 0 ? x[i] : -x[i];
    if (a > m) m = a;
  }
  return m;
}

/* residual (float) = b - A x, accumulated in double */
static void residual_f(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                       const double *x, const double *b, double *work, float *res) {
  oracle_matmul(n, Ap, Ai, Ax, x, work);
  for (oi i = 0; i < n; i++) res[i] = (float)(b[i] - work[i]);
}

int oracle_luir_f32(oi n, const oi *Ap, const oi *Ai, const double *Ax,
                    const double *b, double *x, int maxiter, double *info) {
  oi *iwork = malloc(sizeof(oi) * 3 * (size_t)(n > 0 ? n : 1));
  oi *Lnz = malloc(sizeof(oi) * (size_t)(n > 0 ? n : 1));
  oi *et = malloc(sizeof(oi) * (size_t)(n > 0 ? n : 1));
  const oi sum = oracle_etree(n, Ap, Ai, iwork, Lnz, et);
  if (sum < 0) {
    free(iwork); free(Lnz); free(et);
    return -1;
  }
  oi    *Lp = malloc(sizeof(oi) * (size_t)(n + 1));
  oi    *Li = malloc(sizeof(oi) * (size_t)(sum > 0 ? sum : 1));
  float *Lx = malloc(sizeof(float) * (size_t)(sum > 0 ? sum : 1));
  float *D = malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
  float *Dinv = malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
  const oi pos = oracle_factor_f32(n, Ap, Ai, Ax, Lp, Li, Lx, D, Dinv, Lnz, et);
  float  *cf = malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
  double *work = malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  int     steps = 0, rc = pos < 0 ? -1 : 0;
  if (rc == 0) {
    if (maxiter == 0) {
      /* luir.hpp:171-179: one solve with x in double */
      for (oi i = 0; i < n; i++) x[i] = b[i];
      oracle_solve_f32_f64(n, Lp, Li, Lx, Dinv, x);
    } else {
      /* luir.hpp:182-232 */
      for (oi i = 0; i < n; i++) cf[i] = (float)b[i];
      oracle_solve_f32_f32(n, Lp, Li, Lx, Dinv, cf);
      for (oi i = 0; i < n; i++) x[i] = (double)cf[i];
      const double eps = 2.220446049250313e-16, thresh = 0.5;
      double       d0 = 1.7976931348623157e308;
      for (int it = 1; it <= maxiter; it++) {
        residual_f(n, Ap, Ai, Ax, x, b, work, cf);
        const double nc = inf_norm_f(n, cf);
        for (oi i = 0; i < n; i++) cf[i] *= 1. / nc;
        oracle_solve_f32_f32(n, Lp, Li, Lx, Dinv, cf);
        for (oi i = 0; i < n; i++) cf[i] *= nc;
        const double dn = inf_norm_f(n, cf), xn = inf_norm_d(n, x);
        const int    stop = dn / xn <= 10 * eps || dn / d0 >= thresh;
        steps = it;
        for (oi i = 0; i < n; i++) x[i] = (double)cf[i] + x[i];
        if (stop) break;
        d0 = dn;
      }
    }
    residual_f(n, Ap, Ai, Ax, x, b, work, cf);
    info[1] = inf_norm_f(n, cf) / inf_norm_d(n, b);
  }
  info[0] = steps;
  info[2] = (double)sum;
  free(iwork); free(Lnz); free(et); free(Lp); free(Li); free(Lx); free(D); free(Dinv);
  free(cf); free(work);
  return rc;
}
