// Vector operations of the GMRES-IR loop (vec.cu).
#pragma once
#include <cstdint>
#include <cstring>

#include "engine.hpp"

namespace mpir {

// Owns the reduction scratch of one solver.  Max-norm results land in eight
// slots read back with read_inf: 0 residual, 1 |d|, 2 |x_old|, 3 |b_scaled|,
// 4..7 backward-error terms.
class VecOps {
 public:
  int64_t      n       = 0;
  int          nblocks = 1;
  DeviceBuffer part, count, infbits;

  int          batch   = 1;  // vectors the batched forms may take at once

  void allocate(int64_t n, int sms, int batch = 1);
  void spmv(const int64_t *Kp, const int32_t *Kj, const double *Kv, const double *x,
            double *y, cudaStream_t s);
  void residual(const int64_t *Kp, const int32_t *Kj, const double *Kv, const double *x,
                const double *b, double *r, bool dd, int slot, cudaStream_t s);
  void backward_terms(const int64_t *Kp, const int32_t *Kj, const double *Korig,
                      const double *x, const double *ADp, const double *bp,
                      cudaStream_t s);
  void mgs_pass(double *w, const double *v, const double *hsrc, const double *u, int mode,
                double *out, cudaStream_t s);
  void scale(const double *x, double a, double *y, cudaStream_t s);
  void combine(const double *V, int64_t ldv, int k, const double *y, double *res,
               cudaStream_t s);
  // d *= scale, x += d; infinity norms of d and of the old x (each entry
  // times w[i] when w is given: the norms of the unscaled vectors).
  void ir_update(double *d, double scale, double *x, cudaStream_t s,
                 const double *w = nullptr);
  // x <- x rounded to the factor's storage type (1 float32, 2 bfloat16,
  // 3 float16; float64 leaves x unchanged).
  void round_to(int prec, double *x, cudaStream_t s);
  void rhs_in(const int64_t *perm, const double *AD, const double *b, double *bs,
              double *ADp, double *bp, cudaStream_t s);
  void sol_out(const int64_t *perm, const double *ADp, const double *x, double *out,
               cudaStream_t s);
  void read_inf(double *h, int first, int cnt, cudaStream_t s);

  // Batched forms: nb vectors vs apart (k*vs for vector k), vector k's
  // max-norm slots in bank k (8 slots each, the same meaning as above),
  // vector k skipped where act[k] == 0 (act NULL: none skipped).  Per
  // vector the arithmetic is that of the single form.
  void spmv_b(int nb, const int64_t *Kp, const int32_t *Kj, const double *Kv, const double *x,
              double *y, int64_t vs, const int32_t *act, cudaStream_t s);
  void residual_b(int nb, const int64_t *Kp, const int32_t *Kj, const double *Kv,
                  const double *x, const double *b, double *r, bool dd, int64_t vs,
                  const int32_t *act, cudaStream_t s);
  void backward_terms_b(int nb, const int64_t *Kp, const int32_t *Kj, const double *Korig,
                        const double *x, const double *ADp, const double *bp, int64_t vs,
                        cudaStream_t s);
  // h and out of vector k at hsrc + k*hs and out + k*hs.
  void mgs_pass_b(int nb, double *w, const double *v, const double *hsrc, const double *u,
                  int mode, double *out, int64_t vs, int64_t hs, const int32_t *act,
                  cudaStream_t s);
  // y_k = x_k * fac[k] (fac on the device).
  void scale_b(int nb, const double *x, const double *fac, double *y, int64_t vs,
               const int32_t *act, cudaStream_t s);
  // res_k = sum_{j < kq[k]} V_j,k y[k*ys + j], V_j,k at V + j*ldv + k*vs.
  void combine_b(int nb, const double *V, int64_t ldv, const double *y, int64_t ys,
                 const int32_t *kq, double *res, int64_t vs, const int32_t *act,
                 cudaStream_t s);
  // d_k *= fac[k]; x_k += d_k; |d_k|, |x_k old| (weighted by w) into bank k.
  void ir_update_b(int nb, double *d, const double *fac, double *x, int64_t vs,
                   const int32_t *act, cudaStream_t s, const double *w = nullptr);
  void rhs_in_b(int nb, const int64_t *perm, const double *AD, const double *b, double *bs,
                double *ADp, double *bp, int64_t vs, cudaStream_t s);
  void sol_out_b(int nb, const int64_t *perm, const double *ADp, const double *x, double *out,
                 int64_t vs, cudaStream_t s);
  // All 8 slots of banks 0 .. nb-1 into h[8k + slot].
  void read_inf_b(int nb, double *h, cudaStream_t s);
};

}  // namespace mpir
