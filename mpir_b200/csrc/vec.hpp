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

  void allocate(int64_t n, int sms);
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
};

}  // namespace mpir
