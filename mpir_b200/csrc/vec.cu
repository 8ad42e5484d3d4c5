// Vector kernels of the GMRES-IR loop: the symmetric SpMV and residual in
// float64 or double-double (MatrixMultiply / VectorSubtract, ops.hpp:25-96),
// norms (Dnrm2 / InfNrm, ops.hpp:231-329), dot products (ops.hpp:195-200),
// the fused modified Gram-Schmidt passes of PrecondGmres
// (gmres_ir.hpp:676-691) and the refinement update (gmres_ir.hpp:562-579).
//
// Sums and norms are two-stage reductions whose second stage adds the
// per-block partials in block order, so results are reproducible.
#include <cfloat>
#include <cmath>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "vec.hpp"

namespace mpir {

constexpr int kRedThreads = 256;

// ---------------------------------------------------------------------------
// Double-double helpers (Knuth's TwoSum and the FMA form of Dekker's
// TwoProduct): a value is the unevaluated sum hi + lo.
struct dd {
  double hi, lo;
};
__device__ __forceinline__ dd two_sum(double a, double b) {
  const double s  = a + b;
  const double bb = s - a;
  const double e  = (a - (s - bb)) + (b - bb);
  return {s, e};
}
__device__ __forceinline__ dd quick_two_sum(double a, double b) {
  const double s = a + b;
  return {s, b - (s - a)};
}
__device__ __forceinline__ dd two_prod(double a, double b) {
  const double p = a * b;
  return {p, fma(a, b, -p)};
}
__device__ __forceinline__ dd dd_add(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi);
  dd t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}

__device__ __forceinline__ void atomic_max_abs(unsigned long long *slot, double v) {
  atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(fabs(v))));
}

// Max of |v| over the warp, then one atomic per warp.  The maximum is taken
// on the bit patterns of |v| (non-negative doubles order as their bits), so a
// NaN (whose |v| pattern lies above infinity's) wins and is reported: fmax
// would drop it and a non-finite residual would pass for a small one.
__device__ __forceinline__ void warp_max_abs(unsigned long long *slot, double v,
                                             bool active) {
  unsigned long long a =
      active ? static_cast<unsigned long long>(__double_as_longlong(fabs(v))) : 0ull;
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long b = __shfl_xor_sync(0xffffffffu, a, o);
    a                          = b > a ? b : a;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(slot, a);
}

// ---------------------------------------------------------------------------
// SpMV with G lanes per row over the full symmetric CSR.
//   MODE 0: y = K x
//   MODE 1: y = b - K x,           max|y| into inf[0]
//   MODE 2: y = b - K x in double-double, rounded to float64, max into inf[0]
//
// Batched form (all kernels below): blockIdx.y selects vector k of a batch,
// the vectors k*vs apart, its max-norm slots at inf + 8k, and k is skipped
// when act[k] == 0 (act NULL: every k).  One vector is gridDim.y == 1.
__device__ __forceinline__ bool batch_skip(const int32_t *vact) {
  return vact != nullptr && vact[blockIdx.y] == 0;
}

template <int G, int MODE>
__global__ void k_spmv(int64_t n, const int64_t *Kp, const int32_t *Kj,
                       const double *Kv, const double *x, const double *b,
                       double *y, unsigned long long *inf, int64_t vs,
                       const int32_t *vact) {
  if (batch_skip(vact)) return;
  x += blockIdx.y * vs;
  y += blockIdx.y * vs;
  if (b) b += blockIdx.y * vs;
  if (inf) inf += 8 * blockIdx.y;
  const int64_t gid  = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t row  = gid / G;
  const int     lane = threadIdx.x % G;
  const bool    act  = row < n;
  if (MODE == 2) {
    dd s{0.0, 0.0};
    if (act)
      for (int64_t e = Kp[row] + lane; e < Kp[row + 1]; e += G)
        s = dd_add(s, two_prod(Kv[e], x[Kj[e]]));
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      dd t{__shfl_xor_sync(0xffffffffu, s.hi, o, G),
           __shfl_xor_sync(0xffffffffu, s.lo, o, G)};
      s = dd_add(s, t);
    }
    double r = 0.0;
    if (act && lane == 0) {
      dd rr = dd_add(dd{b[row], 0.0}, dd{-s.hi, -s.lo});
      r     = rr.hi + rr.lo;
      y[row] = r;
    }
    warp_max_abs(inf, r, act && lane == 0);
    return;
  }
  double s = 0.0;
  if (act)
    for (int64_t e = Kp[row] + lane; e < Kp[row + 1]; e += G) s += Kv[e] * x[Kj[e]];
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, G);
  if (MODE == 0) {
    if (act && lane == 0) y[row] = s;
  } else {
    double r = 0.0;
    if (act && lane == 0) {
      r      = b[row] - s;
      y[row] = r;
    }
    warp_max_abs(inf, r, act && lane == 0);
  }
}

// Backward-error terms on the original (unscaled) system in permuted order:
// inf = {max|b - K xo|, max_i sum_j |k_ij|, max|xo|, max|b|}, where
// xo = x .* ADp.
template <int G>
__global__ void k_backward_terms(int64_t n, const int64_t *Kp, const int32_t *Kj,
                                 const double *Korig, const double *x,
                                 const double *ADp, const double *b,
                                 unsigned long long *inf, int64_t vs,
                                 const int32_t *vact) {
  if (batch_skip(vact)) return;
  x += blockIdx.y * vs;
  b += blockIdx.y * vs;
  inf += 8 * blockIdx.y;
  const int64_t gid  = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t row  = gid / G;
  const int     lane = threadIdx.x % G;
  const bool    act  = row < n;
  double        s = 0.0, a = 0.0;
  if (act)
    for (int64_t e = Kp[row] + lane; e < Kp[row + 1]; e += G) {
      const int32_t j = Kj[e];
      s += Korig[e] * (x[j] * ADp[j]);
      a += fabs(Korig[e]);
    }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o, G);
    a += __shfl_xor_sync(0xffffffffu, a, o, G);
  }
  const bool lead = act && lane == 0;
  warp_max_abs(inf + 0, lead ? b[row] - s : 0.0, lead);
  warp_max_abs(inf + 1, lead ? a : 0.0, lead);
  warp_max_abs(inf + 2, lead ? x[row] * ADp[row] : 0.0, lead);
  warp_max_abs(inf + 3, lead ? b[row] : 0.0, lead);
}

// ---------------------------------------------------------------------------
// Two-stage reductions.  Stage 1 writes one partial per block; the last block
// to finish combines them in block order and resets the counter.
__device__ __forceinline__ double block_sum(double v, double *sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int q = 0; q < (int)(blockDim.x / 32); q++) t += sh[q];
  return t;
}

// LAPACK-style scaled sum of squares: the pair (scale, ssq) stands for
// scale^2 * ssq.
__device__ __forceinline__ void ssq_add(double &scale, double &ssq, double x) {
  if (x != 0.0) {
    const double a = fabs(x);
    if (scale < a) {
      ssq   = 1.0 + ssq * ((scale / a) * (scale / a));
      scale = a;
    } else {
      ssq += (a / scale) * (a / scale);
    }
  }
}
__device__ __forceinline__ void ssq_merge(double &s1, double &q1, double s2, double q2) {
  if (s2 == 0.0) return;
  if (s1 == 0.0) {
    s1 = s2;
    q1 = q2;
    return;
  }
  if (s1 >= s2) {
    q1 += q2 * ((s2 / s1) * (s2 / s1));
  } else {
    q1 = q2 + q1 * ((s1 / s2) * (s1 / s2));
    s1 = s2;
  }
}
__device__ __forceinline__ void block_ssq(double &s, double &q, double *sh) {
  for (int o = 16; o > 0; o >>= 1) {
    const double s2 = __shfl_xor_sync(0xffffffffu, s, o);
    const double q2 = __shfl_xor_sync(0xffffffffu, q, o);
    ssq_merge(s, q, s2, q2);
  }
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();
  if (lane == 0) {
    sh[2 * warp]     = s;
    sh[2 * warp + 1] = q;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s = 0.0;
    q = 1.0;
    for (int w = 0; w < (int)(blockDim.x / 32); w++) ssq_merge(s, q, sh[2 * w], sh[2 * w + 1]);
  }
}

// Finalisation helper: returns true in thread 0 of the last block.
__device__ __forceinline__ bool last_block(unsigned int *count) {
  __shared__ bool is_last;
  __threadfence();
  if (threadIdx.x == 0) is_last = atomicInc(count, gridDim.x) == gridDim.x - 1;
  __syncthreads();
  return is_last;
}

// MGS pass: w -= h * v (h read from *hsrc, skipped when hsrc is null), then
// either dot(w, u) (mode 0) or ||w||_2 (mode 1) into *out.
// Batched: vectors k*vs apart, h and out k*hs apart, scratch part + 2048 k
// and count + k.
__global__ void __launch_bounds__(kRedThreads)
    k_mgs_pass(int64_t n, double *w, const double *v, const double *hsrc,
               const double *u, int mode, double *part, unsigned int *count,
               double *out, int64_t vs, int64_t hs, const int32_t *vact) {
  __shared__ double sh[2 * kRedThreads / 32];
  if (batch_skip(vact)) return;
  {
    const int64_t k = blockIdx.y;
    w += k * vs;
    if (v) v += k * vs;
    if (u) u += k * vs;
    if (hsrc) hsrc += k * hs;
    out += k * hs;
    part += 2048 * k;
    count += k;
  }
  const double      h = hsrc ? *hsrc : 0.0;
  double            acc = 0.0, sc = 0.0, sq = 1.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double wi = w[i];
    if (hsrc) {
      wi   = wi - v[i] * h;
      w[i] = wi;
    }
    if (mode == 0)
      acc += wi * u[i];
    else
      ssq_add(sc, sq, wi);
  }
  if (mode == 0) {
    const double t = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
  } else {
    block_ssq(sc, sq, sh);
    if (threadIdx.x == 0) {
      part[2 * blockIdx.x]     = sc;
      part[2 * blockIdx.x + 1] = sq;
    }
  }
  if (!last_block(count)) return;
  // The last block adds the blocks' partials: thread j takes partials j,
  // j + blockDim.x, ... in that order, then the fixed tree of the block
  // reductions (the loads are independent, so none waits for another).
  if (mode == 0) {
    double t = 0.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += __ldcg(part + b);
    t = block_sum(t, sh);
    if (threadIdx.x == 0) *out = t;
  } else {
    double s = 0.0, q = 1.0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
      ssq_merge(s, q, __ldcg(part + 2 * b), __ldcg(part + 2 * b + 1));
    block_ssq(s, q, sh);
    if (threadIdx.x == 0) *out = s * sqrt(q);
  }
  if (threadIdx.x == 0) *count = 0;
}

// y = a * x (a the host argument, or fac[k] for vector k when fac is given).
__global__ void k_scale(int64_t n, const double *x, double a, double *y, int64_t vs,
                        const double *fac, const int32_t *vact) {
  if (batch_skip(vact)) return;
  x += blockIdx.y * vs;
  y += blockIdx.y * vs;
  if (fac) a = fac[blockIdx.y];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i] * a;
}

// res = sum_j V_j y_j for j < k (gmres_ir.hpp:735-739).
// Batched: vector q's basis at V + q*vs (ldv apart), its coefficients at
// y + q*ys and its count kq[q] (kq NULL: k for all).
__global__ void k_combine(int64_t n, const double *V, int64_t ldv, int k,
                          const double *y, double *res, int64_t vs, int64_t ys,
                          const int32_t *kq, const int32_t *vact) {
  if (batch_skip(vact)) return;
  V += blockIdx.y * vs;
  res += blockIdx.y * vs;
  y += blockIdx.y * ys;
  if (kq) k = kq[blockIdx.y];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double r = 0.0;
  for (int j = 0; j < k; j++) r += V[j * ldv + i] * y[j];
  res[i] = r;
}

// d *= scale; inf[0] = max|d|; inf[1] = max|x_old|; x += d
// (gmres_ir.hpp:574-577).
__global__ void k_ir_update(int64_t n, double *d, double scale, double *x,
                            const double *w, unsigned long long *inf, int64_t vs,
                            const double *fac, const int32_t *vact) {
  if (batch_skip(vact)) return;
  d += blockIdx.y * vs;
  x += blockIdx.y * vs;
  inf += 8 * blockIdx.y;
  if (fac) scale = fac[blockIdx.y];
  const int64_t i   = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool    act = i < n;
  double        di = 0.0, xi = 0.0, wi = 1.0;
  if (act) {
    di   = d[i] * scale;
    xi   = x[i];
    d[i] = di;
    x[i] = xi + di;
    if (w) wi = w[i];
  }
  warp_max_abs(inf + 0, di * wi, act);
  warp_max_abs(inf + 1, xi * wi, act);
}

// x <- x rounded to float32 (1), bfloat16 (2) or float16 (3).
__global__ void k_round_to(int64_t n, int prec, double *x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  if (prec == 1)
    x[i] = static_cast<double>(__double2float_rn(v));
  else if (prec == 2)
    x[i] = static_cast<double>(__bfloat162float(__double2bfloat16(v)));
  else if (prec == 3)
    x[i] = static_cast<double>(__half2float(__double2half(v)));
}

// bs[i] = b[perm[i]] * AD[perm[i]]; ADp[i] = AD[perm[i]]; bp[i] = b[perm[i]];
// inf[0] = max|bs|.
// Batched: b, bs, bp of vector k at k*vs; ADp is written by k == 0 only.
__global__ void k_rhs_in(int64_t n, const int64_t *perm, const double *AD,
                         const double *b, double *bs, double *ADp, double *bp,
                         unsigned long long *inf, int64_t vs) {
  b += blockIdx.y * vs;
  bs += blockIdx.y * vs;
  bp += blockIdx.y * vs;
  inf += 8 * blockIdx.y;
  if (blockIdx.y != 0) ADp = nullptr;
  const int64_t i   = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool    act = i < n;
  double        v   = 0.0;
  if (act) {
    const int64_t o = perm[i];
    const double  a = AD[o];
    v               = b[o] * a;
    bs[i]           = v;
    if (ADp) ADp[i] = a;
    bp[i]           = b[o];
  }
  warp_max_abs(inf, v, act);
}

// out[perm[i]] = x[i] * ADp[i] (ADp NULL: out[perm[i]] = x[i]).
__global__ void k_sol_out(int64_t n, const int64_t *perm, const double *ADp,
                          const double *x, double *out, int64_t vs) {
  x += blockIdx.y * vs;
  out += blockIdx.y * vs;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) out[perm[i]] = ADp ? x[i] * ADp[i] : x[i];
}

// ---------------------------------------------------------------------------
// Host wrappers.
static unsigned blocks_for(int64_t n, int t) {
  return static_cast<unsigned>(std::max<int64_t>(1, (n + t - 1) / t));
}

void VecOps::allocate(int64_t n_, int sms, int batch_) {
  n       = n_;
  batch   = std::max(batch_, 1);
  nblocks = std::max(1, std::min<int>(2 * sms, static_cast<int>((n + kRedThreads - 1) / kRedThreads)));
  part.resize(sizeof(double) * 2048 * batch);
  count.resize(sizeof(unsigned int) * batch);
  infbits.resize(sizeof(unsigned long long) * 8 * batch);
  device_zero(count.as<void>(), sizeof(unsigned int) * batch);
}

// Zeroes slots [first, first + cnt) of banks 0 .. nb-1.
static void clear_slots(unsigned long long *bits, int nb, int first, int cnt, cudaStream_t s) {
  MPIR_CUDA(cudaMemset2DAsync(bits + first, 8 * sizeof(unsigned long long), 0,
                              cnt * sizeof(unsigned long long), nb, s));
}

static dim3 grid_b(int64_t work, int threads, int nb) {
  return dim3(blocks_for(work, threads), static_cast<unsigned>(nb), 1);
}

void VecOps::spmv_b(int nb, const int64_t *Kp, const int32_t *Kj, const double *Kv,
                    const double *x, double *y, int64_t vs, const int32_t *act,
                    cudaStream_t s) {
  constexpr int G = 8;
  launch(k_spmv<G, 0>, grid_b(n * G, 256, nb), 256, 0, s, n, Kp, Kj, Kv, x, nullptr, y,
         nullptr, vs, act);
}

void VecOps::residual_b(int nb, const int64_t *Kp, const int32_t *Kj, const double *Kv,
                        const double *x, const double *b, double *r, bool dd, int64_t vs,
                        const int32_t *act, cudaStream_t s) {
  constexpr int G = 8;
  unsigned long long *inf = infbits.as<unsigned long long>();
  clear_slots(inf, nb, 0, 1, s);
  if (dd)
    launch(k_spmv<G, 2>, grid_b(n * G, 256, nb), 256, 0, s, n, Kp, Kj, Kv, x, b, r, inf, vs,
           act);
  else
    launch(k_spmv<G, 1>, grid_b(n * G, 256, nb), 256, 0, s, n, Kp, Kj, Kv, x, b, r, inf, vs,
           act);
}

void VecOps::backward_terms_b(int nb, const int64_t *Kp, const int32_t *Kj, const double *Korig,
                              const double *x, const double *ADp, const double *bp, int64_t vs,
                              cudaStream_t s) {
  constexpr int G = 8;
  unsigned long long *inf = infbits.as<unsigned long long>();
  clear_slots(inf, nb, 4, 4, s);
  launch(k_backward_terms<G>, grid_b(n * G, 256, nb), 256, 0, s, n, Kp, Kj, Korig, x, ADp, bp,
         inf + 4, vs, static_cast<const int32_t *>(nullptr));
}

void VecOps::mgs_pass_b(int nb, double *w, const double *v, const double *hsrc, const double *u,
                        int mode, double *out, int64_t vs, int64_t hs, const int32_t *act,
                        cudaStream_t s) {
  launch(k_mgs_pass, dim3(nblocks, nb, 1), kRedThreads, 0, s, n, w, v, hsrc, u, mode,
         part.as<double>(), count.as<unsigned int>(), out, vs, hs, act);
}

void VecOps::scale_b(int nb, const double *x, const double *fac, double *y, int64_t vs,
                     const int32_t *act, cudaStream_t s) {
  launch(k_scale, grid_b(n, 256, nb), 256, 0, s, n, x, 0.0, y, vs, fac, act);
}

void VecOps::combine_b(int nb, const double *V, int64_t ldv, const double *y, int64_t ys,
                       const int32_t *kq, double *res, int64_t vs, const int32_t *act,
                       cudaStream_t s) {
  launch(k_combine, grid_b(n, 256, nb), 256, 0, s, n, V, ldv, 0, y, res, vs, ys, kq, act);
}

void VecOps::ir_update_b(int nb, double *d, const double *fac, double *x, int64_t vs,
                         const int32_t *act, cudaStream_t s, const double *w) {
  unsigned long long *inf = infbits.as<unsigned long long>();
  clear_slots(inf, nb, 1, 2, s);
  launch(k_ir_update, grid_b(n, 256, nb), 256, 0, s, n, d, 0.0, x, w, inf + 1, vs, fac, act);
}

void VecOps::rhs_in_b(int nb, const int64_t *perm, const double *AD, const double *b, double *bs,
                      double *ADp, double *bp, int64_t vs, cudaStream_t s) {
  unsigned long long *inf = infbits.as<unsigned long long>();
  clear_slots(inf, nb, 3, 1, s);
  launch(k_rhs_in, grid_b(n, 256, nb), 256, 0, s, n, perm, AD, b, bs, ADp, bp, inf + 3, vs);
}

void VecOps::sol_out_b(int nb, const int64_t *perm, const double *ADp, const double *x,
                       double *out, int64_t vs, cudaStream_t s) {
  launch(k_sol_out, grid_b(n, 256, nb), 256, 0, s, n, perm, ADp, x, out, vs);
}

void VecOps::read_inf_b(int nb, double *h, cudaStream_t s) {
  static_assert(sizeof(double) == sizeof(unsigned long long), "bit copy");
  MPIR_CUDA(cudaMemcpyAsync(h, infbits.as<void>(), nb * 8 * sizeof(double), cudaMemcpyDeviceToHost,
                            s));
  MPIR_CUDA(cudaStreamSynchronize(s));
}

void VecOps::spmv(const int64_t *Kp, const int32_t *Kj, const double *Kv,
                  const double *x, double *y, cudaStream_t s) {
  constexpr int G = 8;
  launch(k_spmv<G, 0>, blocks_for(n * G, 256), 256, 0, s, n, Kp, Kj, Kv, x, nullptr, y, nullptr,
         int64_t{0}, nullptr);
}

void VecOps::residual(const int64_t *Kp, const int32_t *Kj, const double *Kv,
                      const double *x, const double *b, double *r, bool dd,
                      int slot, cudaStream_t s) {
  constexpr int G = 8;
  unsigned long long *inf = infbits.as<unsigned long long>() + slot;
  MPIR_CUDA(cudaMemsetAsync(inf, 0, sizeof(unsigned long long), s));
  if (dd)
    launch(k_spmv<G, 2>, blocks_for(n * G, 256), 256, 0, s, n, Kp, Kj, Kv, x, b, r, inf,
           int64_t{0}, nullptr);
  else
    launch(k_spmv<G, 1>, blocks_for(n * G, 256), 256, 0, s, n, Kp, Kj, Kv, x, b, r, inf,
           int64_t{0}, nullptr);
}

void VecOps::backward_terms(const int64_t *Kp, const int32_t *Kj, const double *Korig,
                            const double *x, const double *ADp, const double *bp,
                            cudaStream_t s) {
  constexpr int G = 8;
  unsigned long long *inf = infbits.as<unsigned long long>() + 4;
  MPIR_CUDA(cudaMemsetAsync(inf, 0, 4 * sizeof(unsigned long long), s));
  launch(k_backward_terms<G>, blocks_for(n * G, 256), 256, 0, s, n, Kp, Kj, Korig, x, ADp, bp, inf,
         int64_t{0}, nullptr);
}

void VecOps::mgs_pass(double *w, const double *v, const double *hsrc, const double *u,
                      int mode, double *out, cudaStream_t s) {
  launch(k_mgs_pass, nblocks, kRedThreads, 0, s, n, w, v, hsrc, u, mode, part.as<double>(),
         count.as<unsigned int>(), out, int64_t{0}, int64_t{0}, nullptr);
}

void VecOps::scale(const double *x, double a, double *y, cudaStream_t s) {
  launch(k_scale, blocks_for(n, 256), 256, 0, s, n, x, a, y, int64_t{0}, nullptr, nullptr);
}

void VecOps::combine(const double *V, int64_t ldv, int k, const double *y, double *res,
                     cudaStream_t s) {
  launch(k_combine, blocks_for(n, 256), 256, 0, s, n, V, ldv, k, y, res, int64_t{0}, int64_t{0},
         nullptr, nullptr);
}

void VecOps::ir_update(double *d, double scale, double *x, cudaStream_t s, const double *w) {
  unsigned long long *inf = infbits.as<unsigned long long>() + 1;
  MPIR_CUDA(cudaMemsetAsync(inf, 0, 2 * sizeof(unsigned long long), s));
  launch(k_ir_update, blocks_for(n, 256), 256, 0, s, n, d, scale, x, w, inf, int64_t{0}, nullptr,
         nullptr);
}

void VecOps::round_to(int prec, double *x, cudaStream_t s) {
  if (prec < 1 || prec > 3) return;
  launch(k_round_to, blocks_for(n, 256), 256, 0, s, n, prec, x);
}

void VecOps::rhs_in(const int64_t *perm, const double *AD, const double *b, double *bs,
                    double *ADp, double *bp, cudaStream_t s) {
  unsigned long long *inf = infbits.as<unsigned long long>() + 3;
  MPIR_CUDA(cudaMemsetAsync(inf, 0, sizeof(unsigned long long), s));
  launch(k_rhs_in, blocks_for(n, 256), 256, 0, s, n, perm, AD, b, bs, ADp, bp, inf, int64_t{0});
}

void VecOps::sol_out(const int64_t *perm, const double *ADp, const double *x, double *out,
                     cudaStream_t s) {
  launch(k_sol_out, blocks_for(n, 256), 256, 0, s, n, perm, ADp, x, out, int64_t{0});
}

void VecOps::read_inf(double *h, int first, int cnt, cudaStream_t s) {
  unsigned long long bits[8];
  MPIR_CUDA(cudaMemcpyAsync(bits, infbits.as<unsigned long long>() + first,
                            cnt * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < cnt; i++) {
    double v;
    std::memcpy(&v, &bits[i], sizeof v);
    h[i] = v;
  }
}

}  // namespace mpir
