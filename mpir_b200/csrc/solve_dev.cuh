// Device helpers shared by the single- and multi-right-hand-side triangular
// solves (solve.cu, solve_multi.cu): asynchronous copies into shared memory
// and the ready-value hand-over of block results between CTAs.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace mpir {

// Factor values are read as float32, or from the 16-bit copy of the panels
// that the bfloat16 / float16 tiers keep for the solves; arithmetic is in
// float64 either way.
__device__ __forceinline__ float to_f(float v) { return v; }
__device__ __forceinline__ float to_f(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float to_f(__half v) { return __half2float(v); }

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(double *dst, const double *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                   static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
               "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Block results go from the CTA that computes them to the CTAs that wait on
// them through the ready buffer: each entry holds the pending marker (a
// signalling NaN, which no arithmetic produces) until its value is stored,
// and a waiting lane polls its own entry at GPU scope, so the value is its
// own ready signal (no flag, no fence, no second load).  The producer stores
// kReadyCopies copies; the warps of the ~150 CTAs that wait for the same
// block poll different copies.  A wait gives up after a bounded number of
// polls (about a second by default), sets the sticky error word and returns
// 0; it looks at that word every 64 polls, so one failure ends the launch
// quickly.
//
// The control words beside the error word (SolveCtl) let a test make a wait
// run out on purpose: a smaller poll limit, and one work item whose block
// result is never published.  Both are read once per CTA with its ticket.
constexpr unsigned long long kPending = 0x7ff0deadbeef0001ull;
constexpr int kReadyCopies = 16;
constexpr long kDefaultPolls = 1L << 22;
struct SolveCtl {
  int32_t err;        // sticky: 1 once a bounded wait gave up
  int32_t poll_log2;  // 0: kDefaultPolls; else 2^poll_log2 polls per wait
  int32_t withhold;   // 0: none; else item + 1 whose result is not published
  int32_t pad;
};
__device__ __forceinline__ long poll_limit(int32_t poll_log2) {
  return poll_log2 > 0 ? (1L << poll_log2) : kDefaultPolls;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const double *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_f64(double *p, double v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(__double_as_longlong(v))
               : "memory");
}
__device__ __forceinline__ double wait_value(const double *p, int32_t *err,
                                             long lim = kDefaultPolls) {
  for (long it = 0; it < lim; it++) {
    const unsigned long long v = ld_relaxed_u64(p);
    if (v != kPending) return __longlong_as_double(static_cast<long long>(v));
    if ((it & 63) == 63) {
      if (*reinterpret_cast<volatile int32_t *>(err) != 0) return 0.0;
      __nanosleep(32);
    }
  }
  atomicExch(err, 1);
  return 0.0;
}

}  // namespace mpir
