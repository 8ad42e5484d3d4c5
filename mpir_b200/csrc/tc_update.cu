// Tensor-core GEMM updates of the blocked partial LDL^T (sm_100a, tcgen05):
// C -= (A D) A^T for the left-looking block-column updates of a front and for
// its update matrix (GemmProb), the work that dominates the factorization.
//
// Operands come from the packed copy of the front (PackedFront), where every
// stage of 16 or 32 columns of a 128-row tile is one contiguous, 16-byte
// aligned block already in the tensor cores' K-major core-matrix layout.  One
// CTA computes a 128 x 128 tile of C over its K range (one split of K) with
// warp-specialised roles around a ring of kStages shared-memory stages:
//
//   warp 0 (one lane)  producer: cp.async.bulk of the A block, the B block
//                      and the stage's pivots into a free stage; the copies
//                      complete on the stage's `full` mbarrier (tx bytes);
//   warps 4..7         converters: thread m takes packed row m of A and B,
//                      scales by the pivots and rounds in place (3xTF32: the
//                      tf32 high part in place, the low part beside it;
//                      16-bit: bfloat16 / float16 into the first half), then
//                      arrives on the stage's `conv` mbarrier;
//   warp 1 (one lane)  MMA issuer: tcgen05.mma into a 128 x 128 float32
//                      accumulator in tensor memory; tcgen05.commit frees the
//                      stage (`empty`) once its MMAs have read it;
//   warps 4..7         epilogue: tcgen05.ld of the accumulator (warp w reads
//                      lanes 32(w-4) .. = tile rows) and C -= tile with
//                      coalesced column stores, or the split partial.
//
//   kind::tf32 3xTF32: A_hi B_hi + A_hi B_lo + A_lo B_hi per 8-wide K step,
//                      float32-level accuracy (round-to-nearest splits).
//   kind::f16 bfloat16 / float16: balanced operands (A sqrt|D| sign D) and
//                      (A sqrt|D|), which keep both in range.
//   kind::f16 3xBF16:  the balanced operands split into bfloat16 high and
//                      low parts, A_hi B_hi + A_hi B_lo + A_lo B_hi per
//                      16-wide K step (about 16 significant bits: between
//                      tf32 and float32), at the bfloat16 rate.
//
// Every mbarrier wait is bounded; on expiry the kernel records a timeout in
// the factor status, stops issuing work, waits (bounded) for its own copies
// and MMAs, frees its tensor memory and returns.
#include <atomic>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "engine.hpp"

namespace mpir {

namespace tc {

constexpr int      kTileM     = 128;
constexpr int      kTileN     = 128;
constexpr int      kThreads   = 256;
#ifndef MPIR_TC_STAGES
#define MPIR_TC_STAGES 3
#endif
constexpr int      kStages    = MPIR_TC_STAGES;
constexpr uint32_t kTmemCols  = 128;
constexpr uint32_t kGroup     = 2048;  // bytes of one K-group (128 rows x 16 B)
constexpr uint32_t kLBO       = 2048;  // bytes between K-adjacent core matrices
constexpr uint32_t kSBO       = 128;   // bytes between 8-row groups
constexpr long     kSpinLimit = 20000000;

// Stage layout of a mode (bytes): A block, B block, [A low, B low], pivots.
template <int MODE>
struct Cfg {
  static constexpr bool     kHalf  = MODE != 1;
  static constexpr int      kKC    = kHalf ? 32 : 16;  // float32 columns per stage
  static constexpr int      kKG    = kKC / 4;          // packed K-groups per stage
  static constexpr uint32_t kRaw   = kKG * kGroup;     // bytes of one operand block
  static constexpr uint32_t kA     = 0;
  static constexpr uint32_t kB     = kRaw;
  static constexpr uint32_t kAlo   = 2 * kRaw;
  static constexpr uint32_t kBlo   = 3 * kRaw;
  static constexpr uint32_t kD     = kHalf ? 2 * kRaw : 4 * kRaw;
  static constexpr uint32_t kStage = kD + 1024;        // keeps 1024-byte alignment
  static constexpr uint32_t kTx    = 2 * kRaw + kKC * 4;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start, LBO, SBO (>> 4), version 1,
// no swizzle.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((kLBO >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((kSBO >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// Instruction descriptor: float32 accumulator, A/B format, both K-major,
// N = 128, M = 128.
__host__ __device__ constexpr uint32_t make_idesc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((kTileN >> 3) << 17) |
         ((kTileM >> 4) << 24);
}
constexpr uint32_t kFmtF16 = 0, kFmtBF16 = 1, kFmtTF32 = 2;

template <bool TF32>
__device__ __forceinline__ void mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accum) {
  if (TF32) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accum));
  }
}

__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool wait_bounded(uint32_t mbar, uint32_t parity) {
  for (long it = 0; it < kSpinLimit; it++)
    if (try_wait(mbar, parity)) return true;
  return false;
}

__device__ __forceinline__ void arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
               "r"(bytes) : "memory");
}

// Bulk global -> shared copy (16-byte aligned addresses, size a multiple of
// 16) completing on an mbarrier.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes,
                                          uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t pack_f16(float a, float b) {
  const __half2 v = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&v);
}

template <int MODE>
__device__ __forceinline__ uint32_t pack16(float a, float b) {
  return MODE == 2 ? pack_f16(a, b) : pack_bf16(a, b);
}

// bfloat16 high part of a and b (round to nearest) and the bfloat16 of what
// the high part leaves.
__device__ __forceinline__ void split_bf16(float a, float b, uint32_t &hi, uint32_t &lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2         f = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - f.x, b - f.y);
  hi                     = *reinterpret_cast<const uint32_t *>(&h);
  lo                     = *reinterpret_cast<const uint32_t *>(&l);
}

// tf32 high and low parts of four values (round to nearest both times).
__device__ __forceinline__ void split4(const float (&v)[4], uint4 &hi, uint4 &lo) {
  uint32_t *hp = &hi.x, *lp = &lo.x;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    const uint32_t h = to_tf32(v[e]);
    hp[e]            = h;
    lp[e]            = to_tf32(v[e] - __uint_as_float(h));
  }
}

// Round packed row m of one stage in place (see the file comment).  PRE: B
// arrived already split (k_convert_b), so only A is converted.
template <int MODE, bool PRE>
__device__ __forceinline__ void convert_row(uint8_t *stage, int m) {
  using C         = Cfg<MODE>;
  const float *dv = reinterpret_cast<const float *>(stage + C::kD);
  if (MODE == 1) {
#pragma unroll
    for (int g = 0; g < C::kKG; g++) {
      float4      *pa    = reinterpret_cast<float4 *>(stage + C::kA + g * kGroup + m * 16);
      const float4 a     = *pa;
      const float  av[4] = {a.x, a.y, a.z, a.w};
      uint4        ah, al;
      split4(av, ah, al);
      *reinterpret_cast<uint4 *>(pa)                                    = ah;
      *reinterpret_cast<uint4 *>(stage + C::kAlo + g * kGroup + m * 16) = al;
      if (!PRE) {
        float4      *pb    = reinterpret_cast<float4 *>(stage + C::kB + g * kGroup + m * 16);
        const float4 b     = *pb;
        const float4 d     = *reinterpret_cast<const float4 *>(dv + 4 * g);
        const float  bv[4] = {b.x * d.x, b.y * d.y, b.z * d.z, b.w * d.w};
        uint4        bh, bl;
        split4(bv, bh, bl);
        *reinterpret_cast<uint4 *>(pb)                                    = bh;
        *reinterpret_cast<uint4 *>(stage + C::kBlo + g * kGroup + m * 16) = bl;
      }
    }
  } else {
    // 32 columns of row m: read all (8 float32 K-groups), then write 4
    // 16-bit K-groups of 8 over the first half of the block.
    float av[32], bv[32];
#pragma unroll
    for (int g = 0; g < C::kKG; g++) {
      const float4 a = *reinterpret_cast<const float4 *>(stage + C::kA + g * kGroup + m * 16);
      const float4 b = *reinterpret_cast<const float4 *>(stage + C::kB + g * kGroup + m * 16);
      const float4 s = *reinterpret_cast<const float4 *>(dv + 4 * g);
      av[4 * g + 0] = a.x * s.x;
      av[4 * g + 1] = a.y * s.y;
      av[4 * g + 2] = a.z * s.z;
      av[4 * g + 3] = a.w * s.w;
      bv[4 * g + 0] = b.x * fabsf(s.x);
      bv[4 * g + 1] = b.y * fabsf(s.y);
      bv[4 * g + 2] = b.z * fabsf(s.z);
      bv[4 * g + 3] = b.w * fabsf(s.w);
    }
    if (MODE == 3) {
      // high parts over the first half of each block, low parts over the
      // second half (row m's 16 bytes of each K-group are this thread's)
#pragma unroll
      for (int q = 0; q < C::kKG / 2; q++) {
        uint4 ah, al, bh, bl;
        split_bf16(av[8 * q + 0], av[8 * q + 1], ah.x, al.x);
        split_bf16(av[8 * q + 2], av[8 * q + 3], ah.y, al.y);
        split_bf16(av[8 * q + 4], av[8 * q + 5], ah.z, al.z);
        split_bf16(av[8 * q + 6], av[8 * q + 7], ah.w, al.w);
        split_bf16(bv[8 * q + 0], bv[8 * q + 1], bh.x, bl.x);
        split_bf16(bv[8 * q + 2], bv[8 * q + 3], bh.y, bl.y);
        split_bf16(bv[8 * q + 4], bv[8 * q + 5], bh.z, bl.z);
        split_bf16(bv[8 * q + 6], bv[8 * q + 7], bh.w, bl.w);
        *reinterpret_cast<uint4 *>(stage + C::kA + q * kGroup + m * 16)                = ah;
        *reinterpret_cast<uint4 *>(stage + C::kA + (q + C::kKG / 2) * kGroup + m * 16) = al;
        *reinterpret_cast<uint4 *>(stage + C::kB + q * kGroup + m * 16)                = bh;
        *reinterpret_cast<uint4 *>(stage + C::kB + (q + C::kKG / 2) * kGroup + m * 16) = bl;
      }
      return;
    }
#pragma unroll
    for (int q = 0; q < C::kKG / 2; q++) {
      uint4 pa, pbk;
      pa.x  = pack16<MODE>(av[8 * q + 0], av[8 * q + 1]);
      pa.y  = pack16<MODE>(av[8 * q + 2], av[8 * q + 3]);
      pa.z  = pack16<MODE>(av[8 * q + 4], av[8 * q + 5]);
      pa.w  = pack16<MODE>(av[8 * q + 6], av[8 * q + 7]);
      pbk.x = pack16<MODE>(bv[8 * q + 0], bv[8 * q + 1]);
      pbk.y = pack16<MODE>(bv[8 * q + 2], bv[8 * q + 3]);
      pbk.z = pack16<MODE>(bv[8 * q + 4], bv[8 * q + 5]);
      pbk.w = pack16<MODE>(bv[8 * q + 6], bv[8 * q + 7]);
      *reinterpret_cast<uint4 *>(stage + C::kA + q * kGroup + m * 16) = pa;
      *reinterpret_cast<uint4 *>(stage + C::kB + q * kGroup + m * 16) = pbk;
    }
  }
}

}  // namespace tc

// One unit of work: a 128 x 128 tile of one problem over one split of K.
struct Unit {
  const GemmProb *pb;
  int             tile, sp, mt, j, k_lo, nch;
};

// Units of a launch in order: problem by binary search on the problems'
// first units (kept in shared memory when they fit), then the tile of the
// (lower) tile pattern and the split.
template <int KC>
__device__ __forceinline__ Unit locate_unit(const GemmProb *probs, int nprob, const int *t0s,
                                            int u) {
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    const int t0  = t0s ? t0s[mid] : probs[mid].tile0;
    if (t0 <= u) lo = mid; else hi = mid - 1;
  }
  Unit U;
  U.pb            = probs + lo;
  const int local = u - U.pb->tile0;
  const int splits = U.pb->splits, ntm = U.pb->ntm, K = U.pb->K;
  U.sp   = local % splits;
  int tl = local / splits;
  U.tile = tl;
  int j  = 0;
  if (U.pb->lower) {
    while (tl >= ntm - j) {
      tl -= ntm - j;
      j++;
    }
  } else {
    j  = tl / ntm;
    tl = tl % ntm;
  }
  U.mt          = U.pb->lower ? j + tl : tl;
  U.j           = j;
  const int ks  = ((K + splits - 1) / splits + 31) / 32 * 32;
  U.k_lo        = U.sp * ks;
  const int khi = min(K, U.k_lo + ks);
  U.nch         = khi > U.k_lo ? (khi - U.k_lo + KC - 1) / KC : 0;
  return U;
}

constexpr int kMaxProbSmem = 2048;  // problems whose first units go to shared memory

// MODE 0: bfloat16 single pass; MODE 1: 3xTF32; MODE 2: float16 single pass;
// MODE 3: 3xBF16.
// Persistent: CTA b takes units b, b + gridDim.x, ...; the ring stages run on
// across units (the producer loads the next unit's first stages while the
// epilogue drains the accumulator of the current one); the accumulator is
// handed between the MMA issuer and the epilogue by the acc_full / acc_free
// mbarriers.
template <int MODE>
__global__ void __launch_bounds__(tc::kThreads, tc::kStages <= 3 ? 2 : 1)
    k_gemm_tc(const GemmProb *probs, int nprob, int units, const float *pack,
              const float *packd, const float *packs, const float *bconv, float *panel,
              float *uarena, float *ws, FactorStatus *st) {
  using namespace tc;
  using C = Cfg<MODE>;
  // 3xTF32 with B converted ahead (k_convert_b): the producer copies B's
  // high and low parts and the converters round A only.
  const bool pre = MODE == 1 && bconv != nullptr;
  extern __shared__ __align__(1024) uint8_t smem[];
  // full[kStages], conv[kStages], empty[kStages], acc_full, acc_free, drain
  __shared__ __align__(8) uint64_t bars[3 * kStages + 3];
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int s_fail;

  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  int      *t0s = nprob <= kMaxProbSmem
                      ? reinterpret_cast<int *>(smem + kStages * C::kStage)
                      : nullptr;
  const uint32_t full0 = smem_u32(&bars[0]), conv0 = smem_u32(&bars[kStages]),
                 empty0 = smem_u32(&bars[2 * kStages]),
                 acc_full = smem_u32(&bars[3 * kStages]),
                 acc_free = smem_u32(&bars[3 * kStages + 1]),
                 drain = smem_u32(&bars[3 * kStages + 2]);
  // ---- tensor memory, barriers, problem table
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    s_fail = 0;
    for (int s = 0; s < kStages; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(full0 + 8 * s) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(conv0 + 8 * s) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(empty0 + 8 * s) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(acc_full) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(acc_free) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(drain) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (t0s)
    for (int q = tid; q < nprob; q += kThreads) t0s[q] = probs[q].tile0;
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    // ---------------- producer
    if (lane == 0) {
      long g = 0;
      for (int u = blockIdx.x; u < units && !s_fail; u += gridDim.x) {
        const Unit   U  = locate_unit<C::kKC>(probs, nprob, t0s, u);
        const float *Ag = pack + U.pb->pa + static_cast<int64_t>(U.mt) * U.pb->prow +
                          static_cast<int64_t>(U.k_lo / 4) * PackedFront::kGroupFloats;
        const float *Bg = pack + U.pb->pb + static_cast<int64_t>(U.j) * U.pb->prow +
                          static_cast<int64_t>(U.k_lo / 4) * PackedFront::kGroupFloats;
        const float *Dg = (C::kHalf ? packs : packd) + U.pb->pd + U.k_lo;
        const int64_t bo = static_cast<int64_t>(U.j) * U.pb->bprow +
                           static_cast<int64_t>(U.k_lo / 4) * PackedFront::kGroupFloats;
        const float *Bh = pre ? bconv + U.pb->bc + bo : nullptr;
        const float *Bl = pre ? bconv + U.pb->bc_lo + bo : nullptr;
        for (int c = 0; c < U.nch; c++, g++) {
          const int s = static_cast<int>(g % kStages);
          const int round = static_cast<int>(g / kStages);
          if (round > 0 && !wait_bounded(empty0 + 8 * s, (round - 1) & 1)) {
            s_fail = 1;
            break;
          }
          const uint32_t base = smem_u32(smem + s * C::kStage);
          const int64_t  ko   = static_cast<int64_t>(c) * C::kKG * PackedFront::kGroupFloats;
          if (pre) {
            arrive_expect_tx(full0 + 8 * s, 3 * C::kRaw);
            bulk_load(base + C::kA, Ag + ko, C::kRaw, full0 + 8 * s);
            bulk_load(base + C::kB, Bh + ko, C::kRaw, full0 + 8 * s);
            bulk_load(base + C::kBlo, Bl + ko, C::kRaw, full0 + 8 * s);
          } else {
            arrive_expect_tx(full0 + 8 * s, C::kTx);
            bulk_load(base + C::kA, Ag + ko, C::kRaw, full0 + 8 * s);
            bulk_load(base + C::kB, Bg + ko, C::kRaw, full0 + 8 * s);
            bulk_load(base + C::kD, Dg + c * C::kKC, C::kKC * 4, full0 + 8 * s);
          }
        }
      }
      // No copy may still target shared memory at exit: the last stage issued
      // into each slot has landed (no later round was issued into it).
      for (long c = g > kStages ? g - kStages : 0; c < g; c++)
        wait_bounded(full0 + 8 * static_cast<int>(c % kStages),
                     static_cast<uint32_t>(c / kStages) & 1);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc =
          make_idesc(MODE == 1 ? kFmtTF32 : MODE == 2 ? kFmtF16 : kFmtBF16);
      long           g     = 0;
      int            jn    = 0;
      for (int u = blockIdx.x; u < units && !s_fail; u += gridDim.x, jn++) {
        const Unit U = locate_unit<C::kKC>(probs, nprob, t0s, u);
        // the epilogue has read the previous unit's accumulator
        if (jn > 0 && !wait_bounded(acc_free, (jn - 1) & 1)) {
          s_fail = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        bool ok = true;
        for (int c = 0; c < U.nch; c++, g++) {
          const int s = static_cast<int>(g % kStages);
          const int round = static_cast<int>(g / kStages);
          if (!wait_bounded(conv0 + 8 * s, round & 1)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t base = smem_u32(smem + s * C::kStage);
          // Each MMA consumes two K-groups: 8 tf32 or 16 16-bit columns.
          constexpr int kSteps = MODE == 1 ? C::kKG / 2 : C::kKG / 4;
#pragma unroll
          for (int q = 0; q < kSteps; q++) {
            const uint32_t off = q * 2 * kGroup;
            const uint32_t acc = (c > 0 || q > 0) ? 1u : 0u;
            if (MODE == 1) {
              const uint64_t ahd = make_desc(base + C::kA + off);
              const uint64_t bhd = make_desc(base + C::kB + off);
              const uint64_t ald = make_desc(base + C::kAlo + off);
              const uint64_t bld = make_desc(base + C::kBlo + off);
              mma<true>(tmem, ahd, bhd, idesc, acc);
              mma<true>(tmem, ahd, bld, idesc, 1u);
              mma<true>(tmem, ald, bhd, idesc, 1u);
            } else if (MODE == 3) {
              constexpr uint32_t kLo = C::kKG / 2 * kGroup;  // low parts' offset
              const uint64_t ahd = make_desc(base + C::kA + off);
              const uint64_t bhd = make_desc(base + C::kB + off);
              const uint64_t ald = make_desc(base + C::kA + kLo + off);
              const uint64_t bld = make_desc(base + C::kB + kLo + off);
              mma<false>(tmem, ahd, bhd, idesc, acc);
              mma<false>(tmem, ahd, bld, idesc, 1u);
              mma<false>(tmem, ald, bhd, idesc, 1u);
            } else {
              mma<false>(tmem, make_desc(base + C::kA + off), make_desc(base + C::kB + off),
                         idesc, acc);
            }
          }
          commit(empty0 + 8 * s);
        }
        if (!ok) {
          s_fail = 1;
          break;
        }
        commit(acc_full);  // tracks every MMA issued so far
      }
      // Every MMA of this CTA has completed before the memory is released.
      commit(drain);
      wait_bounded(drain, 0);
    }
    __syncwarp();
  } else if (warp >= 4) {
    // ---------------- converters, then the epilogue of each unit
    const int m  = tid - 128;
    const int ew = warp - 4;  // tensor-memory lanes 32 ew .. 32 ew + 31
    long      g  = 0;
    int       jn = 0;
    for (int u = blockIdx.x; u < units && !s_fail; u += gridDim.x, jn++) {
      const Unit U  = locate_unit<C::kKC>(probs, nprob, t0s, u);
      bool       ok = true;
      for (int c = 0; c < U.nch; c++, g++) {
        const int s = static_cast<int>(g % kStages);
        const int round = static_cast<int>(g / kStages);
        if (!wait_bounded(full0 + 8 * s, round & 1)) {
          ok = false;
          break;
        }
        if (pre)
          convert_row<MODE, true>(smem + s * C::kStage, m);
        else
          convert_row<MODE, false>(smem + s * C::kStage, m);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        arrive(conv0 + 8 * s);
      }
      ok = ok && wait_bounded(acc_full, jn & 1);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        s_fail = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const GemmProb &pb   = *U.pb;
      const int       lr   = ew * 32 + lane;
      const int       mrow = U.mt * kTileM + lr;
      const int       row  = mrow < pb.M ? gemm_out_row(pb, mrow) : -1;
      const int       n0   = U.j * kTileN;
      float          *Cout = (pb.c_in_u ? uarena : panel) + pb.c_ofs;
      float          *W    = pb.splits > 1
                                 ? ws + pb.ws_ofs +
                                    (static_cast<int64_t>(U.tile) * pb.splits + U.sp) *
                                        (kTileM * kTileN)
                                 : nullptr;
      const int       N = pb.N, ldc = pb.ldc, lower = pb.lower, c_in_u = pb.c_in_u;
#pragma unroll
      for (int cb = 0; cb < kTileN / 32; cb++) {
        uint32_t       r[32];
        const uint32_t taddr = tmem + (static_cast<uint32_t>(ew * 32) << 16) + cb * 32;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
              "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
              "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (U.nch == 0)  // an empty K range leaves the accumulator unwritten
#pragma unroll
          for (int q = 0; q < 32; q++) r[q] = 0u;
        if (W) {
#pragma unroll
          for (int q = 0; q < 32; q++) W[lr + (cb * 32 + q) * kTileM] = __uint_as_float(r[q]);
        } else if (row >= 0) {
          // Loads of 16 columns first, then their stores: one memory latency
          // per 16 columns (as a read-modify-write loop the loads could not
          // move above the preceding stores).
#pragma unroll
          for (int hh = 0; hh < 2; hh++) {
            float cv[16];
#pragma unroll
            for (int q = 0; q < 16; q++) {
              const int col = n0 + cb * 32 + 16 * hh + q;
              // an update matrix is defined by this product (stored, not updated)
              cv[q] = (!c_in_u && col < N && (!lower || row >= col))
                          ? Cout[row + (int64_t)col * ldc]
                          : 0.0f;
            }
#pragma unroll
            for (int q = 0; q < 16; q++) {
              const int col = n0 + cb * 32 + 16 * hh + q;
              if (col < N && (!lower || row >= col))
                Cout[row + (int64_t)col * ldc] = cv[q] - __uint_as_float(r[16 * hh + q]);
            }
          }
        }
      }
      // The accumulator may be overwritten by the next unit's MMAs.
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      arrive(acc_free);
    }
  }
  if (tid == 0 && s_fail) atomicExch(&st->timeout, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols) : "memory");
}

int tc_ctas_per_sm() { return tc::kStages <= 3 ? 2 : 1; }

int tc_gemm_smem_bytes(int mode) {
  const uint32_t stage = mode == 1 ? tc::Cfg<1>::kStage : tc::Cfg<0>::kStage;
  // stages, then the problems' first units
  return static_cast<int>(tc::kStages * stage + kMaxProbSmem * sizeof(int));
}

// B of each problem of a launch, scaled by the pivots and split into tf32
// high and low parts once (the 3xTF32 product would otherwise redo this in
// every CTA that shares B): CTA t converts kConvGroups K-groups of one row
// tile, thread (g, m) one packed row of one K-group, with the same
// arithmetic as the in-kernel conversion.
__global__ void __launch_bounds__(256)
    k_convert_b(const GemmProb *probs, int nprob, const float *pack, const float *packd,
                float *bconv) {
  using namespace tc;
  const int t  = blockIdx.x;
  int       lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (probs[mid].cv0 <= t) lo = mid; else hi = mid - 1;
  }
  const GemmProb &pb     = probs[lo];
  const int       chunks = (pb.bgroups + kConvGroups - 1) / kConvGroups;
  const int       local  = t - pb.cv0;
  const int       tile   = local / chunks;
  const int       g0     = (local % chunks) * kConvGroups;
  const int       g1     = min(g0 + kConvGroups, pb.bgroups);
  const int       m      = threadIdx.x % 128;
  // All loads of the thread's K-groups first, then the stores (the
  // conversion buffer and the packed fronts are separate arrays, but the
  // compiler cannot tell).
  constexpr int kPer = kConvGroups / 2;
  float4        b[kPer], d[kPer];
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int g = g0 + threadIdx.x / 128 + 2 * u;
    if (g < g1) {
      b[u] = *reinterpret_cast<const float4 *>(
          pack + pb.pb + static_cast<int64_t>(tile) * pb.prow +
          static_cast<int64_t>(g) * PackedFront::kGroupFloats + m * 4);
      d[u] = *reinterpret_cast<const float4 *>(packd + pb.pd + 4 * g);
    }
  }
#pragma unroll
  for (int u = 0; u < kPer; u++) {
    const int g = g0 + threadIdx.x / 128 + 2 * u;
    if (g >= g1) continue;
    const float bv[4] = {b[u].x * d[u].x, b[u].y * d[u].y, b[u].z * d[u].z, b[u].w * d[u].w};
    uint4       bh, bl;
    split4(bv, bh, bl);
    const int64_t o = static_cast<int64_t>(tile) * pb.bprow +
                      static_cast<int64_t>(g) * PackedFront::kGroupFloats + m * 4;
    *reinterpret_cast<uint4 *>(bconv + pb.bc + o)    = bh;
    *reinterpret_cast<uint4 *>(bconv + pb.bc_lo + o) = bl;
  }
}

void launch_convert_b(const GemmProb *probs, int nprob, int convs, const float *pack,
                      const float *packd, float *bconv, cudaStream_t s) {
  if (convs > 0) launch(k_convert_b, convs, 256, 0, s, probs, nprob, pack, packd, bconv);
}

// ---------------------------------------------------------------------------
// Panel solve of a block step on the tensor cores (3xTF32):
//   W = F X^T diag(Dinv)
// for one 128-row tile of the rows below the step's diagonal block: F the
// tile's nbk columns of the panel, X the inverse of the block's unit-lower
// factor (linv, column-major, leading dimension kNB), Dinv the block's
// pivots' reciprocals.  Outputs as k_step_gemm<true>: W over F in the panel
// and, as whole K-groups, into the packed front.
//
// Shared memory (K-major core-matrix layout, K-group g at g * 2048 bytes,
// row m at m * 16): B = X diag(Dinv) in tf32 high and low parts for all 128
// columns of K (2 x 64 KB), A in halves of 64 columns (high and low parts,
// 2 x 32 KB).  All 256 threads load A (both halves) and X into registers
// first, then convert B and A's first half; one lane issues its 8 x 3 MMAs
// (M = N = 128, K = 8) and commits; the threads write A's second half once
// the commit shows the first half's MMAs done.  Epilogue: warps w and w + 4 drain
// tensor-memory lanes 32 (w % 4) .. (rows), columns 0-63 and 64-127.
namespace tc {
constexpr uint32_t kTrsmB     = 32 * kGroup;           // one part of B (bytes)
constexpr uint32_t kTrsmA     = 16 * kGroup;           // one part of an A half
constexpr uint32_t kTrsmSmem  = 2 * kTrsmB + 2 * kTrsmA;  // 192 KB
}  // namespace tc

__global__ void __launch_bounds__(256, 1)
    k_trsm_tc(const StepDesc *descs, int ndesc, float *panel, const float *linv,
              const float *Dinv, float *pack, FactorStatus *st) {
  using namespace tc;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int t   = blockIdx.x;
  int       lo = 0, hi = ndesc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (descs[mid].trsm_tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const StepDesc d  = descs[lo];
  const int      m0 = (t - d.trsm_tile0) * kTileM;
  const int64_t  h  = d.h;
  const int      kb = d.kb, nbk = d.nbk, w = d.w;
  const int      M  = static_cast<int>(h) - kb - nbk;
  float         *C  = panel + d.panel + (kb + nbk) + static_cast<int64_t>(kb) * h;
  const float   *X  = linv + d.linv;
  const uint32_t bar   = smem_u32(&done_bar);
  const uint32_t sbase = smem_u32(smem);

  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }

  // Thread (row m, K-group pair) of a half: m = tid % 128, K-groups
  // tid / 128 + 2 i of the half, i < 8.
  const int  m    = tid & 127;
  const int  gsel = tid >> 7;
  const bool rok  = m0 + m < M;
  auto load_a = [&](int half, float (&v)[32]) {
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int k = 64 * half + 4 * (gsel + 2 * i) + j;
        v[4 * i + j] = (rok && k < nbk) ? C[m0 + m + static_cast<int64_t>(k) * h] : 0.0f;
      }
  };
  auto store_a = [&](const float (&v)[32]) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const float av[4] = {v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]};
      uint4       ah, al;
      split4(av, ah, al);
      const uint32_t o = (gsel + 2 * i) * kGroup + m * 16;
      *reinterpret_cast<uint4 *>(smem + 2 * kTrsmB + o)          = ah;
      *reinterpret_cast<uint4 *>(smem + 2 * kTrsmB + kTrsmA + o) = al;
    }
  };
  // Every global load of the CTA is issued before the first is used (one
  // memory latency instead of one per batch): A's two halves, and B = X
  // diag(Dinv) by thread (row n = m, K-groups gsel + 2 i, i < 16).
  const int halves = nbk > 64 ? 2 : 1;
  float     a[32], a1[32], xv[64];
  load_a(0, a);
  const float dv = m < nbk ? Dinv[static_cast<int64_t>(d.col0) + kb + m] : 0.0f;
#pragma unroll
  for (int i = 0; i < 16; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) xv[4 * i + j] = X[m + (4 * (gsel + 2 * i) + j) * kNB];
  if (halves == 2) load_a(1, a1);
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const float bv[4] = {xv[4 * i] * dv, xv[4 * i + 1] * dv, xv[4 * i + 2] * dv,
                         xv[4 * i + 3] * dv};
    uint4       bh, bl;
    split4(bv, bh, bl);
    const uint32_t o = (gsel + 2 * i) * kGroup + m * 16;
    *reinterpret_cast<uint4 *>(smem + o)          = bh;
    *reinterpret_cast<uint4 *>(smem + kTrsmB + o) = bl;
  }
  store_a(a);
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem   = tmem_slot;
  const uint32_t idesc  = make_idesc(kFmtTF32);
  auto issue = [&](int half) {
    if (tid != 32) return;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const uint32_t ao  = 2 * kTrsmB + q * 2 * kGroup;
      const uint32_t bo  = (16 * half + 2 * q) * kGroup;
      const uint64_t ahd = make_desc(sbase + ao), ald = make_desc(sbase + ao + kTrsmA);
      const uint64_t bhd = make_desc(sbase + bo), bld = make_desc(sbase + bo + kTrsmB);
      mma<true>(tmem, ahd, bhd, idesc, (half > 0 || q > 0) ? 1u : 0u);
      mma<true>(tmem, ahd, bld, idesc, 1u);
      mma<true>(tmem, ald, bhd, idesc, 1u);
    }
    commit(bar);
  };
  issue(0);
  bool ok = true;
  if (halves == 2) {
    ok = wait_bounded(bar, 0);  // the first half's MMAs have read A
    if (ok) {
      store_a(a1);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    ok = __syncthreads_and(ok);
    if (ok) issue(1);
  }
  ok = ok && wait_bounded(bar, (halves - 1) & 1);
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int lr = (warp & 3) * 32 + lane;  // tile row of this thread's lane
    const int r  = m0 + lr;
    float    *pk = pack != nullptr && d.pk >= 0 ? pack + d.pk : nullptr;
    int64_t   prow = 0;
    if (pk) {
      const int rf = kb + nbk + r;  // row of the front
      const int p  = rf < w ? rf : rf - w + d.pk_wt;
      prow = static_cast<int64_t>(p >> 7) * d.pk_g * PackedFront::kGroupFloats + (p & 127) * 4;
    }
#pragma unroll
    for (int cc = 0; cc < 2; cc++) {
      const int cb = (warp >> 2) * 2 + cc;  // 32-column block
      if (cb * 32 >= nbk) break;
      uint32_t       v[32];
      const uint32_t taddr = tmem + (static_cast<uint32_t>((warp & 3) * 32) << 16) + cb * 32;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
            "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
            "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
            "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (r < M) {
#pragma unroll
        for (int q = 0; q < 32; q++) {
          const int c = cb * 32 + q;
          if (c < nbk) C[r + static_cast<int64_t>(c) * h] = __uint_as_float(v[q]);
        }
        if (pk) {
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const int c0 = cb * 32 + 4 * q;
            if (c0 >= nbk) break;
            float4 o;
            o.x = __uint_as_float(v[4 * q + 0]);
            o.y = __uint_as_float(v[4 * q + 1]);
            o.z = __uint_as_float(v[4 * q + 2]);
            o.w = __uint_as_float(v[4 * q + 3]);
            *reinterpret_cast<float4 *>(pk + prow +
                                        static_cast<int64_t>((kb + c0) >> 2) *
                                            PackedFront::kGroupFloats) = o;
          }
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(&st->timeout, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols) : "memory");
}

void launch_trsm_tc(const StepDesc *descs, int ndesc, int tiles, float *panel, const float *linv,
                    const float *Dinv, float *pack, FactorStatus *st, cudaStream_t s) {
  if (tiles <= 0) return;
  static std::atomic<bool> attr{false};
  if (!attr) {
    MPIR_CUDA(cudaFuncSetAttribute(k_trsm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(tc::kTrsmSmem)));
    attr = true;
  }
  launch(k_trsm_tc, tiles, 256, tc::kTrsmSmem, s, descs, ndesc, panel, linv, Dinv, pack, st);
}

template <int MODE>
static void launch_mode(const GemmProb *probs, int nprob, int units, const float *pack,
                        const float *packd, const float *packs, const float *bconv,
                        float *panel, float *uarena, float *ws, FactorStatus *st,
                        cudaStream_t s) {
  static std::atomic<bool> attr{false};
  const int   smem = tc_gemm_smem_bytes(MODE);
  if (!attr) {
    MPIR_CUDA(cudaFuncSetAttribute(k_gemm_tc<MODE>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  const int grid = std::min(units, kSMs * tc_ctas_per_sm());
  launch(k_gemm_tc<MODE>, grid, tc::kThreads, smem, s, probs, nprob, units, pack, packd, packs,
         MODE == 1 ? bconv : nullptr, panel, uarena, ws, st);
}

void launch_gemm_tc(int mode, const GemmProb *probs, int nprob, int units, const float *pack,
                    const float *packd, const float *packs, const float *bconv, float *panel,
                    float *uarena, float *ws, FactorStatus *st, cudaStream_t s) {
  if (units <= 0) return;
  if (mode == 0)
    launch_mode<0>(probs, nprob, units, pack, packd, packs, bconv, panel, uarena, ws, st, s);
  else if (mode == 1)
    launch_mode<1>(probs, nprob, units, pack, packd, packs, bconv, panel, uarena, ws, st, s);
  else if (mode == 3)
    launch_mode<3>(probs, nprob, units, pack, packd, packs, bconv, panel, uarena, ws, st, s);
  else
    launch_mode<2>(probs, nprob, units, pack, packd, packs, bconv, panel, uarena, ws, st, s);
}

}  // namespace mpir
