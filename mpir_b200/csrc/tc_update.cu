// Tensor-core GEMM updates of the blocked partial LDL^T (sm_100a, tcgen05):
// C -= (A D) A^T for the left-looking block-column updates of a front and for
// its update matrix (GemmProb), the work that dominates the factorization.
//
// One CTA of 128 threads computes a 128 x 128 tile of C over its K range
// (one split of K).  Per K-chunk every thread loads one row of A and one of
// B (= rows of A) from the float32 panel, scales them by the pivots,
// converts it (bfloat16, or tf32 hi + lo parts for the 3xTF32 product) and
// stores it into shared memory in the K-major canonical layout without
// swizzle (8-row x 16-byte core matrices, rows 16 bytes apart, K-chunks
// 2048 bytes apart).  One thread issues tcgen05.mma into a 128 x 128 float32
// accumulator in tensor memory and commits to an mbarrier; shared buffers
// alternate so loads of chunk c+1 overlap the MMAs of chunk c.  The
// epilogue reads the accumulator with tcgen05.ld (warp w owns lanes
// 32w..32w+31 = tile rows) and subtracts it from C with coalesced column
// stores.
//
//   kind::f16  with bfloat16 A/B: one MMA per 16-wide K step.
//   kind::tf32 3xTF32: A_hi B_hi + A_hi B_lo + A_lo B_hi per 8-wide K step,
//                      float32-level accuracy.
//
// Every mbarrier wait is bounded; on expiry the kernel records a timeout in
// the factor status, waits (bounded) for its own MMAs, frees its tensor
// memory and returns.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "engine.hpp"

namespace mpir {

namespace tc {

constexpr int      kTileM    = 128;
constexpr int      kTileN    = 128;
constexpr int      kThreads  = 128;
constexpr uint32_t kTmemCols = 128;
constexpr uint32_t kLBO      = 2048;  // bytes between K-direction core matrices
constexpr uint32_t kSBO      = 128;   // bytes between 8-row groups
constexpr long     kSpinLimit = 20000000;
// Raw float32 K-chunks in flight per CTA: 4 for 3xTF32 (16-wide chunks),
// 3 for 16-bit operands (32-wide chunks).
__host__ __device__ constexpr int stages_for(bool half) { return half ? 3 : 4; }

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

__device__ __forceinline__ void mma(uint32_t fmt_is_tf32, uint32_t tmem, uint64_t a,
                                    uint64_t b, uint32_t idesc, uint32_t accum) {
  if (fmt_is_tf32) {
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

// 4-byte asynchronous global->shared copy; src_bytes = 0 fills zeros and
// reads nothing (the source address is then only a placeholder).
__device__ __forceinline__ void cp_async4(uint32_t dst, const void *src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
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

}  // namespace tc

// MODE 0: bfloat16 single pass; MODE 1: 3xTF32; MODE 2: float16 single pass.
template <int MODE>
__global__ void __launch_bounds__(tc::kThreads)
    k_gemm_tc(const GemmProb *probs, int nprob, float *panel, float *uarena, const float *D,
              float *ws, FactorStatus *st) {
  using namespace tc;
  constexpr bool HALF   = MODE != 1;             // 16-bit operands
  constexpr int  KC     = HALF ? 32 : 16;        // K elements per chunk
  constexpr int  CHUNKS = KC * (HALF ? 2 : 4) / 16;  // 16-byte chunks per row
  constexpr int  PARTS  = HALF ? 1 : 2;              // hi (and lo) copies
  constexpr uint32_t kOperandBytes = kTileM * CHUNKS * 16;  // one operand part
  constexpr int      kStages       = stages_for(HALF);
  extern __shared__ __align__(1024) uint8_t smem[];
  // Buffer layout: [buf][A parts][B parts], each kOperandBytes.
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_slot;

  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  // ---- locate problem, tile and K split
  const int t  = blockIdx.x;
  int       lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (probs[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const GemmProb pb    = probs[lo];
  const int      local = t - pb.tile0;
  const int      sp    = local % pb.splits;
  int            tl    = local / pb.splits;
  const int      tile  = tl;
  int            j     = 0;
  if (pb.lower) {
    while (tl >= pb.ntm - j) {
      tl -= pb.ntm - j;
      j++;
    }
  } else {
    j  = tl / pb.ntm;
    tl = tl % pb.ntm;
  }
  const int m0 = (pb.lower ? j + tl : tl) * kTileM;
  const int n0 = j * kTileN;
  const int M = pb.M, N = pb.N, K = pb.K;
  const int ks = ((K + pb.splits - 1) / pb.splits + 31) / 32 * 32;
  const int k_lo = sp * ks, k_hi = min(K, k_lo + ks);
  const float  *A   = panel + pb.a_ofs;
  const int64_t lda = pb.lda;
  const float  *Dk  = D + pb.d_ofs;

  // ---- tensor memory and barriers
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(&tmem_slot)), "r"(kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem  = tmem_slot;
  const uint32_t idesc = make_idesc(MODE == 0 ? kFmtBF16 : MODE == 1 ? kFmtTF32 : kFmtF16);
  const int      nch   = k_hi > k_lo ? (k_hi - k_lo + KC - 1) / KC : 0;
  bool           ok    = true;
  // Raw float32 stages (A then B, column-major 128 x KC each) follow the two
  // operand buffers in shared memory.
  float *raw = reinterpret_cast<float *>(smem + 2 * (2 * PARTS * kOperandBytes));
  auto   issue_stage = [&](int c) {
    if (c < nch) {
      float    *sA = raw + (c % kStages) * (2 * kTileM * KC);
      float    *sB = sA + kTileM * KC;
      const int k0 = k_lo + c * KC;
      const int ra = m0 + tid, rb = n0 + tid;
#pragma unroll
      for (int k = 0; k < KC; k++) {
        const bool kin = k0 + k < k_hi;
        const bool okA = kin && ra < M, okB = kin && rb < N;
        cp_async4(smem_u32(sA + k * kTileM + tid),
                  okA ? A + ra + (int64_t)(k0 + k) * lda : A, okA ? 4u : 0u);
        cp_async4(smem_u32(sB + k * kTileM + tid),
                  okB ? A + rb + (int64_t)(k0 + k) * lda : A, okB ? 4u : 0u);
      }
    }
    cp_async_commit();  // one group per chunk, empty past the end
  };
#pragma unroll
  for (int c = 0; c < kStages - 1; c++) issue_stage(c);

  for (int c = 0; c < nch && ok; c++) {
    const int buf = c & 1;
    issue_stage(c + kStages - 1);
    cp_async_wait<kStages - 1>();  // this thread's copies of chunk c landed
    if (c >= 2) ok = wait_bounded(smem_u32(&mbar[buf]), ((c - 2) >> 1) & 1);
    ok = __syncthreads_and(ok);      // and everyone's
    if (!ok) break;
    uint8_t     *base = smem + buf * (2 * PARTS * kOperandBytes);
    const float *sA   = raw + (c % kStages) * (2 * kTileM * KC);
    const float *sB   = sA + kTileM * KC;
    const int    k0   = k_lo + c * KC;
    float        av[KC], bv[KC];
#pragma unroll
    for (int k = 0; k < KC; k++) {
      const float dk = k0 + k < k_hi ? Dk[k0 + k] : 0.0f;
      // (A D) A^T for 3xTF32; for 16-bit operands the balanced
      // (A sqrt|D| sign D)(A sqrt|D|)^T, which keeps both within the 16-bit
      // range when pivots are tiny and multipliers large.
      float sa = dk, sbv = 1.0f;
      if (HALF) {
        const float r = sqrtf(fabsf(dk));
        sa            = dk < 0.0f ? -r : r;
        sbv           = r;
      }
      av[k] = sA[k * kTileM + tid] * sa;
      bv[k] = sB[k * kTileM + tid] * sbv;
    }
    if (HALF) {
#pragma unroll
      for (int q = 0; q < CHUNKS; q++) {
        uint4 pa, pbk;
        pa.x  = pack16<MODE>(av[8 * q + 0], av[8 * q + 1]);
        pa.y  = pack16<MODE>(av[8 * q + 2], av[8 * q + 3]);
        pa.z  = pack16<MODE>(av[8 * q + 4], av[8 * q + 5]);
        pa.w  = pack16<MODE>(av[8 * q + 6], av[8 * q + 7]);
        pbk.x = pack16<MODE>(bv[8 * q + 0], bv[8 * q + 1]);
        pbk.y = pack16<MODE>(bv[8 * q + 2], bv[8 * q + 3]);
        pbk.z = pack16<MODE>(bv[8 * q + 4], bv[8 * q + 5]);
        pbk.w = pack16<MODE>(bv[8 * q + 6], bv[8 * q + 7]);
        *reinterpret_cast<uint4 *>(base + tid * 16 + q * kLBO)                 = pa;
        *reinterpret_cast<uint4 *>(base + kOperandBytes + tid * 16 + q * kLBO) = pbk;
      }
    } else {
#pragma unroll
      for (int q = 0; q < CHUNKS; q++) {
        uint4     ah, al, bh, bl;
        uint32_t *ahp = &ah.x, *alp = &al.x, *bhp = &bh.x, *blp = &bl.x;
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const float    x  = av[4 * q + e];
          const uint32_t xh = to_tf32(x);
          ahp[e]            = xh;
          alp[e]            = to_tf32(x - __uint_as_float(xh));
          const float    y  = bv[4 * q + e];
          const uint32_t yh = to_tf32(y);
          bhp[e]            = yh;
          blp[e]            = to_tf32(y - __uint_as_float(yh));
        }
        *reinterpret_cast<uint4 *>(base + 0 * kOperandBytes + tid * 16 + q * kLBO) = ah;
        *reinterpret_cast<uint4 *>(base + 1 * kOperandBytes + tid * 16 + q * kLBO) = al;
        *reinterpret_cast<uint4 *>(base + 2 * kOperandBytes + tid * 16 + q * kLBO) = bh;
        *reinterpret_cast<uint4 *>(base + 3 * kOperandBytes + tid * 16 + q * kLBO) = bl;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sbase = smem_u32(base);
      // Each MMA consumes two 16-byte K-chunks (16 half-precision or 8 tf32).
#pragma unroll
      for (int s = 0; s < CHUNKS / 2; s++) {
        const uint32_t off = s * 2 * kLBO;
        if (HALF) {
          mma(0, tmem, make_desc(sbase + off), make_desc(sbase + kOperandBytes + off), idesc,
              (c > 0 || s > 0) ? 1u : 0u);
        } else {
          const uint64_t ahd = make_desc(sbase + 0 * kOperandBytes + off);
          const uint64_t ald = make_desc(sbase + 1 * kOperandBytes + off);
          const uint64_t bhd = make_desc(sbase + 2 * kOperandBytes + off);
          const uint64_t bld = make_desc(sbase + 3 * kOperandBytes + off);
          mma(1, tmem, ahd, bhd, idesc, (c > 0 || s > 0) ? 1u : 0u);
          mma(1, tmem, ahd, bld, idesc, 1u);
          mma(1, tmem, ald, bhd, idesc, 1u);
        }
      }
      commit(smem_u32(&mbar[buf]));
    }
  }
  cp_async_wait<0>();  // no copy may still target shared memory at exit
  // All MMAs done: the last commit tracks every earlier one of this thread.
  if (ok && nch > 0) ok = wait_bounded(smem_u32(&mbar[(nch - 1) & 1]), ((nch - 1) >> 1) & 1);
  ok = __syncthreads_and(ok);
  if (!ok) {
    if (tid == 0) atomicExch(&st->timeout, 1);
    // Let any MMA still in flight finish before the memory is released.
    if (nch > 0) wait_bounded(smem_u32(&mbar[(nch - 1) & 1]), ((nch - 1) >> 1) & 1);
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int row  = m0 + warp * 32 + lane;
    float    *Cout = (pb.c_in_u ? uarena : panel) + pb.c_ofs;
    float    *W    = pb.splits > 1 ? ws + pb.ws_ofs +
                                         (static_cast<int64_t>(tile) * pb.splits + sp) * (kTileM * kTileN)
                                   : nullptr;
#pragma unroll
    for (int cb = 0; cb < kTileN / 32; cb++) {
      uint32_t       r[32];
      const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + cb * 32;
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
      if (nch == 0)  // an empty K range leaves the accumulator unwritten
#pragma unroll
        for (int q = 0; q < 32; q++) r[q] = 0u;
      const int lr = warp * 32 + lane;
      if (W) {
#pragma unroll
        for (int q = 0; q < 32; q++) W[lr + (cb * 32 + q) * kTileM] = __uint_as_float(r[q]);
      } else if (row < M) {
#pragma unroll
        for (int q = 0; q < 32; q++) {
          const int col = n0 + cb * 32 + q;
          if (col < N && (!pb.lower || row >= col))
            Cout[row + (int64_t)col * pb.ldc] -= __uint_as_float(r[q]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols) : "memory");
}

int tc_gemm_smem_bytes(int mode) {
  const bool half = mode != 1;
  const int  kc = half ? 32 : 16, chunks = kc * (half ? 2 : 4) / 16;
  const int  parts = half ? 1 : 2;
  // Two operand buffers of A and B parts, then the raw float32 stages; at
  // least 48 KB so that no more than four CTAs (4 x 128 tensor-memory
  // columns) share an SM.
  const int bytes = 2 * 2 * parts * tc::kTileM * chunks * 16 +
                    tc::stages_for(half) * 2 * tc::kTileM * kc * 4;
  return bytes < 49152 ? 49152 : bytes;
}

template <int MODE>
static void launch_mode(const GemmProb *probs, int nprob, int tiles, float *panel,
                        float *uarena, const float *D, float *ws, FactorStatus *st,
                        cudaStream_t s) {
  static bool attr = false;
  const int   smem = tc_gemm_smem_bytes(MODE);
  if (!attr) {
    MPIR_CUDA(cudaFuncSetAttribute(k_gemm_tc<MODE>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr = true;
  }
  launch(k_gemm_tc<MODE>, tiles, tc::kThreads, smem, s, probs, nprob, panel, uarena, D, ws, st);
}

void launch_gemm_tc(int mode, const GemmProb *probs, int nprob, int tiles, float *panel,
                    float *uarena, const float *D, float *ws, FactorStatus *st, cudaStream_t s) {
  if (mode == 0) launch_mode<0>(probs, nprob, tiles, panel, uarena, D, ws, st, s);
  else if (mode == 1) launch_mode<1>(probs, nprob, tiles, panel, uarena, D, ws, st, s);
  else launch_mode<2>(probs, nprob, tiles, panel, uarena, D, ws, st, s);
}

}  // namespace mpir
