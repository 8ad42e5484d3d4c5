// Numeric multifrontal LDL^T factorization on the GPU.
//
// The factor of P K P^T equals, entry for entry up to rounding, the one
// QDLDL_factor computes row by row (qdldl.hpp:172-345); it is organised here
// as a level-scheduled multifrontal method over the supernodal elimination
// tree instead:
//   * the scaled entries of K are scattered into zeroed panels;
//   * level by level (leaves first), each front gathers its children's
//     update matrices (extend-add), eliminates its own columns with a dense
//     partial LDL^T and leaves its Schur complement as its update matrix;
//   * fronts of at most kSmallFront rows are done whole in shared memory, one
//     thread block each; larger fronts go through a blocked right-looking
//     partial factorization whose steps are batched over all fronts of the
//     level: diagonal-block factor + inverse, a GEMM-shaped panel solve
//     (W = F L^{-T}, L = W D^{-1}) and a GEMM-shaped trailing update
//     C -= (L D) L^T.
// D is left on each panel's diagonal and copied to D / Dinv (permuted order).
#include <atomic>
#include <chrono>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "engine.hpp"

namespace mpir {

// ---------------------------------------------------------------------------
// Scaling and assembly of K's entries.

// AD_i = 1/sqrt|k_ii| when |k_ii| > eps(UF), else 1 (gmres_ir.hpp:347-356).
__global__ void k_scaling(int64_t n, const int64_t *diag_pos, const double *Ax,
                          double eps, double *AD) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double        d = 1.0;
  const int64_t p = diag_pos[i];
  if (p >= 0) {
    const double a = fabs(Ax[p]);
    if (a > eps) d = 1.0 / sqrt(a);
  }
  AD[i] = d;
}

// a_rc *= AD_r AD_c (gmres_ir.hpp:358-363) and scatter into the panels in the
// factor type.
__global__ void k_scatter(int64_t nnz, const double *Ax, const double *AD,
                          const int32_t *arow, const int32_t *acol,
                          const int64_t *amap, double *Axs, float *panel) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  const double v = Ax[p] * (AD[arow[p]] * AD[acol[p]]);
  Axs[p]         = v;
  panel[amap[p]] = static_cast<float>(v);
}

// Values of the full symmetric CSR of P K P^T: scaled and original.
__global__ void k_csr_values(int64_t nnzf, const int64_t *Ksrc,
                             const double *Axs, const double *Ax, double *Kval,
                             double *Korig) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nnzf) return;
  const int64_t p = Ksrc[e];
  Kval[e]         = Axs[p];
  Korig[e]        = Ax[p];
}

__device__ __forceinline__ void note_pivot(FactorStatus *st, int32_t col,
                                           float d, int *npos) {
  if (d == 0.0f) atomicMin(&st->zero_pivot, col);
  if (!isfinite(d)) st->nonfinite = 1;
  if (d > 0.0f) (*npos)++;
}

// ---------------------------------------------------------------------------
// Small fronts: whole front in shared memory.
template <int HMAX>
__global__ void __launch_bounds__(kSmallThreads)
    k_small_fronts(const int32_t *list, const int64_t *sfirst,
                   const int64_t *srowptr, const int64_t *slofs,
                   const int64_t *uofs, const int64_t *child_ptr,
                   const int32_t *child_list, const int32_t *srel,
                   float *panel, float *uarena, float *D, float *Dinv,
                   FactorStatus *st) {
  __shared__ float F[HMAX][HMAX + 1];
  __shared__ float wv[HMAX];
  __shared__ int   s_npos;
  const int        J   = list[blockIdx.x];
  const int        tid = threadIdx.x, bd = blockDim.x;
  const int64_t    f   = sfirst[J];
  const int        w   = static_cast<int>(sfirst[J + 1] - f);
  const int        h   = static_cast<int>(srowptr[J + 1] - srowptr[J]);
  float           *P   = panel + slofs[J];
  if (tid == 0) s_npos = 0;
  for (int idx = tid; idx < h * h; idx += bd) {
    const int i = idx % h, j = idx / h;
    F[i][j]     = (j < w && i >= j) ? P[i + (int64_t)j * h] : 0.0f;
  }
  __syncthreads();
  for (int64_t c = child_ptr[J]; c < child_ptr[J + 1]; c++) {
    const int      C  = child_list[c];
    const int      wc = static_cast<int>(sfirst[C + 1] - sfirst[C]);
    const int      rc = static_cast<int>(srowptr[C + 1] - srowptr[C]) - wc;
    const float   *U  = uarena + uofs[C];
    const int32_t *rl = srel + srowptr[C] + wc;
    for (int idx = tid; idx < rc * rc; idx += bd) {
      const int a = idx % rc, b = idx / rc;
      if (a >= b) F[rl[a]][rl[b]] += U[a + (int64_t)b * rc];
    }
    __syncthreads();
  }
  int npos = 0;
  for (int k = 0; k < w; k++) {
    const float dk = F[k][k];
    for (int i = k + 1 + tid; i < h; i += bd) wv[i] = F[i][k];
    __syncthreads();
    const float dinv = 1.0f / dk;
    const int   m    = h - k - 1;
    for (int idx = tid; idx < m * m; idx += bd) {
      const int ii = idx % m, jj = idx / m;
      if (ii >= jj) {
        const int i = k + 1 + ii, j = k + 1 + jj;
        F[i][j] -= (wv[i] * dinv) * wv[j];
      }
    }
    for (int i = k + 1 + tid; i < h; i += bd) F[i][k] = wv[i] * dinv;
    if (tid == 0) {
      D[f + k]    = dk;
      Dinv[f + k] = dinv;
      note_pivot(st, static_cast<int32_t>(f + k), dk, &npos);
    }
    __syncthreads();
  }
  if (tid == 0) atomicAdd(&st->npos, npos);
  for (int idx = tid; idx < h * w; idx += bd) {
    const int i = idx % h, j = idx / h;
    if (i >= j) P[i + (int64_t)j * h] = F[i][j];
  }
  const int r = h - w;
  if (r > 0) {
    float *U = uarena + uofs[J];
    for (int idx = tid; idx < r * r; idx += bd) {
      const int a = idx % r, b = idx / r;
      U[a + (int64_t)b * r] = a >= b ? F[w + a][w + b] : 0.0f;
    }
  }
}

// ---------------------------------------------------------------------------
// Zero the update matrices of the level's large fronts.

// Extend-add of the children's update matrices into a level's large parents,
// one CTA per chunk of at most kEaChunk parent columns (EaChunk): the
// children that add to those columns, in child order with a barrier between
// them (siblings may add to the same entries), each child's columns of the
// chunk by all threads over the child's rows.  Every parent entry receives
// its children's contributions in child order.  Within a child each thread
// takes one row at a time across the chunk's columns: the row map entry is
// loaded one row ahead and all values of U_C and of the parent are loaded
// before any store (the source and the destination may both lie in the
// update arena, so the compiler would not reorder them itself).
__global__ void __launch_bounds__(256)
    k_extend_add(const EaChunk *chunks, const EaHit *hits, const EaTask *tasks,
                 const int32_t *srel, float *panel, float *uarena) {
  const EaChunk ck   = chunks[blockIdx.x];
  const bool    in_u = ck.c0 >= ck.wp;
  // Parent entry (row ra, column cb) at base + (cb - cbase) * ld + ra: in the
  // panel (rows from 0) or in the update matrix (rows from wp).
  float *const  base  = in_u ? uarena + ck.parent_u - ck.wp : panel + ck.parent_panel;
  const int64_t ld    = in_u ? ck.hp - ck.wp : ck.hp;
  const int     cbase = in_u ? ck.wp : 0;
  for (int hh = ck.hit0; hh < ck.hit1; hh++) {
    const EaHit    hit = hits[hh];
    const EaTask   tk  = tasks[hit.task];
    const int32_t *rl  = srel + tk.rel;
    const float   *U   = uarena + tk.child_u;
    const int      nb  = hit.uhi - hit.ulo, u0 = hit.ulo;
    float         *dst[kEaChunk];
#pragma unroll
    for (int u = 0; u < kEaChunk; u++)
      dst[u] = base + static_cast<int64_t>((u < nb ? rl[u0 + u] : cbase) - cbase) * ld;
    int a  = u0 + threadIdx.x;
    int ra = a < tk.rc ? rl[a] : 0;
    for (; a < tk.rc; a += blockDim.x) {
      const int an     = a + blockDim.x;
      const int ra_nxt = an < tk.rc ? rl[an] : 0;
      float     v[kEaChunk], o[kEaChunk];
#pragma unroll
      for (int u = 0; u < kEaChunk; u++) {
        const bool ok = u < nb && a >= u0 + u;
        v[u]          = ok ? U[a + static_cast<int64_t>(u0 + u) * tk.rc] : 0.0f;
        o[u]          = ok ? dst[u][ra] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < kEaChunk; u++)
        if (u < nb && a >= u0 + u) dst[u][ra] = o[u] + v[u];
      ra = ra_nxt;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Diagonal block of one step: LDL^T of the nbk x nbk block (nbk <= 128) and
// the inverse X = L^{-1} of its unit-lower factor, right-looking by panels of
// 32 columns in shared memory (row-major copies of the block and of X; the
// block is padded with a unit diagonal up to a multiple of 32).  Panel p:
//   A. warp 0 factors the 32 x 32 diagonal block: lane = row, the pivot
//      column is broadcast by shuffles, F[i][j] -= (F[i][k] / d_k) F[j][k]
//      (the reciprocal on this chain is the fast approximate one; D^{-1}
//      itself is the correctly rounded 1 / d_k), then inverts its unit-lower
//      factor by forward substitution (lane = column).  Meanwhile warps on
//      the other three schedulers form T_pb = sum_{b <= c < p} L_pc X_cb for
//      the blocks b < p of X's row block p;
//   B. the rows below take their unscaled panel entries G = F X_pp^T
//      (G = L D) and L = G D^{-1}, both kept transposed, while the warps
//      without rows below finish X_pb = -X_pp T_pb;
//   C. L goes into the block, and the columns right of the panel take the
//      rank-32 update F[i][j] -= sum_k L[i][k] G[j][k] in 4 x 4 tiles.
// One block-wide barrier per phase; nothing of X is left for after the loop.
constexpr int kDiagLD = kNB + 1;  // Fs, Xs row stride (conflict-free columns)
constexpr int kDiagLG = 36;       // Xd row stride (16-byte rows)
constexpr int kDiagLT = 33;       // Ts row stride
constexpr int kDiagSmemFloats =
    2 * kNB * kDiagLD + 2 * 32 * kNB + 32 * kDiagLG + 3 * 32 * kDiagLT;

// Phase A of panel p for warp 0: the diagonal block at (c0, c0).  Kept out
// of line: inlined into the kernel, whose other phases hold many registers,
// its chain of shuffles is scheduled about 1.5x slower.
__device__ __noinline__ void diag_panel(float *Fs, float *Xs, float *Xd, float *dinv_s,
                                           int c0, int n, const StepDesc &d, float *D,
                                           float *Dinv, float *packd, float *packs,
                                           FactorStatus *st, int &npos) {
  constexpr int LD = kDiagLD, LG = kDiagLG;
  const int     lane = threadIdx.x % 32, r = c0 + lane;
  float         a[32];
#pragma unroll
  for (int j = 0; j < 32; j++) a[j] = Fs[r * LD + c0 + j];
  float piv = 1.0f;
#pragma unroll
  for (int k = 0; k < 32; k++) {
    const float dk = __shfl_sync(0xffffffffu, a[k], k);
    const float dv = __fdividef(1.0f, dk);
    const float l  = a[k] * dv;  // L[r][k]
#pragma unroll
    for (int j = 0; j < 32; j++) {
      if (j > k) {
        const float fjk = __shfl_sync(0xffffffffu, a[k], j);  // F[c0 + j][k]
        if (j <= lane) a[j] -= l * fjk;
      }
    }
    if (lane > k) a[k] = l;
    if (lane == k) piv = dk;
  }
  const float pinv = 1.0f / piv;
#pragma unroll
  for (int j = 0; j < 32; j++) Fs[r * LD + c0 + j] = a[j];
  dinv_s[r] = pinv;
  if (r < n) {
    const int64_t cidx = (int64_t)d.col0 + d.kb + r;
    D[cidx]            = piv;
    Dinv[cidx]         = pinv;
    if (packd != nullptr && d.pd >= 0) {
      packd[d.pd + d.kb + r] = piv;
      packs[d.pd + d.kb + r] = copysignf(sqrtf(fabsf(piv)), piv);
    }
    note_pivot(st, static_cast<int32_t>(cidx), piv, &npos);
  }
  __syncwarp();
  // X of the diagonal block (lane = column)
  float x[32];
#pragma unroll
  for (int ii = 0; ii < 32; ii++) {
    float acc = 0.0f;
#pragma unroll
    for (int kk = 0; kk < ii; kk++) acc += Fs[(c0 + ii) * LD + c0 + kk] * x[kk];
    x[ii] = ii == lane ? 1.0f : (ii > lane ? -acc : 0.0f);
  }
#pragma unroll
  for (int ii = 0; ii < 32; ii++) {
    Xs[(c0 + ii) * LD + c0 + lane] = x[ii];
    Xd[ii * LG + lane]             = x[ii];
  }
}

__global__ void __launch_bounds__(kDiagThreads)
    k_diag_block(const StepDesc *descs, float *panel, float *linv, float *D, float *Dinv,
                 float *packd, float *packs, FactorStatus *st) {
  static_assert(kDiagThreads == 4 * kNB, "diag kernel thread mapping");
  constexpr int LD = kDiagLD, LG = kDiagLG, LT = kDiagLT;
  extern __shared__ __align__(16) float sm[];
  float          *Fs = sm;             // the block, row-major
  float          *Xs = Fs + kNB * LD;  // X, row-major
  float          *Gt = Xs + kNB * LD;  // G^T of the current panel (rows below it)
  float          *Lt = Gt + 32 * kNB;  // L^T of the current panel (rows below it)
  float          *Xd = Lt + 32 * kNB;  // X of the current panel's diagonal block
  float          *Ts = Xd + 32 * LG;   // T_pb, b < p
  __shared__ float dinv_s[kNB];
  const StepDesc   d    = descs[blockIdx.x];
  const int        n    = d.nbk;
  const int        nblk = (n + 31) / 32, n32 = 32 * nblk;
  const int64_t    h    = d.h;
  const int        tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int        ri = tid % kNB, c = tid / kNB;
  float           *P  = panel + d.panel + d.kb + (int64_t)d.kb * h;
  {
    // Thread (ri, c): row ri, columns c + 4m; all loads in flight before the
    // first store.
    float v[32];
#pragma unroll
    for (int m = 0; m < 32; m++) {
      const int j = c + 4 * m;
      v[m] = (ri >= j && ri < n) ? P[ri + (int64_t)j * h] : (ri == j ? 1.0f : 0.0f);
    }
#pragma unroll
    for (int m = 0; m < 32; m++) Fs[ri * LD + c + 4 * m] = v[m];
  }
  __syncthreads();
  int npos = 0;
  for (int p = 0;; p++) {
    const int c0 = 32 * p;
    // A.
    if (warp == 0) {
      diag_panel(Fs, Xs, Xd, dinv_s, c0, n, d, D, Dinv, packd, packs, st, npos);
    } else if (warp % 4 != 0) {
      // T_pb (thread: rows 4 tr .. 4 tr + 3, columns 2 tc, 2 tc + 1 of block
      // b); these warps share no scheduler with warp 0.
      const int item = 32 * ((warp / 4) * 3 + warp % 4 - 1) + lane;
      if (item < 128 * p) {
        const int    b = item / 128, q = item % 128, tc = q % 16, tr = q / 16;
        const float *Fr = Fs + (c0 + 4 * tr) * LD;
        const float *Xc = Xs + 32 * b + 2 * tc;
        float        acc[4][2] = {};
#pragma unroll 4
        for (int k = 32 * b; k < c0; k++) {
          const float x0 = Xc[k * LD], x1 = Xc[k * LD + 1];
#pragma unroll
          for (int rr = 0; rr < 4; rr++) {
            const float f = Fr[rr * LD + k];
            acc[rr][0] += f * x0;
            acc[rr][1] += f * x1;
          }
        }
#pragma unroll
        for (int rr = 0; rr < 4; rr++) {
          Ts[b * 32 * LT + (4 * tr + rr) * LT + 2 * tc]     = acc[rr][0];
          Ts[b * 32 * LT + (4 * tr + rr) * LT + 2 * tc + 1] = acc[rr][1];
        }
      }
    }
    __syncthreads();
    // B.
    const bool below = c0 + 32 < n32;
    if (ri >= c0 + 32 && ri < n32) {
      // G = F X_pp^T (thread: row ri, columns c + 4t)
      float f[32];
#pragma unroll
      for (int k = 0; k < 32; k++) f[k] = Fs[ri * LD + c0 + k];
#pragma unroll
      for (int t = 0; t < 8; t++) {
        const int     jj  = c + 4 * t;
        const float4 *xr  = reinterpret_cast<const float4 *>(Xd + jj * LG);
        float         acc = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const float4 xv = xr[q];
          acc += f[4 * q] * xv.x;
          acc += f[4 * q + 1] * xv.y;
          acc += f[4 * q + 2] * xv.z;
          acc += f[4 * q + 3] * xv.w;
        }
        Gt[jj * kNB + ri] = acc;
        Lt[jj * kNB + ri] = acc * dinv_s[c0 + jj];
      }
    } else if (ri < c0 + 32 && p > 0) {
      // X_pb = -X_pp T_pb (lane = column) on the warps without rows below.
      const int u = (warp / 4) * (p + 1) + warp % 4, nu = 4 * (p + 1);
      for (int e = u; e < 32 * p; e += nu) {
        const int     b = e / 32, rr = e % 32;
        const float4 *xr = reinterpret_cast<const float4 *>(Xd + rr * LG);
        const float  *tb = Ts + b * 32 * LT + lane;
        float         acc[4] = {};
#pragma unroll
        for (int q = 0; q < 8; q++) {
          if (4 * q <= rr) {  // row rr of X_pp is zero right of rr
            const float4 xv = xr[q];
            acc[0] += xv.x * tb[(4 * q) * LT];
            acc[1] += xv.y * tb[(4 * q + 1) * LT];
            acc[2] += xv.z * tb[(4 * q + 2) * LT];
            acc[3] += xv.w * tb[(4 * q + 3) * LT];
          }
        }
        Xs[(c0 + rr) * LD + 32 * b + lane] = -((acc[0] + acc[1]) + (acc[2] + acc[3]));
      }
    }
    if (!below) break;
    __syncthreads();
    // C. (the panel's L into the block; the update by 4 x 4 tiles of the
    // lower triangle, row-major over the tiles)
    if (ri >= c0 + 32 && ri < n32) {
#pragma unroll
      for (int t = 0; t < 8; t++) Fs[ri * LD + c0 + c + 4 * t] = Lt[(c + 4 * t) * kNB + ri];
    }
    {
      const int mt = (n32 - c0 - 32) / 4, ntiles = mt * (mt + 1) / 2;
      if (tid < ntiles) {
        int ti = static_cast<int>((sqrtf(8.0f * tid + 1.0f) - 1.0f) * 0.5f);
        if ((ti + 1) * (ti + 2) / 2 <= tid) ti++;
        if (ti * (ti + 1) / 2 > tid) ti--;
        const int tj = tid - ti * (ti + 1) / 2;
        const int i0 = c0 + 32 + 4 * ti, j0 = c0 + 32 + 4 * tj;
        float     acc[4][4] = {};
#pragma unroll 8
        for (int k = 0; k < 32; k++) {
          const float4 lv = *reinterpret_cast<const float4 *>(Lt + k * kNB + i0);
          const float4 gv = *reinterpret_cast<const float4 *>(Gt + k * kNB + j0);
          const float  la[4] = {lv.x, lv.y, lv.z, lv.w}, ga[4] = {gv.x, gv.y, gv.z, gv.w};
#pragma unroll
          for (int r = 0; r < 4; r++)
#pragma unroll
            for (int s = 0; s < 4; s++) acc[r][s] += la[r] * ga[s];
        }
#pragma unroll
        for (int r = 0; r < 4; r++)
#pragma unroll
          for (int s = 0; s < 4; s++)
            if (j0 + s <= i0 + r) Fs[(i0 + r) * LD + j0 + s] -= acc[r][s];
      }
    }
    __syncthreads();
  }
  if (warp == 0) {
    npos = __reduce_add_sync(0xffffffffu, npos);
    if (lane == 0 && npos > 0) atomicAdd(&st->npos, npos);
  }
  __syncthreads();
  // The factor back into the panel (lower triangle) and X (blocks above the
  // diagonal blocks are zero).
#pragma unroll 4
  for (int m = 0; m < 32; m++) {
    const int j = c + 4 * m;
    if (ri >= j && ri < n) P[ri + (int64_t)j * h] = Fs[ri * LD + j];
  }
  float *Lv = linv + d.linv;
#pragma unroll 4
  for (int m = 0; m < 32; m++) {
    const int j = c + 4 * m;
    Lv[ri + j * kNB] = (ri < n && j < n && ri / 32 >= j / 32) ? Xs[ri * LD + j] : 0.0f;
  }
}

// ---------------------------------------------------------------------------
// GEMM-shaped kernels of a step (FP32 SIMT, 128x128 tiles, K in slices of 16).
//   TRSM:   C = (A B^T) .* dinv(cols), in place over A's block column;
//           A = panel rows below the block, B = Linv of the block.
//   UPDATE: C -= (A .* d(k)) B^T on the lower part; A = B = the eliminated
//           block column (rows below), C = trailing panel or update matrix.
constexpr int kBM = 128, kBN = 128, kBK = 16;

template <bool TRSM>
__global__ void __launch_bounds__(kGemmThreads)
    k_step_gemm(const StepDesc *descs, int ndesc, float *panel, float *uarena,
                const float *linv, const float *Dinv, float *pack) {
  // Two slices in shared memory: slice s+1 is loaded into registers while
  // slice s is multiplied, then stored into the other buffer.
  __shared__ float As[2][kBK][kBM];
  __shared__ float Bs[2][kBK][kBN];
  __shared__ float sd[kNB];
  const int        t  = blockIdx.x;
  int              lo = 0, hi = ndesc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    const int t0  = TRSM ? descs[mid].trsm_tile0 : descs[mid].upd_tile0;
    if (t0 <= t) lo = mid; else hi = mid - 1;
  }
  const StepDesc d     = descs[lo];
  int            local = t - (TRSM ? d.trsm_tile0 : d.upd_tile0);
  const int64_t  h     = d.h;
  const int      kb = d.kb, nbk = d.nbk, w = d.w;
  const float   *A, *B;
  float         *C;
  int64_t        lda, ldb, ldc;
  int            M, N, m0, n0;
  const int      K = nbk;
  float         *Pp = panel + d.panel;
  if (TRSM) {
    M   = static_cast<int>(h) - kb - nbk;
    N   = nbk;
    A   = Pp + (kb + nbk) + (int64_t)kb * h;
    lda = h;
    B   = linv + d.linv;
    ldb = kNB;
    C   = Pp + (kb + nbk) + (int64_t)kb * h;
    ldc = h;
    m0  = local * kBM;
    n0  = 0;
  } else {
    if (local < d.upd_panel_tiles) {
      M = static_cast<int>(h) - kb - nbk;
      N = w - kb - nbk;
      A = Pp + (kb + nbk) + (int64_t)kb * h;
      C = Pp + (kb + nbk) + (int64_t)(kb + nbk) * h;
      ldc = h;
    } else {
      local -= d.upd_panel_tiles;
      M = N = static_cast<int>(h) - w;
      A     = Pp + w + (int64_t)kb * h;
      C     = uarena + d.uofs;
      ldc   = M;
    }
    lda = ldb = h;
    B         = A;
    const int ntr = (M + kBM - 1) / kBM;
    int       j   = 0;
    while (local >= ntr - j) {
      local -= ntr - j;
      j++;
    }
    m0 = (j + local) * kBM;
    n0 = j * kBN;
    for (int k = threadIdx.x; k < nbk; k += blockDim.x)
      sd[k] = Pp[(kb + k) + (int64_t)(kb + k) * h];
  }
  const int tid = threadIdx.x;
  const int tr = tid / 16, tc = tid % 16;
  float     acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
  __syncthreads();
  constexpr int kLoads = (kBM * kBK) / kGemmThreads;
  float         ra[kLoads], rb[kLoads];
  auto          load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < kLoads; q++) {
      const int idx = tid + q * kGemmThreads;
      const int i = idx % kBM, kk = idx / kBM;
      const int r = m0 + i, k = k0 + kk;
      float     v = 0.0f;
      if (r < M && k < K) {
        v = A[r + (int64_t)k * lda];
        if (!TRSM) v *= sd[k];
      }
      ra[q]       = v;
      const int c = n0 + i;
      rb[q]       = (c < N && k < K) ? B[c + (int64_t)k * ldb] : 0.0f;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int q = 0; q < kLoads; q++) {
      const int idx = tid + q * kGemmThreads;
      As[buf][idx / kBM][idx % kBM] = ra[q];
      Bs[buf][idx / kBM][idx % kBM] = rb[q];
    }
  };
  load(0);
  store(0);
  __syncthreads();
  int buf = 0;
  for (int k0 = 0; k0 < K; k0 += kBK) {
    if (k0 + kBK < K) load(k0 + kBK);  // in flight during this slice
#pragma unroll
    for (int kk = 0; kk < kBK; kk++) {
      float a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = As[buf][kk][tr * 8 + i];
#pragma unroll
      for (int j = 0; j < 8; j++) b[j] = Bs[buf][kk][tc * 8 + j];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    if (k0 + kBK < K) {
      store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
  if (!TRSM) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = n0 + tc * 8 + j;
      if (c >= N) continue;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int r = m0 + tr * 8 + i;
        if (r < M && r >= c) C[r + (int64_t)c * ldc] -= acc[i][j];
      }
    }
    return;
  }
  // TRSM epilogue: the tile times Dinv goes through shared memory, then to
  // the panel as 128-row column segments (one warp per column) and to the
  // packed front as whole 2 KB K-groups (PackedFront), both coalesced.
  extern __shared__ float tile_s[];  // kBM x (kBN + 1)
  constexpr int           LT = kBN + 1;
  float                   dvs[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int c = n0 + tc * 8 + j;
    dvs[j]      = c < N ? Dinv[(int64_t)d.col0 + kb + c] : 0.0f;
  }
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) tile_s[(tr * 8 + i) * LT + tc * 8 + j] = acc[i][j] * dvs[j];
  __syncthreads();
  const int warp = tid / 32, lane = tid % 32;
  for (int c = warp; c < N; c += kGemmThreads / 32)
#pragma unroll
    for (int q = 0; q < kBM / 32; q++) {
      const int r = lane + 32 * q;
      if (m0 + r < M) C[m0 + r + (int64_t)c * ldc] = tile_s[r * LT + c];
    }
  if (pack != nullptr && d.pk >= 0) {
    float *pk = pack + d.pk;
    for (int e = tid; e < kBM * (kBN / 4); e += kGemmThreads) {
      const int m = e % kBM, g = e / kBM, c0 = 4 * g;
      if (c0 >= N || m0 + m >= M) continue;
      const int rf = kb + nbk + m0 + m;  // row of the front
      const int p  = rf < w ? rf : rf - w + d.pk_wt;
      float4    v;
      v.x = tile_s[m * LT + c0 + 0];
      v.y = tile_s[m * LT + c0 + 1];
      v.z = tile_s[m * LT + c0 + 2];
      v.w = tile_s[m * LT + c0 + 3];
      *reinterpret_cast<float4 *>(pk +
                                  static_cast<int64_t>(p >> 7) * d.pk_g * PackedFront::kGroupFloats +
                                  static_cast<int64_t>((kb + c0) >> 2) * PackedFront::kGroupFloats +
                                  (p & 127) * 4) = v;
    }
  }
}

// ---------------------------------------------------------------------------
// GemmProb updates on the SIMT units (float32), the same tile and split
// mapping as the tensor-core kernel.
__device__ __forceinline__ void locate_tile(const GemmProb &pb, int local, int &sp, int &tile,
                                            int &m0, int &n0) {
  sp     = local % pb.splits;
  int tl = local / pb.splits;
  tile   = tl;
  int j  = 0;
  if (pb.lower) {
    while (tl >= pb.ntm - j) {
      tl -= pb.ntm - j;
      j++;
    }
    m0 = (j + tl) * kBM;
  } else {
    j  = tl / pb.ntm;
    m0 = (tl % pb.ntm) * kBM;
  }
  n0 = j * kBN;
}

__global__ void __launch_bounds__(kGemmThreads)
    k_gemm_simt(const GemmProb *probs, int nprob, float *panel, float *uarena, const float *D,
                float *ws) {
  __shared__ float As[kBK][kBM];
  __shared__ float Bs[kBK][kBN];
  const int        t  = blockIdx.x;
  int              lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (probs[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const GemmProb pb = probs[lo];
  int            sp, tile, m0, n0;
  locate_tile(pb, t - pb.tile0, sp, tile, m0, n0);
  const int     M = pb.M, N = pb.N, K = pb.K;
  const int     ks   = ((K + pb.splits - 1) / pb.splits + 31) / 32 * 32;
  const int     k_lo = sp * ks, k_hi = min(K, k_lo + ks);
  const float  *A    = panel + pb.a_ofs;
  const int64_t lda  = pb.lda;
  const float  *Dk   = D + pb.d_ofs;
  const int     tid  = threadIdx.x;
  const int     tr = tid / 16, tc = tid % 16;
  float         acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
  for (int k0 = k_lo; k0 < k_hi; k0 += kBK) {
#pragma unroll
    for (int q = 0; q < (kBM * kBK) / kGemmThreads; q++) {
      const int idx = tid + q * kGemmThreads;
      const int i = idx % kBM, kk = idx / kBM;
      const int k = k0 + kk;
      const bool kin = k < k_hi;
      const int r = m0 + i < M ? gemm_out_row(pb, m0 + i) : -1, c = n0 + i;
      As[kk][i] = (r >= 0 && kin) ? A[r + (int64_t)k * lda] * Dk[k] : 0.0f;
      Bs[kk][i] = (c < N && kin) ? A[c + (int64_t)k * lda] : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kBK; kk++) {
      float a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; i++) a[i] = As[kk][tr * 8 + i];
#pragma unroll
      for (int j = 0; j < 8; j++) b[j] = Bs[kk][tc * 8 + j];
#pragma unroll
      for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  if (pb.splits > 1) {
    float *W = ws + pb.ws_ofs + (static_cast<int64_t>(tile) * pb.splits + sp) * (kBM * kBN);
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int i = 0; i < 8; i++) W[(tr * 8 + i) + (tc * 8 + j) * kBM] = acc[i][j];
    return;
  }
  float *C = (pb.c_in_u ? uarena : panel) + pb.c_ofs;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int c = n0 + tc * 8 + j;
    if (c >= N) continue;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const int r = m0 + tr * 8 + i < M ? gemm_out_row(pb, m0 + tr * 8 + i) : -1;
      if (r >= 0 && (!pb.lower || r >= c))
        C[r + (int64_t)c * pb.ldc] = (pb.c_in_u ? 0.0f : C[r + (int64_t)c * pb.ldc]) - acc[i][j];
    }
  }
}

// C -= sum of the split partials of one tile, added in split order.  A tile
// is reduced by kReduceSlices CTAs, one float4 group (4 consecutive rows of a
// column) per thread: the late left-looking steps of a large front have a
// few tiles and many splits, so one CTA per tile would sum long chains
// alone.  The partials are loaded four splits at a time and added in order.
constexpr int kReduceSlices = 16;

__global__ void __launch_bounds__(256)
    k_split_reduce(const GemmProb *probs, int nprob, float *panel, float *uarena,
                   const float *ws) {
  static_assert(kBM * kBN / 4 == kReduceSlices * 256, "one float4 group per thread");
  const int t = blockIdx.x / kReduceSlices, slice = blockIdx.x % kReduceSlices;
  int       lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (probs[mid].rtile0 <= t) lo = mid; else hi = mid - 1;
  }
  const GemmProb pb = probs[lo];
  int            sp, tile, m0, n0;
  locate_tile(pb, (t - pb.rtile0) * pb.splits, sp, tile, m0, n0);
  float         *C  = (pb.c_in_u ? uarena : panel) + pb.c_ofs;
  const int      g  = slice * 256 + threadIdx.x;
  const float4  *W  = reinterpret_cast<const float4 *>(
                         ws + pb.ws_ofs + static_cast<int64_t>(tile) * pb.splits * (kBM * kBN)) + g;
  constexpr int  kT = kBM * kBN / 4;  // float4 groups of a tile
  float4         acc = make_float4(0.f, 0.f, 0.f, 0.f);
  int            q   = 0;
  for (; q + 4 <= pb.splits; q += 4) {
    float4 v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) v[u] = __ldcs(W + static_cast<int64_t>(q + u) * kT);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      acc.x += v[u].x;
      acc.y += v[u].y;
      acc.z += v[u].z;
      acc.w += v[u].w;
    }
  }
  for (; q < pb.splits; q++) {
    const float4 v = __ldcs(W + static_cast<int64_t>(q) * kT);
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
    acc.w += v.w;
  }
  const int   e = 4 * g;
  const int   c = n0 + e / kBM;
  int64_t     at[4];
  float       cv[4];
  const float a[4] = {acc.x, acc.y, acc.z, acc.w};
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const int m = m0 + e % kBM + v;
    const int r = m < pb.M ? gemm_out_row(pb, m) : -1;
    at[v] = (r < 0 || c >= pb.N || (pb.lower && r < c)) ? -1 : r + (int64_t)c * pb.ldc;
    cv[v] = (!pb.c_in_u && at[v] >= 0) ? C[at[v]] : 0.0f;
  }
#pragma unroll
  for (int v = 0; v < 4; v++)
    if (at[v] >= 0) C[at[v]] = cv[v] - a[v];
}

// Inverses, in float64, of the unit-lower diagonal blocks of the large
// fronts, for the triangular solves: run once after a factorization (off its
// critical path), and for a factor supplied by the caller (the QDLDL_solve
// entry point).
__global__ void __launch_bounds__(kDiagThreads)
    k_invert_blocks(const StepDesc *descs, const float *panel, double *linv64,
                    double *linv64t) {
  extern __shared__ double smd[];
  constexpr int            LD = kNB + 1;
  double                  *X  = smd;
  float                   *F  = reinterpret_cast<float *>(smd + kNB * LD);
  const StepDesc           d  = descs[blockIdx.x];
  const int                n  = d.nbk;
  const int64_t            h  = d.h;
  const int                tid = threadIdx.x, bd = blockDim.x;
  const float             *P   = panel + d.panel + d.kb + (int64_t)d.kb * h;
  for (int idx = tid; idx < n * n; idx += bd) {
    const int i = idx % n, j = idx / n;
    F[i * LD + j] = i > j ? P[i + (int64_t)j * h] : 0.0f;
    X[i * LD + j] = i == j ? 1.0 : 0.0;
  }
  __syncthreads();
  // Step k subtracts L[i][k] X[k][j] from X[i][j] for all i > k, j <= k:
  // thread (i, g) = (tid % kNB, tid / kNB) takes row i and the columns
  // j = g, g + 4, ... (every entry gets its terms in increasing k).
  static_assert(kDiagThreads == 4 * kNB, "invert thread mapping");
  const int ri = tid % kNB, g = tid / kNB;
  for (int k = 0; k < n; k++) {
    if (ri > k && ri < n) {
      const double f = static_cast<double>(F[ri * LD + k]);
      for (int j = g; j <= k; j += 4) X[ri * LD + j] -= f * X[k * LD + j];
    }
    __syncthreads();
  }
  double *Ld = linv64 + d.linv, *Lt = linv64t + d.linv;
  for (int idx = tid; idx < kNB * kNB; idx += bd) {
    const int    i = idx % kNB, j = idx / kNB;
    const double v = (i < n && j < n) ? X[i * LD + j] : 0.0;
    Ld[i + j * kNB] = v;
    Lt[i * kNB + j] = v;
  }
}

// The panels rounded to bfloat16 (bf != 0) or float16 for the solves of the
// 16-bit tiers: L is stored in the tier's type and the solves read half the
// bytes (their arithmetic stays float64).
__global__ void k_panel_to16(int64_t n, const float *in, uint16_t *out, int bf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (bf) {
      const __nv_bfloat16 v = __float2bfloat16_rn(in[i]);
      out[i]                = *reinterpret_cast<const uint16_t *>(&v);
    } else {
      const __half v = __float2half_rn(in[i]);
      out[i]         = *reinterpret_cast<const uint16_t *>(&v);
    }
  }
}

void invert_diag_blocks(const Plan &P, Numeric &F, cudaStream_t s) {
  if (P.ndesc == 0) return;
  const int smem = kNB * (kNB + 1) * (sizeof(double) + sizeof(float));
  MPIR_CUDA(cudaFuncSetAttribute(k_invert_blocks,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  launch(k_invert_blocks, static_cast<unsigned>(P.ndesc), kDiagThreads, smem, s,
         P.steps.as<StepDesc>(), F.panel.as<float>(), F.linv64.as<double>(),
         F.linv64t.as<double>());
  MPIR_CHECK_LAUNCH();
}

// ---------------------------------------------------------------------------
// Plan construction.

void Plan::build(Symbolic &&sym, cudaStream_t s, bool upload) {
  S              = std::move(sym);
  const int64_t ns = S.ns;
  nnz_full         = static_cast<int64_t>(S.Kj.size());
  // Persistent Linv storage for the large fronts.
  linv_ofs.assign(ns, -1);
  linv_elems   = 0;
  spart_elems  = 0;
  nblock_fronts = 0;
  h_swarp.clear();
  h_sblock.clear();
  std::vector<int64_t> gp_h, gsrc_h;
  std::vector<int32_t>   chunk_map_h;
  std::vector<SolveItem> fwd_item_h, own_item_h;
  std::vector<SolveFront> sfronts;
  update_flops = 0;
  trsm_flops   = 0;
  pk_ofs.assign(ns, -1);
  pd_ofs.assign(ns, -1);
  pk_elems = pd_elems = 0;
  for (int64_t J = 0; J < ns; J++)
    if (is_large(J)) {
      linv_ofs[J] = linv_elems;
      linv_elems += ((S.w(J) + kNB - 1) / kNB) * (int64_t)kNB * kNB;
      pk_ofs[J] = pk_elems;
      pk_elems += pk_tiles(J) * pk_groups(J) * PackedFront::kGroupFloats;
      pd_ofs[J] = pd_elems;
      pd_elems += pk_groups(J) * 4;
    }
  // Per-level launch lists.
  levels.assign(S.nlevels, LevelPlan{});
  h_small.clear();
  h_large.clear();
  std::vector<StepDesc> descs;
  std::vector<EaTask>   tasks;
  std::vector<EaChunk>  chunks_h;
  std::vector<EaHit>    hits_h;
  std::vector<GemmProb> probs;
  ws_elems    = 0;
  bconv_elems = 0;
  // Tiles, K splits, launch offsets and workspace of the problems
  // [begin, begin + count) of one launch.  With fewer tiles than about two
  // per SM, K is split (at least 256 per split) and the partials reduced.
  auto finish_launch = [&](int32_t begin, int32_t count, int32_t &tiles, int32_t &rtiles,
                           int32_t &convs) {
    int64_t total = 0;
    for (int32_t q = begin; q < begin + count; q++) {
      GemmProb &g  = probs[q];
      g.ntm        = (g.M + kBM - 1) / kBM;
      const int nn = (g.N + kBN - 1) / kBN;
      g.ntiles     = g.lower ? nn * g.ntm - nn * (nn - 1) / 2 : nn * g.ntm;
      total += g.ntiles;
      const double Mr = g.M, Nc = g.N;
      update_flops += 2.0 * g.K * (g.lower ? Nc * Mr - Nc * (Nc - 1) / 2 : Nc * Mr);
    }
    // Splits of K: the count s (at least 256 of K per split) that minimises
    // waves(total tiles x s over the resident CTAs) x (K / s + a fixed cost
    // per CTA of about 128 columns of K); partial tiles are reduced after.
    const int64_t resident = static_cast<int64_t>(kSMs) * tc_ctas_per_sm();
    int64_t       kmax     = 0;
    for (int32_t q = begin; q < begin + count; q++) kmax = std::max<int64_t>(kmax, probs[q].K);
    int64_t best_s = 1;
    double  best_c = 1e300;
    for (int64_t sp = 1; sp <= std::max<int64_t>(1, kmax / 256); sp++) {
      const double waves = static_cast<double>((total * sp + resident - 1) / resident);
      const double c     = waves * (static_cast<double>((kmax + sp - 1) / sp) + 128.0);
      if (c < best_c - 1e-9) {
        best_c = c;
        best_s = sp;
      }
    }
    int64_t t0 = 0, r0 = 0, w0 = 0;
    for (int32_t q = begin; q < begin + count; q++) {
      GemmProb &g = probs[q];
      g.splits    = 1;
      const int64_t want = std::max<int64_t>(1, std::min<int64_t>(best_s, g.K / 256));
      if (want > 1) {
        // Split length as the kernels compute it (a multiple of 32); then as
        // many splits as that length needs, so no split is empty.
        const int64_t ks = ((g.K + want - 1) / want + 31) / 32 * 32;
        g.splits         = static_cast<int32_t>((g.K + ks - 1) / ks);
      }
      g.tile0  = static_cast<int32_t>(t0);
      t0 += static_cast<int64_t>(g.ntiles) * g.splits;
      g.rtile0 = static_cast<int32_t>(r0);
      g.ws_ofs = -1;
      if (g.splits > 1) {
        r0 += g.ntiles;
        g.ws_ofs = w0;
        w0 += static_cast<int64_t>(g.ntiles) * g.splits * kBM * kBN;
      }
    }
    tiles    = static_cast<int32_t>(t0);
    rtiles   = static_cast<int32_t>(r0);
    ws_elems = std::max(ws_elems, w0);
    // B converted once per launch for the 3xTF32 product: the problem's B
    // row tiles, all K-groups its K range reads.
    int64_t c0 = 0, b0 = 0;
    for (int32_t q = begin; q < begin + count; q++) {
      GemmProb &g = probs[q];
      g.btiles    = (g.N + kBN - 1) / kBN;
      g.bgroups   = static_cast<int32_t>((g.K + 31) / 32 * 8);
      g.bprow     = static_cast<int64_t>(g.bgroups) * PackedFront::kGroupFloats;
      g.bc        = b0;
      g.bc_lo     = b0 + g.btiles * g.bprow;
      b0 += 2 * g.btiles * g.bprow;
      g.cv0 = static_cast<int32_t>(c0);
      c0 += static_cast<int64_t>(g.btiles) * ((g.bgroups + kConvGroups - 1) / kConvGroups);
    }
    convs       = static_cast<int32_t>(c0);
    bconv_elems = std::max(bconv_elems, b0);
  };
  for (int32_t t = 0; t < S.nlevels; t++) {
    LevelPlan &L = levels[t];
    L.small_begin = static_cast<int32_t>(h_small.size());
    L.large_begin = static_cast<int32_t>(h_large.size());
    for (int64_t q = S.level_ptr[t]; q < S.level_ptr[t + 1]; q++) {
      const int32_t J = S.level_sup[q];
      (is_large(J) ? h_large : h_small).push_back(J);
    }
    L.small_count = static_cast<int32_t>(h_small.size()) - L.small_begin;
    L.large_count = static_cast<int32_t>(h_large.size()) - L.large_begin;
    // Extend-add: per phase (the parents' panel columns, then their update
    // matrices' columns) one CTA per chunk of kEaChunk parent columns that a
    // child adds to, with those children's hits in child order.
    std::vector<int32_t> task0(L.large_count);
    for (int32_t q = L.large_begin; q < L.large_begin + L.large_count; q++) {
      const int64_t P = h_large[q];
      task0[q - L.large_begin] = static_cast<int32_t>(tasks.size());
      for (int64_t c = S.child_ptr[P]; c < S.child_ptr[P + 1]; c++) {
        const int64_t C = S.child_list[c];
        EaTask        tk;
        tk.child_u = S.uofs[C];
        tk.rel     = S.srowptr[C] + S.w(C);
        tk.rc      = static_cast<int32_t>(S.h(C) - S.w(C));
        tk.pad     = 0;
        tasks.push_back(tk);
      }
    }
    for (int ph = 0; ph < 2; ph++) {
      L.ea_begin[ph] = static_cast<int32_t>(chunks_h.size());
      for (int32_t q = L.large_begin; q < L.large_begin + L.large_count; q++) {
        const int64_t P  = h_large[q];
        const int64_t nk = S.child_ptr[P + 1] - S.child_ptr[P];
        const int32_t hp = static_cast<int32_t>(S.h(P)), wp = static_cast<int32_t>(S.w(P));
        const int32_t lo = ph == 0 ? 0 : wp, hi = ph == 0 ? wp : hp;
        if (nk == 0 || hi <= lo) continue;
        const int32_t nch = (hi - lo + kEaChunk - 1) / kEaChunk;
        // Hits per chunk (counted, then placed), children in order: a child's
        // columns in one chunk are consecutive (its row map increases).
        std::vector<int32_t> cnt(nch + 1, 0);
        auto walk = [&](auto &&emit) {
          for (int64_t k = 0; k < nk; k++) {
            const int32_t  tix = task0[q - L.large_begin] + static_cast<int32_t>(k);
            const EaTask  &tk  = tasks[tix];
            const int32_t *rl  = S.srel.data() + tk.rel;
            int32_t        u   = 0;
            while (u < tk.rc && rl[u] < lo) u++;
            while (u < tk.rc && rl[u] < hi) {
              const int32_t ch = (rl[u] - lo) / kEaChunk, end = lo + (ch + 1) * kEaChunk;
              int32_t       v  = u;
              while (v < tk.rc && rl[v] < std::min(end, hi)) v++;
              emit(ch, tix, u, v);
              u = v;
            }
          }
        };
        walk([&](int32_t ch, int32_t, int32_t, int32_t) { cnt[ch + 1]++; });
        for (int32_t c = 0; c < nch; c++) cnt[c + 1] += cnt[c];
        const int32_t        hbase = static_cast<int32_t>(hits_h.size());
        std::vector<int32_t> fill(cnt.begin(), cnt.end() - 1);
        hits_h.resize(hits_h.size() + cnt[nch]);
        walk([&](int32_t ch, int32_t tix, int32_t u, int32_t v) {
          hits_h[hbase + fill[ch]++] = EaHit{tix, u, v, 0};
        });
        for (int32_t c = 0; c < nch; c++) {
          if (cnt[c + 1] == cnt[c]) continue;  // no child adds to these columns
          EaChunk ck;
          ck.parent_panel = S.slofs[P];
          ck.parent_u     = S.uofs[P];
          ck.hp           = hp;
          ck.wp           = wp;
          ck.c0           = lo + c * kEaChunk;
          ck.nc           = std::min(kEaChunk, hi - ck.c0);
          ck.hit0         = hbase + cnt[c];
          ck.hit1         = hbase + cnt[c + 1];
          chunks_h.push_back(ck);
        }
      }
      L.ea_count[ph] = static_cast<int32_t>(chunks_h.size()) - L.ea_begin[ph];
    }
    // Blocked steps.  Step kb: the left-looking update of block column kb
    // by the columns before it, then its diagonal block and panel solve;
    // after the last step the update matrix, in one product.
    int64_t maxw = 0;
    for (int32_t q = L.large_begin; q < L.large_begin + L.large_count; q++)
      maxw = std::max(maxw, S.w(h_large[q]));
    for (int64_t kb = 0; kb < maxw; kb += kNB) {
      LevelPlan::Step st{static_cast<int32_t>(descs.size()), 0, 0, 0,
                         static_cast<int32_t>(probs.size()), 0, 0, 0, 0};
      for (int32_t q = L.large_begin; q < L.large_begin + L.large_count; q++) {
        const int64_t J = h_large[q], w = S.w(J), h = S.h(J);
        if (w <= kb) continue;
        StepDesc d;
        d.panel  = S.slofs[J];
        d.uofs   = S.uofs[J];
        d.linv   = linv_ofs[J] + (kb / kNB) * (int64_t)kNB * kNB;
        d.h      = static_cast<int32_t>(h);
        d.w      = static_cast<int32_t>(w);
        d.kb     = static_cast<int32_t>(kb);
        d.nbk    = static_cast<int32_t>(std::min<int64_t>(kNB, w - kb));
        d.col0   = static_cast<int32_t>(S.sfirst[J]);
        const int64_t M = h - kb - d.nbk;
        d.trsm_tile0    = st.trsm_tiles;
        st.trsm_tiles += static_cast<int32_t>((M + kBM - 1) / kBM);
        d.upd_tile0       = 0;
        d.upd_panel_tiles = 0;
        trsm_flops += 2.0 * d.nbk * static_cast<double>(d.nbk) * static_cast<double>(M);
        if (kb > 0) {
          // Rows kb .. h-1 in the packed numbering: kb .. w-1, the gap up to
          // Wt, then the off-diagonal rows.
          const int64_t wt = pk_wt(J);
          GemmProb g{};
          g.a_ofs  = S.slofs[J] + kb;
          g.lda    = static_cast<int32_t>(h);
          g.c_ofs  = S.slofs[J] + kb + kb * h;
          g.ldc    = static_cast<int32_t>(h);
          g.d_ofs  = S.sfirst[J];
          g.prow   = pk_groups(J) * PackedFront::kGroupFloats;
          g.pa     = pk_ofs[J] + (kb / PackedFront::kRowTile) * g.prow;
          g.pb     = g.pa;
          g.pd     = pd_ofs[J];
          g.gap_at = static_cast<int32_t>(w - kb);
          g.gap    = static_cast<int32_t>(h > w ? wt - w : 0);
          g.M      = static_cast<int32_t>(h > w ? wt + (h - w) - kb : w - kb);
          g.N      = d.nbk;
          g.K      = static_cast<int32_t>(kb);
          g.c_in_u = 0;
          g.lower  = 1;
          probs.push_back(g);
        }
        d.pk           = pk_ofs[J];
        d.pd           = pd_ofs[J];
        d.pk_g         = static_cast<int32_t>(pk_groups(J));
        d.pk_wt        = static_cast<int32_t>(pk_wt(J));
        descs.push_back(d);
        st.count++;
      }
      st.ll_count = static_cast<int32_t>(probs.size()) - st.ll_begin;
      finish_launch(st.ll_begin, st.ll_count, st.ll_tiles, st.ll_rtiles, st.ll_convs);
      L.steps.push_back(st);
    }
    // Solve work of the level: narrow, short fronts one warp each, the rest
    // through SolveFront entries.
    L.sw_begin = static_cast<int32_t>(h_swarp.size());
    L.sf_begin = static_cast<int32_t>(sfronts.size());
    for (int32_t q = L.small_begin; q < L.small_begin + L.small_count; q++)
      h_swarp.push_back(h_small[q]);
    int64_t spart = 0;
    for (int32_t q = L.large_begin; q < L.large_begin + L.large_count; q++) {
      const int64_t J = h_large[q], w = S.w(J), h = S.h(J);
      if (w <= kWarpSolveW && h <= kWarpSolveH) {
        h_swarp.push_back(J);
        continue;
      }
      h_sblock.push_back(J);
      SolveFront    f{};
      // Child contributions per row, in child order (the forward solve adds
      // them in this order).
      f.rows = S.srowptr[J];
      f.gptr = static_cast<int64_t>(gp_h.size());
      {
        std::vector<int64_t> cnt(h + 1, 0);
        for (int64_t c = S.child_ptr[J]; c < S.child_ptr[J + 1]; c++) {
          const int64_t C = S.child_list[c], wc = S.w(C), rc = S.h(C) - wc;
          for (int64_t a = 0; a < rc; a++) cnt[S.srel[S.srowptr[C] + wc + a] + 1]++;
        }
        for (int64_t i = 0; i < h; i++) cnt[i + 1] += cnt[i];
        const int64_t base = static_cast<int64_t>(gsrc_h.size());
        for (int64_t i = 0; i <= h; i++) gp_h.push_back(base + cnt[i]);
        gsrc_h.resize(base + cnt[h]);
        for (int64_t c = S.child_ptr[J]; c < S.child_ptr[J + 1]; c++) {
          const int64_t C = S.child_list[c], wc = S.w(C), rc = S.h(C) - wc;
          for (int64_t a = 0; a < rc; a++)
            gsrc_h[base + cnt[S.srel[S.srowptr[C] + wc + a]]++] = S.zofs[C] + wc + a;
        }
      }
      f.panel  = S.slofs[J];
      f.zofs   = S.zofs[J];
      f.linv   = linv_ofs[J];
      f.h      = static_cast<int32_t>(h);
      f.w      = static_cast<int32_t>(w);
      f.nb     = static_cast<int32_t>((w + kNB - 1) / kNB);
      f.col0   = static_cast<int32_t>(S.sfirst[J]);
      f.n      = static_cast<int32_t>(S.n);
      nblock_fronts++;
      L.fwd_items += static_cast<int32_t>((h + kNB - 1) / kNB);
      f.chunks = static_cast<int32_t>((h - w + kNB - 1) / kNB);
      f.chunk0 = L.bwd_chunk_items;
      L.bwd_chunk_items += f.chunks;
      f.part   = spart;
      spart += static_cast<int64_t>(f.chunks) * w;
      f.own0   = L.bwd_owner_items;
      L.bwd_owner_items += f.nb;
      sfronts.push_back(f);
    }
    L.sf_count  = static_cast<int32_t>(sfronts.size()) - L.sf_begin;
    // Item -> front maps of the level's solve launches.
    L.fwd_map0   = static_cast<int64_t>(fwd_item_h.size());
    L.chunk_map0 = static_cast<int64_t>(chunk_map_h.size());
    L.own_map0   = static_cast<int64_t>(own_item_h.size());
    // Forward: every front's diagonal row blocks first (their chains start
    // together), then the off-diagonal row blocks, which wait on them.
    for (int32_t q = 0; q < L.sf_count; q++) {
      const SolveFront &f = sfronts[L.sf_begin + q];
      for (int32_t i = 0; i < f.nb; i++) fwd_item_h.push_back(SolveItem{f, i, 0});
    }
    for (int32_t q = 0; q < L.sf_count; q++) {
      const SolveFront &f = sfronts[L.sf_begin + q];
      for (int32_t i = f.nb; i < (f.h + kNB - 1) / kNB; i++)
        fwd_item_h.push_back(SolveItem{f, i, 0});
    }
    // Backward: each front's column blocks, last first.
    for (int32_t q = 0; q < L.sf_count; q++) {
      const SolveFront &f = sfronts[L.sf_begin + q];
      for (int32_t i = 0; i < f.chunks; i++) chunk_map_h.push_back(q);
      for (int32_t i = 0; i < f.nb; i++) own_item_h.push_back(SolveItem{f, f.nb - 1 - i, 0});
    }
    L.sw_count  = static_cast<int32_t>(h_swarp.size()) - L.sw_begin;
    spart_elems = std::max(spart_elems, spart);
    L.u_begin = static_cast<int32_t>(probs.size());
    for (int32_t q = L.large_begin; q < L.large_begin + L.large_count; q++) {
      const int64_t J = h_large[q], w = S.w(J), h = S.h(J), r = h - w;
      if (r <= 0) continue;
      GemmProb g{};
      g.a_ofs  = S.slofs[J] + w;
      g.lda    = static_cast<int32_t>(h);
      g.c_ofs  = S.uofs[J];
      g.ldc    = static_cast<int32_t>(r);
      g.d_ofs  = S.sfirst[J];
      g.prow   = pk_groups(J) * PackedFront::kGroupFloats;
      g.pa     = pk_ofs[J] + (pk_wt(J) / PackedFront::kRowTile) * g.prow;
      g.pb     = g.pa;
      g.pd     = pd_ofs[J];
      g.gap_at = static_cast<int32_t>(r);
      g.gap    = 0;
      g.M = g.N = static_cast<int32_t>(r);
      g.K      = static_cast<int32_t>(w);
      g.c_in_u = 1;
      g.lower  = 1;
      probs.push_back(g);
    }
    L.u_count = static_cast<int32_t>(probs.size()) - L.u_begin;
    finish_launch(L.u_begin, L.u_count, L.u_tiles, L.u_rtiles, L.u_convs);
  }
  ndesc = static_cast<int64_t>(descs.size());
  panel_read_bytes = 0;
  for (int64_t J = 0; J < ns; J++) {
    const double w = static_cast<double>(S.w(J)), h = static_cast<double>(S.h(J));
    panel_read_bytes += 4.0 * (w * h - w * (w - 1) / 2);
  }
  sync_elems = 2 * static_cast<int64_t>(levels.size());
  // The host arrays stay with the plan, so an evicted plan can go back to
  // the device without being built again.
  host_.descs       = std::move(descs);
  host_.tasks       = std::move(tasks);
  host_.chunks      = std::move(chunks_h);
  host_.hits        = std::move(hits_h);
  host_.probs       = std::move(probs);
  host_.sfronts     = std::move(sfronts);
  host_.gp          = std::move(gp_h);
  host_.gsrc        = std::move(gsrc_h);
  host_.fwd_item    = std::move(fwd_item_h);
  host_.chunk_map   = std::move(chunk_map_h);
  host_.own_item    = std::move(own_item_h);
  if (upload) upload_all(s);
}

size_t Plan::upload_bytes() const {
  auto b = [](const auto &v) { return v.size() * sizeof(v[0]); };
  return b(S.amap) + b(S.arow) + b(S.acol) + b(S.diag_pos) + b(S.Kp) + b(S.Kj) + b(S.Ksrc) +
         b(S.sfirst) + b(S.srowptr) + b(S.srows) + b(S.srel) + b(S.slofs) + b(S.uofs) +
         b(S.zofs) + b(S.child_ptr) + b(S.child_list) + b(S.perm) + b(h_small) + b(h_large) +
         b(host_.descs) + b(host_.tasks) + b(host_.chunks) + b(host_.hits) + b(host_.probs) +
         b(linv_ofs) + b(host_.sfronts) + b(h_swarp) + b(h_sblock) + b(host_.gp) +
         b(host_.gsrc) + b(host_.fwd_item) + b(host_.chunk_map) + b(host_.own_item);
}

void Plan::upload_all(cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
  amap       = upload(S.amap, s);
  arow       = upload(S.arow, s);
  acol       = upload(S.acol, s);
  diag_pos   = upload(S.diag_pos, s);
  Kp         = upload(S.Kp, s);
  Kj         = upload(S.Kj, s);
  Ksrc       = upload(S.Ksrc, s);
  sfirst     = upload(S.sfirst, s);
  srowptr    = upload(S.srowptr, s);
  srows      = upload(S.srows, s);
  srel       = upload(S.srel, s);
  slofs      = upload(S.slofs, s);
  uofs       = upload(S.uofs, s);
  zofs       = upload(S.zofs, s);
  child_ptr  = upload(S.child_ptr, s);
  child_list = upload(S.child_list, s);
  perm       = upload(S.perm, s);
  small_list = upload(h_small, s);
  large_list = upload(h_large, s);
  steps      = upload(host_.descs, s);
  ea_tasks   = upload(host_.tasks, s);
  ea_chunks  = upload(host_.chunks, s);
  ea_hits    = upload(host_.hits, s);
  gemm_probs = upload(host_.probs, s);
  linv_ofs_d = upload(linv_ofs, s);
  solve_fronts = upload(host_.sfronts, s);
  swarp_list   = upload(h_swarp, s);
  sblock_list  = upload(h_sblock, s);
  gp           = upload(host_.gp, s);
  gsrc         = upload(host_.gsrc, s);
  fwd_item     = upload(host_.fwd_item, s);
  chunk_map    = upload(host_.chunk_map, s);
  own_item     = upload(host_.own_item, s);
  MPIR_CUDA(cudaStreamSynchronize(s));
  upload_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  on_device = true;
}

void Plan::release_device() {
  for (DeviceBuffer *d :
       {&amap, &arow, &acol, &diag_pos, &Kp, &Kj, &Ksrc, &sfirst, &srowptr, &srows, &srel,
        &slofs, &uofs, &zofs, &child_ptr, &child_list, &perm, &ea_chunks, &ea_hits, &small_list,
        &large_list, &steps, &ea_tasks, &linv_ofs_d, &gemm_probs, &solve_fronts, &swarp_list,
        &sblock_list, &gp, &gsrc, &fwd_item, &chunk_map, &own_item})
    d->release();
  on_device = false;
}

void Numeric::allocate(const Plan &P) {
  release_graph();
  const Symbolic &S = P.S;
  panel.resize(std::max<int64_t>(S.panel_elems, 1) * sizeof(float));
  if (store_prec == 2 || store_prec == 3)
    panel16.resize(std::max<int64_t>(S.panel_elems, 1) * 2);
  else
    panel16.release();
  linv64.resize(std::max<int64_t>(P.linv_elems, 1) * sizeof(double));
  linv64t.resize(std::max<int64_t>(P.linv_elems, 1) * sizeof(double));
  D.resize(std::max<int64_t>(S.n, 1) * sizeof(float));
  Dinv.resize(std::max<int64_t>(S.n, 1) * sizeof(float));
  status.resize(sizeof(FactorStatus));
  AD.resize(std::max<int64_t>(S.n, 1) * sizeof(double));
  Kval.resize(std::max<int64_t>(P.nnz_full, 1) * sizeof(double));
  Korig.resize(std::max<int64_t>(P.nnz_full, 1) * sizeof(double));
  has_scratch = false;
  ensure_scratch(P);
  valid = false;
}

void Numeric::ensure_scratch(const Plan &P) {
  if (has_scratch) return;
  release_graph();  // a recorded factorization points at the old buffers
  const Symbolic &S = P.S;
  if (!panel.bytes()) panel.resize(std::max<int64_t>(S.panel_elems, 1) * sizeof(float));
  uarena.resize(std::max<int64_t>(S.uarena_elems, 1) * sizeof(float));
  linv.resize(std::max<int64_t>(P.linv_elems, 1) * sizeof(float));
  ws.resize(std::max<int64_t>(P.ws_elems, 1) * sizeof(float));
  // Packed fronts: positions that hold no value of L are never written and
  // stay zero from here on.
  bconv.resize(std::max<int64_t>(P.bconv_elems, 1) * sizeof(float));
  pack.resize(std::max<int64_t>(P.pk_elems, 1) * sizeof(float));
  packd.resize(std::max<int64_t>(2 * P.pd_elems, 1) * sizeof(float));
  device_zero(pack.as<void>(), pack.bytes());
  device_zero(packd.as<void>(), packd.bytes());
  Axs.resize(std::max<int64_t>(S.nnz, 1) * sizeof(double));
  Ax.resize(std::max<int64_t>(S.nnz, 1) * sizeof(double));
  has_scratch = true;
}

void Numeric::trim() {
  release_graph();
  for (DeviceBuffer *b : {&uarena, &linv, &ws, &bconv, &pack, &packd, &Axs, &Ax}) b->release();
  if (panel16.bytes()) panel.release();  // the solves read the 16-bit copy
  has_scratch = false;
}

size_t Numeric::bytes_for(const Plan &P, int store_prec) {
  const Symbolic &S  = P.S;
  auto            at = [](int64_t e, size_t b) { return std::max<int64_t>(e, 1) * b; };
  return at(S.panel_elems, store_prec == 1 ? 4 : 6) + at(S.uarena_elems, 4) + at(P.linv_elems, 4) +
         2 * at(P.linv_elems, 8) + at(P.ws_elems, 4) + at(P.bconv_elems, 4) +
         at(P.pk_elems, 4) + at(2 * P.pd_elems, 4) + 2 * at(S.n, 4) + sizeof(FactorStatus) +
         at(S.n, 8) + 2 * at(S.nnz, 8) + 2 * at(P.nnz_full, 8);
}

size_t Numeric::device_bytes() const {
  size_t b = 0;
  for (const DeviceBuffer *d : {&panel, &panel16, &uarena, &linv, &linv64, &linv64t, &D, &Dinv, &status,
                                &ws, &pack, &packd, &bconv, &AD, &Axs, &Kval, &Korig, &Ax})
    b += d->bytes();
  return b;
}

size_t Plan::device_bytes() const {
  size_t b = 0;
  for (const DeviceBuffer *d :
       {&amap, &arow, &acol, &diag_pos, &Kp, &Kj, &Ksrc, &sfirst, &srowptr, &srows, &srel,
        &slofs, &uofs, &zofs, &child_ptr, &child_list, &perm, &ea_chunks, &ea_hits, &small_list,
        &large_list, &steps, &ea_tasks, &linv_ofs_d, &gemm_probs, &solve_fronts, &swarp_list,
        &sblock_list, &gp, &gsrc, &fwd_item, &chunk_map, &own_item})
    b += d->bytes();
  return b;
}

static unsigned grid_for(int64_t n, int threads) {
  return static_cast<unsigned>((n + threads - 1) / threads);
}

__global__ void k_status_reset(FactorStatus *st) {
  if (threadIdx.x == 0) *st = FactorStatus{INT_MAX, 0, 0, 0};
}

void Numeric::release_graph() {
  if (graph) cudaGraphExecDestroy(graph);
  graph     = nullptr;
  ran_plain = false;
}

cudaGraph_t Numeric::record(const Plan &P, const double *d_Ax, double eps,
                            cudaStream_t capture_stream, int64_t *launches) {
  cudaGraph_t g = nullptr;
  MPIR_CUDA(cudaStreamSynchronize(capture_stream));
  MPIR_CUDA(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
  LaunchCapture cap;
  try {
    run(P, d_Ax, eps, capture_stream);
  } catch (...) {
    cudaStreamEndCapture(capture_stream, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  MPIR_CUDA(cudaStreamEndCapture(capture_stream, &g));
  valid = false;  // recorded, not run
  if (launches) *launches = cap.count();
  return g;
}

void Numeric::run_graph(const Plan &P, const double *d_Ax, double eps, cudaStream_t s,
                        cudaStream_t capture_stream) {
  if (kernel_timer().enabled || P.S.n == 0) {  // per-class timing needs the plain launches
    run(P, d_Ax, eps, s);
    return;
  }
  const bool current = graph && graph_ax == d_Ax && graph_eps == eps && graph_mode == update_mode;
  // A factorization that may be the only one of these buffers (a new factor
  // of the serving engine, a drop-in Compute) runs its launches directly: a
  // recording pays the capture and the instantiation for a single replay.
  // The second one records the graph that every later one replays.
  if (!current && !ran_plain) {
    release_graph();
    run(P, d_Ax, eps, s);
    ran_plain = true;
    return;
  }
  if (!current) {
    release_graph();
    cudaGraph_t g = record(P, d_Ax, eps, capture_stream, &graph_launches);
    const cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    MPIR_CUDA(e);
    graph_ax   = d_Ax;
    graph_eps  = eps;
    graph_mode = update_mode;
  }
  eps_uf = eps;
  MPIR_CUDA(cudaGraphLaunch(graph, s));
  launch_add(graph_launches);
  valid = true;
}

void Numeric::run(const Plan &P, const double *d_Ax, double eps, cudaStream_t s) {
  if (!has_scratch) throw std::logic_error("factorization scratch released (ensure_scratch)");
  const Symbolic &S  = P.S;
  KernelTimer    &kt = kernel_timer();
  eps_uf             = eps;
  valid              = false;
  launch(k_status_reset, 1, 32, 0, s, status.as<FactorStatus>());
  MPIR_CUDA(cudaMemsetAsync(panel.as<void>(), 0, S.panel_elems * sizeof(float), s));
  if (S.n == 0) return;
  kt.begin(kKcScatter, s);
  launch(k_scaling, grid_for(S.n, 256), 256, 0, s, S.n, P.diag_pos.as<int64_t>(), d_Ax,
                                               eps, AD.as<double>());
  launch(k_scatter, grid_for(S.nnz, 256), 256, 0, s, 
      S.nnz, d_Ax, AD.as<double>(), P.arow.as<int32_t>(), P.acol.as<int32_t>(),
      P.amap.as<int64_t>(), Axs.as<double>(), panel.as<float>());
  launch(k_csr_values, grid_for(P.nnz_full, 256), 256, 0, s, 
      P.nnz_full, P.Ksrc.as<int64_t>(), Axs.as<double>(), d_Ax, Kval.as<double>(),
      Korig.as<double>());
  kt.end(s);
  MPIR_CHECK_LAUNCH();
  float        *pan = panel.as<float>(), *ua = uarena.as<float>();
  FactorStatus *st  = status.as<FactorStatus>();
  static const bool trsm_simt_env = [] {
    const char *e = std::getenv("MPIR_TRSM");
    return e != nullptr && std::string(e) == "simt";
  }();
  const bool trsm_tc = update_mode >= 0 && !trsm_simt_env;
  static std::atomic<bool> trsm_attr{false};
  const int     trsm_smem = kBM * (kBN + 1) * sizeof(float);
  if (!trsm_attr) {
    MPIR_CUDA(cudaFuncSetAttribute(k_step_gemm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   trsm_smem));
    trsm_attr = true;
  }
  static std::atomic<bool> diag_attr{false};
  const int     diag_smem = kDiagSmemFloats * sizeof(float);
  if (!diag_attr) {
    MPIR_CUDA(cudaFuncSetAttribute(k_diag_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   diag_smem));
    diag_attr = true;
  }
  for (const LevelPlan &L : P.levels) {
    // Children's update matrices into the fronts' panels (the update
    // matrices' own columns follow after the product that defines them).
    auto extend_add = [&](int phase) {
      const int ph = phase - 1;
      if (L.ea_count[ph] > 0) {
        kt.begin(kKcExtendAdd, s);
        launch(k_extend_add, L.ea_count[ph], 256, 0, s,
               P.ea_chunks.as<EaChunk>() + L.ea_begin[ph],
               static_cast<const EaHit *>(P.ea_hits.as<EaHit>()),
               static_cast<const EaTask *>(P.ea_tasks.as<EaTask>()), P.srel.as<int32_t>(), pan,
               ua);
        kt.end(s);
      }
    };
    extend_add(1);
    if (L.small_count > 0) {
      kt.begin(kKcSmallFront, s);
      launch(k_small_fronts<kSmallFront>, L.small_count, kSmallThreads, 0, s, 
          P.small_list.as<int32_t>() + L.small_begin, P.sfirst.as<int64_t>(),
          P.srowptr.as<int64_t>(), P.slofs.as<int64_t>(), P.uofs.as<int64_t>(),
          P.child_ptr.as<int64_t>(), P.child_list.as<int32_t>(),
          P.srel.as<int32_t>(), pan, ua, D.as<float>(), Dinv.as<float>(), st);
      kt.end(s);
    }
    const GemmProb *gp = P.gemm_probs.as<GemmProb>();
    auto gemm = [&](int32_t begin, int32_t count, int32_t tiles, int32_t rtiles,
                    int32_t convs) {
      if (count <= 0 || tiles <= 0) return;
      kt.begin(kKcUpdate, s);
      if (update_mode == 1 && convs > 0)
        launch_convert_b(gp + begin, count, convs, pack.as<float>(), packd.as<float>(),
                         bconv.as<float>(), s);
      if (update_mode < 0)
        launch(k_gemm_simt, tiles, kGemmThreads, 0, s, gp + begin, count, pan, ua,
               static_cast<const float *>(D.as<float>()), ws.as<float>());
      else
        launch_gemm_tc(update_mode, gp + begin, count, tiles, pack.as<float>(),
                       packd.as<float>(), packd.as<float>() + P.pd_elems, bconv.as<float>(),
                       pan, ua, ws.as<float>(), st, s);
      kt.end(s);
      if (rtiles > 0) {
        kt.begin(kKcReduce, s);
        launch(k_split_reduce, rtiles * kReduceSlices, 256, 0, s, gp + begin, count,
               pan, ua, static_cast<const float *>(ws.as<float>()));
        kt.end(s);
      }
    };
    for (const auto &stp : L.steps) {
      const StepDesc *dd = P.steps.as<StepDesc>() + stp.begin;
      gemm(stp.ll_begin, stp.ll_count, stp.ll_tiles, stp.ll_rtiles, stp.ll_convs);
      kt.begin(kKcDiag, s);
      launch(k_diag_block, stp.count, kDiagThreads, diag_smem, s, dd, pan, linv.as<float>(),
             D.as<float>(), Dinv.as<float>(), packd.as<float>(),
             packd.as<float>() + P.pd_elems, st);
      kt.end(s);
      if (stp.trsm_tiles > 0) {
        kt.begin(kKcTrsm, s);
        if (trsm_tc)
          launch_trsm_tc(dd, stp.count, stp.trsm_tiles, pan, linv.as<float>(), Dinv.as<float>(),
                         pack.as<float>(), st, s);
        else
          launch(k_step_gemm<true>, stp.trsm_tiles, kGemmThreads, trsm_smem, s, dd, stp.count,
                 pan, ua, linv.as<float>(), Dinv.as<float>(), pack.as<float>());
        kt.end(s);
      }
    }
    gemm(L.u_begin, L.u_count, L.u_tiles, L.u_rtiles, L.u_convs);
    extend_add(2);
    MPIR_CHECK_LAUNCH();
  }
  // Float64 inverses of the diagonal blocks for the triangular solves.
  kt.begin(kKcDiag, s);
  invert_diag_blocks(P, *this, s);
  kt.end(s);
  if (panel16.bytes() && S.panel_elems) {
    kt.begin(kKcScatter, s);
    launch(k_panel_to16, static_cast<unsigned>(std::min<int64_t>((S.panel_elems + 255) / 256, 148 * 16)),
           256, 0, s, S.panel_elems, panel.as<float>(), panel16.as<uint16_t>(),
           store_prec == 2 ? 1 : 0);
    kt.end(s);
  }
  valid = true;
}

int64_t Numeric::result(cudaStream_t s, int32_t *zero_col, bool *nonfinite) const {
  FactorStatus h;
  MPIR_CUDA(cudaMemcpyAsync(&h, status.as<void>(), sizeof h, cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
  if (zero_col) *zero_col = h.zero_pivot;
  if (nonfinite) *nonfinite = h.nonfinite != 0;
  if (h.timeout) return -5;
  if (h.zero_pivot != INT_MAX) return -1;
  return h.npos;
}

// ---------------------------------------------------------------------------
namespace {
std::atomic<int64_t>        g_launches{0};
thread_local LaunchCapture *t_capture = nullptr;
}  // namespace

int64_t launch_total() { return g_launches.load(std::memory_order_relaxed); }

void launch_add(int64_t n) {
  if (t_capture)
    t_capture->add(n);
  else
    g_launches.fetch_add(n, std::memory_order_relaxed);
}

LaunchCapture::LaunchCapture() : outer_(t_capture) { t_capture = this; }
LaunchCapture::~LaunchCapture() { t_capture = outer_; }

KernelTimer &kernel_timer() {
  static KernelTimer t;
  return t;
}

void KernelTimer::begin(int c, cudaStream_t s) {
  if (!enabled) return;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, s);
  ev.push_back(a);
  ev.push_back(b);
  cls.push_back(c);
}

void KernelTimer::end(cudaStream_t s) {
  if (!enabled) return;
  cudaEventRecord(ev.back(), s);
}

void KernelTimer::reset() {
  for (auto e : ev) cudaEventDestroy(e);
  ev.clear();
  cls.clear();
}

void KernelTimer::collect(double *ms, int64_t *count, int nclass) {
  for (int c = 0; c < nclass; c++) {
    ms[c]    = 0;
    count[c] = 0;
  }
  for (size_t i = 0; i < cls.size(); i++) {
    float t = 0;
    cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
    if (cls[i] < nclass) {
      ms[cls[i]] += t;
      count[cls[i]] += 1;
    }
  }
}

}  // namespace mpir
