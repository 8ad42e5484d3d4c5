// Triangular solves with several right-hand sides at once:
// X <- L^{-T} D^{-1} L^{-1} X for an n x NR block X (column-major, leading
// dimension n), the operation QDLDL_solve applies to one vector
// (qdldl.hpp:417-432) and LUIR_QDLDL / PrecondGmres apply once per vector.
//
// The kernels follow the single-vector ones of solve.cu level by level and
// reuse the same plan (the same fronts, work items, tickets and ready-value
// hand-over), but every CTA applies each tile of L it loads to all NR
// vectors: L moves from HBM once per application instead of NR times, and
// the dependent round trips of a chain link (waiting for a block result,
// the block product) are shared by the NR vectors.
//
//   k_fwd_small_m / k_bwd_small_m  fronts solved by one warp, column by
//                       column, each column applied to all vectors; per
//                       vector the operations and their order are those of
//                       k_fwd_small / k_bwd_small, so results are bitwise
//                       the same as NR single solves;
//   k_fwd_fronts_m      one CTA per 128-row block: row i by 4 column
//                       quarters, the NR sums of each row in registers;
//   k_bwd_chunks_m      partial sums of the off-diagonal rows per column;
//   k_bwd_fronts_m      one CTA per column block; each tile of L is staged
//                       through shared memory (coalesced loads by rows, read
//                       by columns), thread (column, vector group) sums.
// Block products use the float64 inverses of the diagonal blocks (staged as
// a packed lower triangle).  Sums inside the large-front kernels run in
// another order than in the single-vector kernels, so their results agree
// with NR single solves to rounding.
#include <atomic>
#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "engine.hpp"
#include "solve.hpp"
#include "solve_dev.cuh"

namespace mpir {

namespace {

constexpr int kTriM      = kNB * (kNB + 1) / 2;  // packed lower triangle of Linv
constexpr int kSmallWarpsM = 2;                  // warps per CTA, small fronts
constexpr int kLsPitch   = kNB + 1;              // staged tile row pitch (floats)

// Copies of each block result in the ready buffer (see solve_dev.cuh).
constexpr int kMultiCopies = 4;

// Stage the lower triangle of the row-major inverse Lt (Lt[i * kNB + j] =
// Linv[i][j]) packed by rows: (i, j <= i) at i (i + 1) / 2 + j.
__device__ __forceinline__ void stage_tri_m(const double *Lt, double *Ls, int nb) {
  const int tid = threadIdx.x, j = tid % kNB, q = tid / kNB;
  for (int ii = 0; ii < kNB / 4; ii++) {
    const int i = q * (kNB / 4) + ii;
    if (i >= j && i < nb) cp_async8(Ls + i * (i + 1) / 2 + j, Lt + i * kNB + j);
  }
}

// Waits for the K entries p[k * stride] (k < K) of block results and stores
// them to dst[k * dstride] (zeros for an inactive lane).  The entries are
// polled in groups of at most 8 loads in flight.
template <int K>
__device__ __forceinline__ void wait_many(const double *p, int64_t stride, bool active,
                                          double *dst, int dstride, int32_t *err, long polls) {
  constexpr int G = K < 8 ? K : 8;
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += G) {
    unsigned need = 0;
#pragma unroll
    for (int k = 0; k < G; k++) {
      if (active) need |= 1u << k;
      else dst[(k0 + k) * dstride] = 0.0;
    }
    for (long it = 0; need != 0 && it < polls; it++) {
      unsigned long long raw[G];
#pragma unroll
      for (int k = 0; k < G; k++)
        raw[k] = (need >> k & 1u) ? ld_relaxed_u64(p + (k0 + k) * stride) : 0ull;
#pragma unroll
      for (int k = 0; k < G; k++)
        if ((need >> k & 1u) && raw[k] != kPending) {
          dst[(k0 + k) * dstride] = __longlong_as_double(static_cast<long long>(raw[k]));
          need &= ~(1u << k);
        }
      if ((it & 63) == 63) {
        if (*reinterpret_cast<volatile int32_t *>(err) != 0) return;
        __nanosleep(32);
      }
    }
    if (need != 0) {
      atomicExch(err, 1);
      return;
    }
  }
}

__global__ void k_mark_pending_m(int64_t count, double *ready) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < count) reinterpret_cast<unsigned long long *>(ready)[i] = kPending;
}

// X[:, k] .*= Dinv for every vector k < nr.
__global__ void k_dscale_m(int64_t n, int nr, const float *Dinv, double *X) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * nr) return;
  X[i] *= static_cast<double>(Dinv[i % n]);
}

// ---------------------------------------------------------------------------
// Fronts solved by one warp (w <= 32, h <= 256), forward.  z[k][i] is front
// row i of vector k; per vector exactly the operations of k_fwd_small.
template <int NR, class T>
__global__ void __launch_bounds__(32 * kSmallWarpsM)
    k_fwd_small_m(const int32_t *list, int count, const int64_t *sfirst,
                  const int64_t *srowptr, const int64_t *slofs, const int64_t *child_ptr,
                  const int32_t *child_list, const int32_t *srel, const int64_t *zofs,
                  const T *panel, double *x, int64_t n, double *zbuf, int64_t zld) {
  extern __shared__ __align__(16) double zsm[];  // [warps][NR][kWarpSolveH]
  constexpr int H    = kWarpSolveH;
  const int     warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int     idx  = blockIdx.x * kSmallWarpsM + warp;
  if (idx >= count) return;
  const int     J = list[idx];
  const int64_t f = sfirst[J];
  const int     w = static_cast<int>(sfirst[J + 1] - f);
  const int     h = static_cast<int>(srowptr[J + 1] - srowptr[J]);
  double       *z = zsm + static_cast<int64_t>(warp) * NR * H;
  for (int k = 0; k < NR; k++)
    for (int i = lane; i < h; i += 32) z[k * H + i] = i < w ? x[k * n + f + i] : 0.0;
  __syncwarp();
  for (int64_t c = child_ptr[J]; c < child_ptr[J + 1]; c++) {
    const int      C  = child_list[c];
    const int      wc = static_cast<int>(sfirst[C + 1] - sfirst[C]);
    const int      rc = static_cast<int>(srowptr[C + 1] - srowptr[C]) - wc;
    const int32_t *rl = srel + srowptr[C] + wc;
    const int64_t  zc = zofs[C] + wc;
    for (int k = 0; k < NR; k++)
      for (int a = lane; a < rc; a += 32) z[k * H + rl[a]] += zbuf[k * zld + zc + a];
    __syncwarp();
  }
  const T      *P  = panel + slofs[J];
  constexpr int RT = H / 32;
  float         cur[4][RT], nxt[4][RT];
  auto          load4 = [&](float (*buf)[RT], int k0) {
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int t = 0; t < RT; t++) {
        const int k = k0 + u, i = lane + 32 * t;
        buf[u][t]   = (k < w && i > k && i < h) ? to_f(P[i + (int64_t)k * h]) : 0.0f;
      }
  };
  load4(cur, 0);
  for (int k0 = 0; k0 < w; k0 += 4) {
    if (k0 + 4 < w) load4(nxt, k0 + 4);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int col = k0 + u;
      if (col >= w) break;
      for (int k = 0; k < NR; k++) {
        double      *zk = z + k * H;
        const double zc = zk[col];
#pragma unroll
        for (int t = 0; t < RT; t++) {
          const int i = lane + 32 * t;
          if (i > col && i < h) zk[i] -= static_cast<double>(cur[u][t]) * zc;
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int t = 0; t < RT; t++) cur[u][t] = nxt[u][t];
  }
  const int64_t zo = zofs[J];
  for (int k = 0; k < NR; k++)
    for (int i = lane; i < h; i += 32) {
      if (i < w) x[k * n + f + i] = z[k * H + i];
      zbuf[k * zld + zo + i] = z[k * H + i];
    }
}

// Backward counterpart of k_fwd_small_m (per vector the operations of
// k_bwd_small).
template <int NR, class T>
__global__ void __launch_bounds__(32 * kSmallWarpsM)
    k_bwd_small_m(const int32_t *list, int count, const int64_t *sfirst,
                  const int64_t *srowptr, const int32_t *srows, const int64_t *slofs,
                  const T *panel, double *x, int64_t n) {
  extern __shared__ __align__(16) double zsm[];
  constexpr int H    = kWarpSolveH;
  const int     warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int     idx  = blockIdx.x * kSmallWarpsM + warp;
  if (idx >= count) return;
  const int      J  = list[idx];
  const int64_t  f  = sfirst[J];
  const int      w  = static_cast<int>(sfirst[J + 1] - f);
  const int      h  = static_cast<int>(srowptr[J + 1] - srowptr[J]);
  const int32_t *rw = srows + srowptr[J];
  double        *z  = zsm + static_cast<int64_t>(warp) * NR * H;
  for (int k = 0; k < NR; k++)
    for (int i = lane; i < h; i += 32) z[k * H + i] = x[k * n + (i < w ? f + i : rw[i])];
  __syncwarp();
  const T      *P  = panel + slofs[J];
  constexpr int RT = H / 32;
  float         cur[4][RT], nxt[4][RT];
  auto          load4 = [&](float (*buf)[RT], int k0) {
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int t = 0; t < RT; t++) {
        const int k = k0 - u, i = lane + 32 * t;
        buf[u][t]   = (k >= 0 && i > k && i < h) ? to_f(P[i + (int64_t)k * h]) : 0.0f;
      }
  };
  load4(cur, w - 1);
  for (int k0 = w - 1; k0 >= 0; k0 -= 4) {
    if (k0 - 4 >= 0) load4(nxt, k0 - 4);
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int col = k0 - u;
      if (col < 0) break;
      for (int k = 0; k < NR; k++) {
        double *zk = z + k * H;
        double  s  = 0.0;
#pragma unroll
        for (int t = 0; t < RT; t++) {
          const int i = lane + 32 * t;
          if (i > col && i < h) s += static_cast<double>(cur[u][t]) * zk[i];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) zk[col] -= s;
      }
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int t = 0; t < RT; t++) cur[u][t] = nxt[u][t];
  }
  for (int k = 0; k < NR; k++)
    for (int i = lane; i < w; i += 32) x[k * n + f + i] = z[k * H + i];
}

// ---------------------------------------------------------------------------
// Forward, large fronts: one CTA per 128-row block R of a front (tickets as
// in k_fwd_fronts).  Thread (qq, rr) = (tid / 128, tid % 128) takes row rr of
// the block and columns 32 qq .. 32 qq + 31 of each tile; each lane waits
// for its entry of y_b in all NR vectors, the warp shares them through
// shared memory, and the row's NR sums stay in registers.
template <int NR>
constexpr int fwd_m_smem_doubles() {
  return kTriM + 2 * NR * kNB + NR * 512;
}

template <int NR, class T>
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_fwd_fronts_m(const SolveItem *items, const T *panel, const double *linv64t,
                   const int64_t *gp, const int64_t *gsrc, double *x, double *zbuf,
                   int64_t zld, int32_t *tickets, double *ready, int32_t *err) {
  extern __shared__ __align__(16) double sm[];
  double *tri = sm;                // packed lower Linv_R
  double *zs  = tri + kTriM;       // [NR][kNB] right-hand side, then z
  double *yb  = zs + NR * kNB;     // [NR][kNB] block result
  double *S   = yb + NR * kNB;     // [16][NR][32] tile values, then [4][NR][kNB]
  __shared__ SolveFront sF;
  __shared__ int        sR, sItem;
  __shared__ long       sPolls;
  __shared__ bool       sPublish;
  if (threadIdx.x == 0) {
    const int it = atomicAdd(tickets, 1);
    sItem        = it;
    sF           = items[it].f;
    sR           = items[it].r;
    const volatile SolveCtl *c = reinterpret_cast<const volatile SolveCtl *>(err);
    sPolls       = poll_limit(c->poll_log2);
    sPublish     = c->withhold != it + 1;
  }
  __syncthreads();
  const int         item  = sItem;
  const SolveFront &F     = sF;
  const int         R     = sR;
  const long        polls = sPolls;
  const int         tid = threadIdx.x, rr = tid % kNB, qq = tid / kNB;
  const int         warp = tid / 32, lane = tid % 32;
  const int64_t     h = F.h, n = F.n;
  const int         w = F.w;
  const int64_t     r = static_cast<int64_t>(R) * kNB + rr;
  const T          *P = panel + F.panel;
  if (R < F.nb) stage_tri_m(linv64t + F.linv + static_cast<int64_t>(R) * kNB * kNB, tri,
                            min(kNB, w - R * kNB));
  // Right-hand side rows: x (rows < w) plus the children's update vectors in
  // child order; thread (qq, rr) fills vectors qq, qq + 4, ...
  for (int k = qq; k < NR; k += 4) {
    double zr = 0.0;
    if (r < h) {
      zr = r < w ? x[k * n + F.col0 + r] : 0.0;
      for (int64_t e = gp[F.gptr + r]; e < gp[F.gptr + r + 1]; e++) zr += zbuf[k * zld + gsrc[e]];
    }
    zs[k * kNB + rr] = zr;
  }
  const int     copy  = (item * 16 + warp) % kMultiCopies;
  const double *yr    = ready + static_cast<int64_t>(copy) * NR * n + F.col0;
  const int     tiles = min(R, F.nb);
  double        acc[NR];
#pragma unroll
  for (int k = 0; k < NR; k++) acc[k] = 0.0;
  // Each tile's L values are loaded before the wait for its block result,
  // so the loads are in flight while the lane polls.
  float   lv[32];
  double *yw = S + warp * NR * 32;  // [NR][32]
  for (int b = 0; b < tiles; b++) {
    const int c0 = b * kNB + qq * 32;
#pragma unroll
    for (int k = 0; k < 32; k++)
      lv[k] = (r < h && c0 + k < w) ? to_f(__ldg(P + r + static_cast<int64_t>(c0 + k) * h)) : 0.0f;
    wait_many<NR>(yr + c0 + lane, n, c0 + lane < w, yw + lane, 32, err, polls);
    __syncwarp();
#pragma unroll
    for (int kk = 0; kk < 32; kk++) {
      const double l = static_cast<double>(lv[kk]);
#pragma unroll
      for (int k = 0; k < NR; k++) acc[k] += l * yw[k * 32 + kk];
    }
    __syncwarp();
  }
  __syncthreads();  // every warp is done with its tile values: S becomes part
  double *part = S;
#pragma unroll
  for (int k = 0; k < NR; k++) part[(qq * NR + k) * kNB + rr] = acc[k];
  __syncthreads();
  for (int k = qq; k < NR; k += 4)
    if (r < h) {
      const double *p = part + k * kNB + rr;
      zs[k * kNB + rr] -= (p[0] + p[NR * kNB]) + (p[2 * NR * kNB] + p[3 * NR * kNB]);
    }
  if (R < F.nb) {
    const int nbk = min(kNB, w - R * kNB);
    cp_async_wait_all();
    __syncthreads();  // z complete, Linv_R staged
    const int i = rr;
    for (int k = qq; k < NR; k += 4) {
      double y = 0.0;
      if (i < nbk) {
        const double *row = tri + i * (i + 1) / 2;
        const double *zk  = zs + k * kNB;
        double        a0 = 0.0, a1 = 0.0;
        int           j = 0;
        for (; j + 1 <= i; j += 2) {
          a0 += row[j] * zk[j];
          a1 += row[j + 1] * zk[j + 1];
        }
        if (j <= i) a0 += row[j] * zk[j];
        y = a0 + a1;
      }
      yb[k * kNB + i] = y;
      if (i < nbk && sPublish) {
        const int64_t gj = F.col0 + static_cast<int64_t>(R) * kNB + i;
#pragma unroll
        for (int c = 0; c < kMultiCopies; c++)
          st_relaxed_f64(ready + (static_cast<int64_t>(c) * NR + k) * n + gj, y);
        x[k * n + gj] = y;
      }
    }
    if ((R + 1) * kNB > w && h > w) {
      // Rows of this block at or past w: their product with the block.
      __syncthreads();
      if (r >= w && r < h) {
        double a[NR / 4 > 0 ? NR / 4 : 1];
        constexpr int KG = NR / 4 > 0 ? NR / 4 : 1;
#pragma unroll
        for (int t = 0; t < KG; t++) a[t] = 0.0;
        for (int k2 = 0; k2 < nbk; k2++) {
          const double l = static_cast<double>(to_f(P[r + static_cast<int64_t>(R * kNB + k2) * h]));
#pragma unroll
          for (int t = 0; t < KG; t++) {
            const int k = qq + 4 * t;
            if (k < NR) a[t] += l * yb[k * kNB + k2];
          }
        }
#pragma unroll
        for (int t = 0; t < KG; t++) {
          const int k = qq + 4 * t;
          if (k < NR) zs[k * kNB + rr] -= a[t];
        }
      }
    }
  }
  if (r >= w && r < h)
    for (int k = qq; k < NR; k += 4) zbuf[k * zld + F.zofs + r] = zs[k * kNB + rr];
}

// ---------------------------------------------------------------------------
// Backward, off-diagonal rows: CTA c takes rows w + 128 c .. of one front and
// writes t_col = sum_r L_{r,col} x_r of every column for all NR vectors (warp
// per column, rows over the lanes; per vector the sums of k_bwd_chunks).
template <int NR, class T>
__global__ void __launch_bounds__(kSolveThreads)
    k_bwd_chunks_m(const SolveFront *fr, const int32_t *fmap, const T *panel,
                   const int32_t *srows, const double *x, double *part, int64_t pld) {
  __shared__ double zr[NR][kNB];
  const SolveFront  F = fr[fmap[blockIdx.x]];
  const int         c = blockIdx.x - F.chunk0;
  const int         tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int64_t     h = F.h, w = F.w, n = F.n;
  const int64_t     r0 = w + static_cast<int64_t>(c) * kNB;
  const int         nr = static_cast<int>(h - r0 < kNB ? h - r0 : kNB);
  for (int e = tid; e < NR * kNB; e += kSolveThreads) {
    const int k = e / kNB, i = e % kNB;
    zr[k][i] = i < nr ? x[k * n + srows[F.rows + r0 + i]] : 0.0;
  }
  __syncthreads();
  const T      *P  = panel + F.panel + r0;
  constexpr int kWarps = kSolveThreads / 32;
  for (int64_t col = warp; col < w; col += kWarps) {
    const T     *cp = P + col * h;
    double       l[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int rr = lane + 32 * i;
      l[i]         = rr < nr ? static_cast<double>(to_f(__ldg(cp + rr))) : 0.0;
    }
#pragma unroll
    for (int k = 0; k < NR; k++) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < 4; i++)
        if (lane + 32 * i < nr) s += l[i] * zr[k][lane + 32 * i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) part[k * pld + F.part + static_cast<int64_t>(c) * w + col] = s;
    }
  }
}

// Backward, column blocks: one CTA per column block b (tickets as in
// k_bwd_fronts).  Thread (c, g) = (tid % 128, tid / 128) takes column c of
// the block and vectors g KG .. g KG + KG - 1.  Each tile of L (row block R
// below the block, last first) is loaded into registers by rows (coalesced)
// while the previous tile is applied, then stored to shared memory and read
// by columns; the CTA waits for x_R of all vectors before applying tile R.
template <int NR>
constexpr int bwd_m_smem_doubles() {
  return kTriM + (kNB * kLsPitch + 1) / 2 + 2 * NR * kNB;
}

template <int NR, class T>
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_bwd_fronts_m(const SolveItem *items, const T *panel, const double *linv64t,
                   double *x, const double *part, int64_t pld, int32_t *tickets,
                   double *ready, int32_t *err) {
  constexpr int KG = NR / 4;
  extern __shared__ __align__(16) double sm[];
  double *tri = sm;                                             // packed lower Linv_b
  float  *Ls  = reinterpret_cast<float *>(tri + kTriM);         // [kNB][kLsPitch]
  double *xs  = tri + kTriM + (kNB * kLsPitch + 1) / 2;         // [kNB][NR]
  double *v   = xs + NR * kNB;                                  // [NR][kNB]
  __shared__ SolveFront sF;
  __shared__ int        sB, sItem;
  __shared__ long       sPolls;
  if (threadIdx.x == 0) {
    const int it = atomicAdd(tickets, 1);
    sItem        = it;
    sF           = items[it].f;
    sB           = items[it].r;
    sPolls       = poll_limit(reinterpret_cast<const volatile SolveCtl *>(err)->poll_log2);
  }
  __syncthreads();
  const int         item  = sItem;
  const SolveFront &F     = sF;
  const int         b     = sB;
  const long        polls = sPolls;
  const int         tid = threadIdx.x, c = tid % kNB, g = tid / kNB;
  const int64_t     h = F.h, n = F.n;
  const int         w = F.w;
  const int         nbk = min(kNB, w - b * kNB);
  stage_tri_m(linv64t + F.linv + static_cast<int64_t>(b) * kNB * kNB, tri, nbk);
  // This block's right-hand side and the chunk partials of its columns.
  double rhs[KG], acc[KG];
#pragma unroll
  for (int t = 0; t < KG; t++) {
    const int k = g * KG + t;
    rhs[t]      = c < nbk ? x[k * n + F.col0 + b * kNB + c] : 0.0;
    double s    = 0.0;
    if (c < nbk)
      for (int ch = 0; ch < F.chunks; ch++)
        s += part[k * pld + F.part + static_cast<int64_t>(ch) * w + b * kNB + c];
    acc[t] = s;
  }
  const T     *P    = panel + F.panel;
  const int    copy = (item * 16 + g) % kMultiCopies;
  // Tile R: thread (rr, cg) = (tid % 128, tid / 128) loads row rr, columns
  // 32 cg .. 32 cg + 31 of the block.
  float     lr[32];
  const int trr = tid % kNB, tcg = tid / kNB;
  auto      load_tile = [&](int R) {
    const int64_t rb   = static_cast<int64_t>(R) * kNB;
    const int     rows = min(kNB, w - R * kNB);
#pragma unroll
    for (int k = 0; k < 32; k++) {
      const int cc = tcg * 32 + k;
      lr[k] = (trr < rows && cc < nbk)
                  ? to_f(__ldg(P + rb + trr + static_cast<int64_t>(b * kNB + cc) * h))
                  : 0.0f;
    }
  };
  if (F.nb - 1 > b) load_tile(F.nb - 1);
  for (int R = F.nb - 1; R > b; R--) {
    const int rows = min(kNB, w - R * kNB);
    // x_R of the KG vectors of this thread's group, row trr.
    wait_many<KG>(ready + (static_cast<int64_t>(copy) * NR + tcg * KG) * n + F.col0 +
                      static_cast<int64_t>(R) * kNB + trr,
                  n, trr < rows, xs + trr * NR + tcg * KG, 1, err, polls);
#pragma unroll
    for (int k = 0; k < 32; k++) Ls[trr * kLsPitch + tcg * 32 + k] = lr[k];
    __syncthreads();
    if (R - 1 > b) load_tile(R - 1);
    for (int rr = 0; rr < rows; rr++) {
      const double l = static_cast<double>(Ls[rr * kLsPitch + c]);
#pragma unroll
      for (int t = 0; t < KG; t++) acc[t] += l * xs[rr * NR + g * KG + t];
    }
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < KG; t++) v[(g * KG + t) * kNB + c] = c < nbk ? rhs[t] - acc[t] : 0.0;
  cp_async_wait_all();
  __syncthreads();
  // x_b = Linv_b^T v: x_c = sum_{i >= c} Linv[i][c] v_i.
  const int i0 = c & ~31;
#pragma unroll
  for (int t = 0; t < KG; t++) {
    const int     k  = g * KG + t;
    const double *vk = v + k * kNB;
    double        s  = 0.0;
    for (int i = i0; i < nbk; i++)
      if (i >= c) s += tri[i * (i + 1) / 2 + c] * vk[i];
    if (c < nbk) {
      const int64_t j = F.col0 + static_cast<int64_t>(b) * kNB + c;
#pragma unroll
      for (int cp = 0; cp < kMultiCopies; cp++)
        st_relaxed_f64(ready + (static_cast<int64_t>(cp) * NR + k) * n + j, s);
      x[k * n + j] = s;
    }
  }
}

template <int NR, class T>
void set_smem_attrs() {
  static std::atomic<bool> done{false};  // idempotent; set once per process
  if (done) return;
  MPIR_CUDA(cudaFuncSetAttribute(k_fwd_fronts_m<NR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(fwd_m_smem_doubles<NR>() * sizeof(double))));
  MPIR_CUDA(cudaFuncSetAttribute(k_bwd_fronts_m<NR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(bwd_m_smem_doubles<NR>() * sizeof(double))));
  const int small = static_cast<int>(kSmallWarpsM * NR * kWarpSolveH * sizeof(double));
  MPIR_CUDA(cudaFuncSetAttribute(k_fwd_small_m<NR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 small));
  MPIR_CUDA(cudaFuncSetAttribute(k_bwd_small_m<NR, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 small));
  done = true;
}

template <int NR, class T>
void solve_multi_nr(const Plan &P, const Numeric &F, const T *pan, double *X,
                    MultiSolveWorkspace &ws, cudaStream_t s, int phases) {
  const Symbolic &S  = P.S;
  KernelTimer    &kt = kernel_timer();
  set_smem_attrs<NR, T>();
  const int64_t     n     = S.n;
  const double     *lvt   = F.linv64t.as<double>();
  double           *zbuf  = ws.zbuf.as<double>();
  const int64_t     zld   = std::max<int64_t>(S.z_elems, 1);
  const int64_t     pld   = std::max<int64_t>(P.spart_elems, 1);
  int32_t          *sync  = ws.sync.as<int32_t>();
  double           *ready = ws.ready.as<double>();
  int32_t          *err   = ws.err.as<int32_t>();
  const SolveFront *sf    = P.solve_fronts.as<SolveFront>();
  const bool        block = P.nblock_fronts > 0;
  const int64_t     nready = static_cast<int64_t>(kMultiCopies) * NR * n;
  const unsigned    nmark  = static_cast<unsigned>((nready + 255) / 256);
  const int         nl     = static_cast<int>(P.levels.size());
  const size_t      small_smem = kSmallWarpsM * NR * kWarpSolveH * sizeof(double);
  if (block) MPIR_CUDA(cudaMemsetAsync(sync, 0, P.sync_elems * sizeof(int32_t), s));
  if (block && (phases & kForward)) launch(k_mark_pending_m, nmark, 256, 0, s, nready, ready);
  kt.begin(kKcSolveFwd, s);
  for (int t = 0; t < nl && (phases & kForward); t++) {
    const LevelPlan &L    = P.levels[t];
    const bool       both = L.sw_count > 0 && L.sf_count > 0;
    cudaStream_t     ss   = both ? ws.side.fork(s) : s;  // warp fronts beside block fronts
    if (L.sw_count > 0)
      launch(k_fwd_small_m<NR, T>, (L.sw_count + kSmallWarpsM - 1) / kSmallWarpsM, 32 * kSmallWarpsM,
             small_smem, ss, P.swarp_list.as<int32_t>() + L.sw_begin, L.sw_count,
             P.sfirst.as<int64_t>(), P.srowptr.as<int64_t>(), P.slofs.as<int64_t>(),
             P.child_ptr.as<int64_t>(), P.child_list.as<int32_t>(), P.srel.as<int32_t>(),
             P.zofs.as<int64_t>(), pan, X, n, zbuf, zld);
    if (L.sf_count > 0)
      launch(k_fwd_fronts_m<NR, T>, L.fwd_items, kSolveThreads,
             fwd_m_smem_doubles<NR>() * sizeof(double), s,
             P.fwd_item.as<SolveItem>() + L.fwd_map0, pan, lvt, P.gp.as<int64_t>(),
             P.gsrc.as<int64_t>(), X, zbuf, zld, sync + 2 * t, ready, err);
    if (both) ws.side.join(s);
  }
  if (phases & kDiagonal)
    launch(k_dscale_m, static_cast<unsigned>((n * NR + 255) / 256), 256, 0, s, n, NR,
           F.Dinv.as<float>(), X);
  kt.end(s);
  if (!(phases & kBackward)) return;
  MPIR_CHECK_LAUNCH();
  kt.begin(kKcSolveBwd, s);
  if (block) launch(k_mark_pending_m, nmark, 256, 0, s, nready, ready);
  for (int t = nl - 1; t >= 0; t--) {
    const LevelPlan &L    = P.levels[t];
    const bool       both = L.sw_count > 0 && L.sf_count > 0;
    cudaStream_t     ss   = both ? ws.side.fork(s) : s;
    if (L.sw_count > 0)
      launch(k_bwd_small_m<NR, T>, (L.sw_count + kSmallWarpsM - 1) / kSmallWarpsM, 32 * kSmallWarpsM,
             small_smem, ss, P.swarp_list.as<int32_t>() + L.sw_begin, L.sw_count,
             P.sfirst.as<int64_t>(), P.srowptr.as<int64_t>(), P.srows.as<int32_t>(),
             P.slofs.as<int64_t>(), pan, X, n);
    if (L.sf_count > 0) {
      if (L.bwd_chunk_items > 0)
        launch(k_bwd_chunks_m<NR, T>, L.bwd_chunk_items, kSolveThreads, 0, s, sf + L.sf_begin,
               P.chunk_map.as<int32_t>() + L.chunk_map0, pan, P.srows.as<int32_t>(),
               static_cast<const double *>(X), ws.part.as<double>(), pld);
      launch(k_bwd_fronts_m<NR, T>, L.bwd_owner_items, kSolveThreads,
             bwd_m_smem_doubles<NR>() * sizeof(double), s,
             P.own_item.as<SolveItem>() + L.own_map0, pan, lvt, X,
             static_cast<const double *>(ws.part.as<double>()), pld, sync + 2 * t + 1, ready,
             err);
    }
    if (both) ws.side.join(s);
  }
  kt.end(s);
  MPIR_CHECK_LAUNCH();
}

}  // namespace

int multi_width(int nrhs) {
  if (nrhs <= 4) return 4;
  if (nrhs <= 8) return 8;
  return 16;
}

void MultiSolveWorkspace::allocate(const Plan &P, int width) {
  const Symbolic &S = P.S;
  nr = width;
  graph.reset();
  xbuf.resize(std::max<int64_t>(S.n, 1) * width * sizeof(double));
  device_zero(xbuf.as<void>(), xbuf.bytes());
  zbuf.resize(std::max<int64_t>(S.z_elems, 1) * width * sizeof(double));
  part.resize(std::max<int64_t>(P.spart_elems, 1) * width * sizeof(double));
  sync.resize(std::max<int64_t>(P.sync_elems, 1) * sizeof(int32_t));
  ready.resize(std::max<int64_t>(static_cast<int64_t>(kMultiCopies) * width * S.n, 1) *
               sizeof(double));
  err.resize(sizeof(SolveCtl));
  device_zero(err.as<void>(), sizeof(SolveCtl));
}

size_t MultiSolveWorkspace::bytes_for(const Plan &P, int width) {
  const Symbolic &S = P.S;
  return (std::max<int64_t>(S.z_elems, 1) + std::max<int64_t>(P.spart_elems, 1) +
          static_cast<int64_t>(kMultiCopies + 1) * S.n) *
             width * sizeof(double) +
         std::max<int64_t>(P.sync_elems, 1) * sizeof(int32_t) + sizeof(SolveCtl);
}

void ldlt_solve_multi(const Plan &P, const Numeric &F, double *X, int width,
                      MultiSolveWorkspace &ws, cudaStream_t s, int phases) {
  if (P.S.n == 0) return;
  if (ws.nr != width) throw std::logic_error("multi-vector workspace of another width");
  if (width != 4 && width != 8 && width != 16)
    throw std::invalid_argument("multi-vector solve width must be 4, 8 or 16");
  auto run = [&](auto *pan) {
    using T = std::remove_const_t<std::remove_pointer_t<decltype(pan)>>;
    if (width == 4) solve_multi_nr<4, T>(P, F, pan, X, ws, s, phases);
    if (width == 8) solve_multi_nr<8, T>(P, F, pan, X, ws, s, phases);
    if (width == 16) solve_multi_nr<16, T>(P, F, pan, X, ws, s, phases);
  };
  switch (F.solve_prec()) {
    case 2: run(F.panel16.as<const __nv_bfloat16>()); break;
    case 3: run(F.panel16.as<const __half>()); break;
    default: run(F.panel.as<const float>());
  }
}

void ldlt_solve_multi_graph(const Plan &P, const Numeric &F, double *X, int width,
                            MultiSolveWorkspace &ws, cudaStream_t s,
                            cudaStream_t capture_stream) {
  const int64_t n = P.S.n;
  if (n == 0) return;
  if (kernel_timer().enabled) {
    ldlt_solve_multi(P, F, X, width, ws, s);
    return;
  }
  if (!ws.graph.g) {
    cudaGraph_t g = nullptr;
    MPIR_CUDA(cudaStreamSynchronize(capture_stream));
    MPIR_CUDA(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
    try {
      LaunchCapture cap;
      ldlt_solve_multi(P, F, ws.xbuf.as<double>(), width, ws, capture_stream);
      ws.graph_launches = cap.count();
    } catch (...) {
      cudaStreamEndCapture(capture_stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    MPIR_CUDA(cudaStreamEndCapture(capture_stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&ws.graph.g, g, 0);
    cudaGraphDestroy(g);
    MPIR_CUDA(e);
  }
  const size_t bytes = static_cast<size_t>(n) * width * sizeof(double);
  MPIR_CUDA(cudaMemcpyAsync(ws.xbuf.as<void>(), X, bytes, cudaMemcpyDeviceToDevice, s));
  MPIR_CUDA(cudaGraphLaunch(ws.graph.g, s));
  launch_add(ws.graph_launches);
  MPIR_CUDA(cudaMemcpyAsync(X, ws.xbuf.as<void>(), bytes, cudaMemcpyDeviceToDevice, s));
}

}  // namespace mpir
