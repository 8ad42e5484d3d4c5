// Triangular solves with the supernodal LDL^T factor on the GPU.
//
// Computes x <- L^{-T} D^{-1} L^{-1} x, the preconditioner application that
// QDLDL_solve performs column by column (qdldl.hpp:362-432), level by level
// over the supernodal elimination tree:
//   forward   each front takes its own right-hand side entries plus its
//             children's update vectors, solves with its unit-lower diagonal
//             block and leaves L_{R,J} x_J (negated, accumulated) as its own
//             update vector for its parent;
//   diagonal  x <- Dinv .* x;
//   backward  each front gathers the finished x of its row set R_J and solves
//             with L_J^T, last column block first.
// Small fronts use one warp each; large fronts run column-block steps batched
// over the level, reusing the inverses of the diagonal blocks kept by the
// factorization so the diagonal solves become small dense products.  Vectors
// are float64, the factor float32 (widened on load), as QDLDL_solve with
// FACTPREC = float and XPREC = double.  Reductions have a fixed order, so
// results do not depend on scheduling.
#include <atomic>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.hpp"
#include "solve.hpp"
#include "solve_dev.cuh"

namespace mpir {

constexpr int kWarpsPerCta = 4;
constexpr int kSmallH      = kWarpSolveH;

// ---------------------------------------------------------------------------
// Products with the float64 inverse of one diagonal block (128 x 128), 512
// threads.  Each thread first copies the inverse entries it will use into
// shared memory with cp.async (asynchronous, no registers held): a CTA does
// this when it starts, so the product at the end of its wait chain reads
// shared memory only, and each thread reads only what it copied itself.
constexpr int kTri = kNB * (kNB + 1) / 2;

// Thread layout of the forward block product: lane l of warp v takes row
// i = 8 v + l / 4 of the block and its slice q = l % 4; the four slices of i
// sit in four neighbouring lanes and are added with two shuffles,
// (s0 + s1) + (s2 + s3), with no CTA barrier.
__device__ __forceinline__ int blk_i() { return (threadIdx.x / 32) * 8 + (threadIdx.x % 32) / 4; }
__device__ __forceinline__ int blk_q() { return threadIdx.x % 4; }
__device__ __forceinline__ int pad(int j) { return (j / 32) * 33 + j % 32; }
__device__ __forceinline__ double quad_sum(double s) {
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  return s;
}

// Forward copy of Linv, by rows in 64-byte segments: row i = 8 a + r holds
// its first 8 (a + 1) entries (those right of the diagonal are zero), and a
// row of an odd group a one segment of padding more, so the 8 rows a warp
// reads start alternately in the two halves of the banks (a warp's 16-byte
// loads then take the minimum of four shared-memory wavefronts).
constexpr int kFwdTri = 64 * (16 * 17 / 2 + 8);
__device__ __forceinline__ int fwd_row_start(int i) {
  const int a = i / 8, r = i % 8;
  return 64 * (a * (a + 1) / 2 + a / 2) + r * 8 * (a + 1 + (a & 1));
}

// Thread (i, q) copies the pairs j = 8 m + 2 q, 8 m + 2 q + 1 (m <= i / 8) of
// row i from the row-major inverse Lt (Lt[i * kNB + j] = Linv[i][j]).
__device__ __forceinline__ void stage_lower(const double *Lt, double *Ls) {
  const int     i = blk_i(), q = blk_q(), a = i / 8;
  double       *d = Ls + fwd_row_start(i) + 2 * q;
  const double *s = Lt + i * kNB + 2 * q;
  for (int m = 0; m <= a; m++) cp_async16(d + 8 * m, s + 8 * m);
}

// y_i = (Linv z)_i from the staged copy, in all four lanes of row i; z holds
// 128 entries (16-byte aligned).  Warp v (rows 8 v .. 8 v + 7) takes the
// segments m <= v: 4 (v + 1) loads of Linv and of z per warp in all.
__device__ __forceinline__ double block_lower_apply(const double *Ls, const double *z) {
  const int     i = blk_i(), q = blk_q(), a = i / 8;
  const double *row = Ls + fwd_row_start(i) + 2 * q;
  const double *zq  = z + 2 * q;
  cp_async_wait_all();
  double a0 = 0.0, a1 = 0.0;
#pragma unroll 4
  for (int m = 0; m <= a; m++) {
    const double2 l = *reinterpret_cast<const double2 *>(row + 8 * m);
    const double2 v = *reinterpret_cast<const double2 *>(zq + 8 * m);
    a0 += l.x * v.x;
    a1 += l.y * v.y;
  }
  return quad_sum(a0 + a1);
}

// Stage the row-major copy Lt (Lt[i * kNB + j] = Linv[i][j]) for x = Linv^T v:
// thread (q, j) = (tid / 128, tid % 128) copies rows i >= j of slice q (a
// warp reads 32 consecutive entries of a row).
__device__ __forceinline__ void stage_upper(const double *Lt, double *Ls, int nb) {
  const int tid = threadIdx.x, j = tid % kNB, q = tid / kNB;
  for (int ii = 0; ii < kNB / 4; ii++) {
    const int i = q * (kNB / 4) + ii;
    if (i >= j && i < nb) cp_async8(Ls + i * (i + 1) / 2 + j, Lt + i * kNB + j);
  }
}

// x_j = (Linv^T v)_j from the staged copy for thread (q, j): the four slices
// are added in order through part (one CTA barrier).
__device__ __forceinline__ double block_upper_apply(const double *Ls, const double *v, int nb,
                                                    double (*part)[kNB]) {
  const int tid = threadIdx.x, j = tid % kNB, q = tid / kNB, i0 = q * (kNB / 4);
  cp_async_wait_all();
  double a0 = 0.0, a1 = 0.0;
  // Row i starts at i (i + 1) / 2: the offset of (i, j) grows by i + 1 from
  // row i to row i + 1.
  int off = i0 * (i0 + 1) / 2 + j;
#pragma unroll
  for (int ii = 0; ii < kNB / 4; ii += 2) {
    const int i = i0 + ii;
    if (i >= j && i < nb) a0 += Ls[off] * v[i];
    off += i + 1;
    if (i + 1 >= j && i + 1 < nb) a1 += Ls[off] * v[i + 1];
    off += i + 2;
  }
  part[q][j] = a0 + a1;
  __syncthreads();
  return (part[0][j] + part[1][j]) + (part[2][j] + part[3][j]);
}

// Forward
template <class T>
__global__ void __launch_bounds__(32 * kWarpsPerCta)
    k_fwd_small(const int32_t *list, int count, const int64_t *sfirst,
                const int64_t *srowptr, const int64_t *slofs,
                const int64_t *child_ptr, const int32_t *child_list,
                const int32_t *srel, const int64_t *zofs, const T *panel,
                double *x, double *zbuf) {
  __shared__ double zs[kWarpsPerCta][kSmallH];
  const int         warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int         idx  = blockIdx.x * kWarpsPerCta + warp;
  if (idx >= count) return;
  const int      J = list[idx];
  const int64_t  f = sfirst[J];
  const int      w = static_cast<int>(sfirst[J + 1] - f);
  const int      h = static_cast<int>(srowptr[J + 1] - srowptr[J]);
  double        *z = zs[warp];
  for (int i = lane; i < h; i += 32) z[i] = i < w ? x[f + i] : 0.0;
  __syncwarp();
  for (int64_t c = child_ptr[J]; c < child_ptr[J + 1]; c++) {
    const int      C  = child_list[c];
    const int      wc = static_cast<int>(sfirst[C + 1] - sfirst[C]);
    const int      rc = static_cast<int>(srowptr[C + 1] - srowptr[C]) - wc;
    const int32_t *rl = srel + srowptr[C] + wc;
    const double  *zc = zbuf + zofs[C] + wc;
    for (int a = lane; a < rc; a += 32) z[rl[a]] += zc[a];
    __syncwarp();
  }
  // Columns four at a time; the next four columns' entries of this lane's
  // rows (lane + 32 t) are loaded while the current four are applied.
  const T      *P  = panel + slofs[J];
  constexpr int RT = kSmallH / 32;
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
      const int k = k0 + u;
      if (k >= w) break;
      const double zk = z[k];
#pragma unroll
      for (int t = 0; t < RT; t++) {
        const int i = lane + 32 * t;
        if (i > k && i < h) z[i] -= static_cast<double>(cur[u][t]) * zk;
      }
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int t = 0; t < RT; t++) cur[u][t] = nxt[u][t];
  }
  double *zo = zbuf + zofs[J];
  for (int i = lane; i < h; i += 32) {
    if (i < w) x[f + i] = z[i];
    zo[i] = z[i];
  }
}


// Waits for this lane's entries p[lane + 32 i] (i < 4) of a block result, the
// entries at or past lim reading as 0; each round polls all four at once.
__device__ __forceinline__ void wait_block4(const double *p, int lim, double (&v)[4],
                                            int32_t *err, long polls) {
  const int lane = threadIdx.x % 32;
  unsigned  need = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) {
    v[i] = 0.0;
    if (lane + 32 * i < lim) need |= 1u << i;
  }
  for (long it = 0; need != 0 && it < polls; it++) {
    unsigned long long raw[4];
#pragma unroll
    for (int i = 0; i < 4; i++) raw[i] = (need >> i & 1u) ? ld_relaxed_u64(p + lane + 32 * i) : 0ull;
#pragma unroll
    for (int i = 0; i < 4; i++)
      if ((need >> i & 1u) && raw[i] != kPending) {
        v[i] = __longlong_as_double(static_cast<long long>(raw[i]));
        need &= ~(1u << i);
      }
    if ((it & 63) == 63) {
      if (*reinterpret_cast<volatile int32_t *>(err) != 0) return;
      __nanosleep(32);
    }
  }
  if (need != 0) atomicExch(err, 1);
}

// The value at p from a load issued ahead (raw) when that load already saw
// it, else the wait for it.
__device__ __forceinline__ double take_value(unsigned long long raw, const double *p,
                                             int32_t *err, long polls) {
  return raw != kPending ? __longlong_as_double(static_cast<long long>(raw))
                         : wait_value(p, err, polls);
}

__global__ void k_mark_pending(int64_t n, double *ready) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) reinterpret_cast<unsigned long long *>(ready)[i] = kPending;
}



// Forward solve of the large fronts of one level: one CTA per 128-row block
// R of a front.  z_R -= L_{R,b} y_b for the column blocks b left of R, in
// order, each as soon as y_b is ready: thread (q, i) = (tid / 128,
// tid % 128) takes row i and the columns 32 q .. 32 q + 31 of each tile (a
// warp's loads are one 128-byte column segment), loads its L values before
// the wait, and each lane waits for its own entry of y_b in the ready buffer
// (no CTA barrier per tile); the four slices are added in order at the end.
// A diagonal row block then solves y_R = Linv_R z_R into x and the ready
// buffer (block product with warp-local slices, see blk_i); rows at or past
// w are the front's update vector for its parent.
template <class T>
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_fwd_fronts(const SolveItem *items, const T *panel, const double *linv64t, const int64_t *gp,
                 const int64_t *gsrc, double *x, double *zbuf, int32_t *tickets,
                 double *ready, int32_t *err) {
  extern __shared__ __align__(16) double tri[];  // kFwdTri doubles: the staged Linv_R
  __shared__ __align__(16) double ys[kNB];
  __shared__ double ys2[4 * 33];
  __shared__ double yw[kSolveThreads / 32][32];
  __shared__ double part[4][kNB];
  // Thread 0 takes the CTA's ticket (the order in which CTAs take their work,
  // so every block a CTA waits for belongs to an earlier ticket) and copies
  // the item's record into shared memory: the code after the tile loop (on
  // the chain of diagonal blocks) reads the descriptor again, and from global
  // memory that took a round trip past an L1 the tiles had flushed.
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
  const int         item = sItem;
  const SolveFront &F    = sF;
  const int         R    = sR;
  const long        polls = sPolls;
  if (R < F.nb)
    stage_lower(linv64t + F.linv + static_cast<int64_t>(R) * kNB * kNB, tri);
  const int     tid = threadIdx.x, rr = tid % kNB, qq = tid / kNB;
  const int     warp = tid / 32, lane = tid % 32;
  const int64_t h = F.h;
  const int     w = F.w;
  const int64_t r = static_cast<int64_t>(R) * kNB + rr;
  const T      *P  = panel + F.panel;
  const int64_t n  = F.n;
  const double *yr = ready + ((item * 16 + threadIdx.x / 32) % kReadyCopies) * n + F.col0;
  const int     tiles = min(R, F.nb);
  // Right-hand side of this row: its entry of x (rows < w), then the
  // children's update vectors in child order.
  __shared__ double zs[kNB];
  if (qq == 0) {
    double zr = 0.0;
    if (r < h) {
      zr = r < w ? x[F.col0 + r] : 0.0;
      for (int64_t e = gp[F.gptr + r]; e < gp[F.gptr + r + 1]; e++) zr += zbuf[gsrc[e]];
    }
    zs[rr] = zr;
  }
  double acc = 0.0;
  // The next tile's L values are loaded while the current one waits for y_b
  // and is applied: two tiles in flight, so a CTA that starts late (when an
  // earlier one leaves its SM) catches up on the tiles already available at
  // about twice the rate of one tile at a time.
  float lv[32], lvn[32];
  auto  load_tile = [&](float (&dst)[32], int b) {
    const int c0 = b * kNB + qq * 32;
#pragma unroll
    for (int k = 0; k < 32; k++)
      dst[k] = (r < h && c0 + k < w) ? to_f(__ldg(P + r + static_cast<int64_t>(c0 + k) * h)) : 0.0f;
  };
  // The lane's entry of y_b is loaded ahead with the tile's L values too;
  // only an entry that was still pending then is waited for.
  auto load_y = [&](int b) {
    const int c0 = b * kNB + qq * 32;
    return c0 + lane < w ? ld_relaxed_u64(yr + c0 + lane) : 0ull;
  };
  unsigned long long yv = 0ull, yvn = 0ull;
  cp_async_wait_all();
  if (tiles > 0) {
    load_tile(lv, 0);
    yv = load_y(0);
  }
  // The last tile's block result is the one just before this block on the
  // chain: the first warp of each column quarter waits for the quarter's 32
  // entries and shares them with the quarter's other three warps through a
  // named barrier (each warp waiting for its own copy saw them up to 2 us
  // apart, and the CTA could only go on with the last).
  __shared__ double ylast[kNB];
  for (int b = 0; b + 1 < tiles; b++) {
    const int c0 = b * kNB + qq * 32;
    load_tile(lvn, b + 1);
    if (b + 2 < tiles) yvn = load_y(b + 1);
    yw[warp][lane] = c0 + lane < w ? take_value(yv, yr + c0 + lane, err, polls) : 0.0;
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 32; k++) acc += static_cast<double>(lv[k]) * yw[warp][k];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 32; k++) lv[k] = lvn[k];
    yv = yvn;
  }
  if (tiles > 0) {
    // The last tile: its L values are widened before the wait (float to
    // double conversions run at a quarter of the FMA rate; done after the
    // wait, by all 16 warps, they took about 0.5 us of the chain).
    const int c0 = (tiles - 1) * kNB + qq * 32;
    double    ld[32];
#pragma unroll
    for (int k = 0; k < 32; k++) ld[k] = static_cast<double>(lv[k]);
    if (warp % 4 == 0)
      ylast[qq * 32 + lane] =
          c0 + lane < w ? wait_value(ready + ((item + qq) % kReadyCopies) * n + F.col0 + c0 + lane,
                                     err, polls)
                        : 0.0;
    asm volatile("bar.sync %0, %1;" ::"r"(1 + qq), "r"(kNB) : "memory");
#pragma unroll
    for (int k = 0; k < 32; k++) acc += ld[k] * ylast[qq * 32 + k];
  }
  part[qq][rr] = acc;
  __syncthreads();
  double z = 0.0;
  if (qq == 0 && r < h) z = zs[rr] - ((part[0][rr] + part[1][rr]) + (part[2][rr] + part[3][rr]));
  if (R < F.nb) {
    const int nbk = min(kNB, w - R * kNB);
    if (qq == 0) ys[rr] = rr < nbk ? z : 0.0;
    __syncthreads();
    const double y  = block_lower_apply(tri, ys);
    const int    iy = blk_i();
    if (blk_q() == 0 && iy < nbk && sPublish) {
      const int64_t j = F.col0 + R * kNB + iy;
#pragma unroll
      for (int c = 0; c < kReadyCopies; c++) st_relaxed_f64(ready + c * n + j, y);
      x[j] = y;
    }
    if ((R + 1) * kNB > w && h > w) {
      // Rows of this block at or past w: their product with the block.
      if (blk_q() == 0) ys2[pad(iy)] = iy < nbk ? y : 0.0;
      __syncthreads();
      double a2 = 0.0;
      if (r >= w && r < h)
        for (int k = qq * 32; k < min(nbk, qq * 32 + 32); k++)
          a2 += static_cast<double>(to_f(P[r + static_cast<int64_t>(R * kNB + k) * h])) * ys2[pad(k)];
      part[qq][rr] = a2;
      __syncthreads();
      if (qq == 0 && r >= w && r < h)
        z -= (part[0][rr] + part[1][rr]) + (part[2][rr] + part[3][rr]);
    }
  }
  if (qq == 0 && r >= w && r < h) zbuf[F.zofs + r] = z;
}

__global__ void k_dscale(int64_t n, const float *Dinv, double *x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] *= static_cast<double>(Dinv[i]);
}

// ---------------------------------------------------------------------------
// Backward
template <class T>
__global__ void __launch_bounds__(32 * kWarpsPerCta)
    k_bwd_small(const int32_t *list, int count, const int64_t *sfirst,
                const int64_t *srowptr, const int32_t *srows,
                const int64_t *slofs, const T *panel, double *x) {
  __shared__ double zs[kWarpsPerCta][kSmallH];
  const int         warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int         idx  = blockIdx.x * kWarpsPerCta + warp;
  if (idx >= count) return;
  const int      J  = list[idx];
  const int64_t  f  = sfirst[J];
  const int      w  = static_cast<int>(sfirst[J + 1] - f);
  const int      h  = static_cast<int>(srowptr[J + 1] - srowptr[J]);
  const int32_t *rw = srows + srowptr[J];
  double        *z  = zs[warp];
  for (int i = lane; i < h; i += 32) z[i] = i < w ? x[f + i] : x[rw[i]];
  __syncwarp();
  // Columns four at a time from the last; the next four columns' entries of
  // this lane's rows (lane + 32 t) are loaded while the current four are used.
  const T      *P  = panel + slofs[J];
  constexpr int RT = kSmallH / 32;
  float         cur[4][RT], nxt[4][RT];
  auto          load4 = [&](float (*buf)[RT], int k0) {  // columns k0, k0-1, ..
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
      const int k = k0 - u;
      if (k < 0) break;
      double s = 0.0;
#pragma unroll
      for (int t = 0; t < RT; t++) {
        const int i = lane + 32 * t;
        if (i > k && i < h) s += static_cast<double>(cur[u][t]) * z[i];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) z[k] -= s;
      __syncwarp();
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int t = 0; t < RT; t++) cur[u][t] = nxt[u][t];
  }
  for (int i = lane; i < w; i += 32) x[f + i] = z[i];
}


// Backward solve, off-diagonal rows: CTA c takes rows w + 128c .. of one
// front and writes t_k = sum_r L_{r,k} z_r for every column k of the front
// (warp per column, rows over the lanes, shuffle reduction) to its partials.
template <class T>
__global__ void __launch_bounds__(kSolveThreads)
    k_bwd_chunks(const SolveFront *fr, const int32_t *fmap, const T *panel,
                 const int32_t *srows,
                 const double *x, double *part) {
  __shared__ double zr[kNB];
  const SolveFront  F = fr[fmap[blockIdx.x]];
  const int         c = blockIdx.x - F.chunk0;
  const int         tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int64_t     h = F.h, w = F.w;
  const int64_t     r0 = w + static_cast<int64_t>(c) * kNB;
  const int         nr = static_cast<int>(h - r0 < kNB ? h - r0 : kNB);
  if (tid < kNB) zr[tid] = tid < nr ? x[srows[F.rows + r0 + tid]] : 0.0;
  __syncthreads();
  const T      *P  = panel + F.panel + r0;
  double       *pp = part + F.part + static_cast<int64_t>(c) * w;
  constexpr int kWarps = kSolveThreads / 32;
#pragma unroll 2
  for (int64_t k = warp; k < w; k += kWarps) {
    const T     *col = P + k * h;
    double       s   = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int rr = lane + 32 * i;
      if (rr < nr) s += static_cast<double>(to_f(__ldg(col + rr))) * zr[rr];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) pp[k] = s;
  }
}

// Backward solve, column blocks of the large fronts of one level: one CTA
// per column block b (last first).  t = (sum of the chunk partials, in chunk
// order) + (sum over the row blocks R > b of the diagonal part, last first,
// each as soon as x_R is in the ready buffer); then x_b = Linv_b^T (z_b - t)
// into x and the ready buffer.  In a tile, warp v takes the block's columns
// 8v .. 8v+7 and the lanes the rows.
template <class T>
__global__ void __launch_bounds__(kSolveThreads, 1)
    k_bwd_fronts(const SolveItem *items, const T *panel,
                 const double *linv64t,
                 double *x, const double *part, int32_t *tickets,
                 double *ready, int32_t *err) {
  extern __shared__ double tri[];  // kTri doubles: the staged Linv_b^T
  __shared__ double v[kNB];
  __shared__ double ts[kNB];
  __shared__ double red[4][kNB];
  // Ticket and item record as in k_fwd_fronts.
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
  const int         item = sItem;
  const SolveFront &F    = sF;
  const int         b    = sB;
  const long        polls = sPolls;
  stage_upper(linv64t + F.linv + static_cast<int64_t>(b) * kNB * kNB, tri,
              min(kNB, F.w - b * kNB));
  const int         tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int64_t     h = F.h;
  const int         w = F.w;
  const int         nbk = min(kNB, w - b * kNB);
  // This block's right-hand side, read now (not on the chain at the end).
  if (tid < nbk) v[tid] = x[F.col0 + b * kNB + tid];
  const T          *P   = panel + F.panel;
  const int64_t     n   = F.n;
  const double     *xr  = ready + ((item * 16 + threadIdx.x / 32) % kReadyCopies) * n + F.col0;
  {
    // Chunk partials of column k (no wait needed): thread (q, k) adds chunks
    // q, q + 4, ...; the four sums are added in order below.
    const int k = tid % kNB, q = tid / kNB;
    double    s = 0.0;
    if (k < nbk)
      for (int c = q; c < F.chunks; c += 4)
        s += part[F.part + static_cast<int64_t>(c) * w + b * kNB + k];
    red[q][k] = s;
  }
  double acc[8];
#pragma unroll
  for (int j = 0; j < 8; j++) acc[j] = 0.0;
  // Tile R (the warp's columns 8 warp + j, rows lane + 32 i of row block R);
  // the next tile (R - 1) is loaded while the current one waits for x_R and
  // is applied, as in the forward solve.
  float lv[8][4], lvn[8][4];
  auto  load_tile = [&](float (&dst)[8][4], int R) {
    const int64_t rb   = static_cast<int64_t>(R) * kNB;
    const int     rows = min(kNB, w - R * kNB);
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int c = warp * 8 + j;
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const int rr = lane + 32 * i;
        dst[j][i]    = (c < nbk && rr < rows)
                           ? to_f(__ldg(P + rb + rr + static_cast<int64_t>(b * kNB + c) * h))
                           : 0.0f;
      }
    }
  };
  // The last tile (R = b + 1) is the block just before this one on the
  // chain: one warp waits for all of x_R and shares it (as in the forward).
  __shared__ double xlast[kNB];
  if (F.nb - 1 > b) load_tile(lv, F.nb - 1);
  for (int R = F.nb - 1; R > b + 1; R--) {
    const int64_t rb   = static_cast<int64_t>(R) * kNB;
    const int     rows = min(kNB, w - R * kNB);
    load_tile(lvn, R - 1);
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int    rr = lane + 32 * i;
      const double zv = rr < rows ? wait_value(xr + rb + rr, err, polls) : 0.0;
#pragma unroll
      for (int j = 0; j < 8; j++) acc[j] += static_cast<double>(lv[j][i]) * zv;
    }
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int i = 0; i < 4; i++) lv[j][i] = lvn[j][i];
  }
  if (F.nb - 1 > b) {
    // The last tile (R = b + 1): its L values are widened before the wait,
    // as in the forward solve.
    const int64_t rb   = static_cast<int64_t>(b + 1) * kNB;
    const int     rows = min(kNB, w - (b + 1) * kNB);
    double        ld[8][4];
#pragma unroll
    for (int j = 0; j < 8; j++)
#pragma unroll
      for (int i = 0; i < 4; i++) ld[j][i] = static_cast<double>(lv[j][i]);
    if (warp == 0) {
      double xv[4];
      wait_block4(ready + (item % kReadyCopies) * n + F.col0 + rb, rows, xv, err, polls);
#pragma unroll
      for (int i = 0; i < 4; i++) xlast[lane + 32 * i] = xv[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const double zv = xlast[lane + 32 * i];
#pragma unroll
      for (int j = 0; j < 8; j++) acc[j] += ld[j][i] * zv;
    }
  }
  // Sums of the warp's 8 columns over its 32 lanes: the usual butterfly
  // (partners lane ^ 16, ^ 8, ^ 4, ^ 2, ^ 1), but at each of the first three
  // levels a lane keeps half of its columns and sends the other half, so it
  // takes 4 + 2 + 1 + 1 + 1 shuffles instead of 8 x 5 (the same additions in
  // the same order).  Lane l ends with column (l >> 2) & 7.
  {
    const unsigned full = 0xffffffffu;
    double         s4[4], s2[2];
    const bool     b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const double keep = b4 ? acc[u + 4] : acc[u], send = b4 ? acc[u] : acc[u + 4];
      s4[u] = keep + __shfl_xor_sync(full, send, 16);
    }
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const double keep = b3 ? s4[u + 2] : s4[u], send = b3 ? s4[u] : s4[u + 2];
      s2[u] = keep + __shfl_xor_sync(full, send, 8);
    }
    double s = (b2 ? s2[1] : s2[0]) + __shfl_xor_sync(full, b2 ? s2[0] : s2[1], 4);
    s += __shfl_xor_sync(full, s, 2);
    s += __shfl_xor_sync(full, s, 1);
    if ((lane & 3) == 0) ts[warp * 8 + ((lane >> 2) & 7)] = s;
  }
  __syncthreads();
  if (tid < nbk)
    v[tid] = v[tid] - (((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid])) + ts[tid]);
  __syncthreads();
  // Lt[i * kNB + j] = Linv[i][j]
  const double xb = block_upper_apply(tri, v, nbk, red);
  if (tid < nbk) {
    const int64_t j = F.col0 + b * kNB + tid;
#pragma unroll
    for (int c = 0; c < kReadyCopies; c++) st_relaxed_f64(ready + c * n + j, xb);
    x[j] = xb;
  }
}

// ---------------------------------------------------------------------------
void SolveWorkspace::allocate(const Plan &P) {
  release_graph();
  zbuf.resize(std::max<int64_t>(P.S.z_elems, 1) * sizeof(double));
  part.resize(std::max<int64_t>(P.spart_elems, 1) * sizeof(double));
  sync.resize(std::max<int64_t>(P.sync_elems, 1) * sizeof(int32_t));
  ready.resize(std::max<int64_t>(kReadyCopies * P.S.n, 1) * sizeof(double));
  err.resize(sizeof(SolveCtl));
  device_zero(err.as<void>(), sizeof(SolveCtl));
  xbuf.resize(std::max<int64_t>(P.S.n, 1) * sizeof(double));
}

cudaStream_t SideStream::fork(cudaStream_t s) {
  if (!st_) {
    MPIR_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    MPIR_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
    MPIR_CUDA(cudaEventCreateWithFlags(&join_, cudaEventDisableTiming));
  }
  MPIR_CUDA(cudaEventRecord(fork_, s));
  MPIR_CUDA(cudaStreamWaitEvent(st_, fork_, 0));
  return st_;
}

void SideStream::join(cudaStream_t s) {
  MPIR_CUDA(cudaEventRecord(join_, st_));
  MPIR_CUDA(cudaStreamWaitEvent(s, join_, 0));
}

void SideStream::reset() {
  if (st_) {
    cudaStreamSynchronize(st_);
    cudaStreamDestroy(st_);
  }
  if (fork_) cudaEventDestroy(fork_);
  if (join_) cudaEventDestroy(join_);
  st_   = nullptr;
  fork_ = join_ = nullptr;
}

void SolveWorkspace::release_graph() {
  if (graph) cudaGraphExecDestroy(graph);
  graph = nullptr;
}

void ldlt_solve_graph(const Plan &P, const Numeric &F, double *x, SolveWorkspace &ws,
                      cudaStream_t s, cudaStream_t capture_stream) {
  const int64_t n = P.S.n;
  if (n == 0) return;
  if (kernel_timer().enabled) {  // per-class timing needs the plain launches
    ldlt_solve(P, F, x, ws, s);
    return;
  }
  if (!ws.graph) {
    cudaGraph_t g = nullptr;
    MPIR_CUDA(cudaStreamSynchronize(capture_stream));
    MPIR_CUDA(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
    {
      LaunchCapture cap;
      ldlt_solve(P, F, ws.xbuf.as<double>(), ws, capture_stream);
      ws.graph_launches = cap.count();
    }
    MPIR_CUDA(cudaStreamEndCapture(capture_stream, &g));
    MPIR_CUDA(cudaGraphInstantiate(&ws.graph, g, 0));
    cudaGraphDestroy(g);
  }
  MPIR_CUDA(cudaMemcpyAsync(ws.xbuf.as<void>(), x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  MPIR_CUDA(cudaGraphLaunch(ws.graph, s));
  launch_add(ws.graph_launches);
  MPIR_CUDA(cudaMemcpyAsync(x, ws.xbuf.as<void>(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

template <class T>
static void ldlt_solve_t(const Plan &P, const Numeric &F, const T *pan, double *x,
                         SolveWorkspace &ws, cudaStream_t s, int phases) {
  const Symbolic &S  = P.S;
  KernelTimer    &kt = kernel_timer();
  if (S.n == 0) return;
  const double *lvt = F.linv64t.as<double>();
  double      *zbuf = ws.zbuf.as<double>();
  const int    nl   = static_cast<int>(P.levels.size());
  // Tickets (2 per level); the ready buffer is marked pending before each
  // direction.
  int32_t          *sync  = ws.sync.as<int32_t>();
  double           *ready = ws.ready.as<double>();
  int32_t          *err   = ws.err.as<int32_t>();
  const SolveFront *sf    = P.solve_fronts.as<SolveFront>();
  const bool        block = P.nblock_fronts > 0;
  const int64_t     nready = kReadyCopies * S.n;
  const unsigned    nmark  = static_cast<unsigned>((nready + 255) / 256);
  if (block) MPIR_CUDA(cudaMemsetAsync(sync, 0, P.sync_elems * sizeof(int32_t), s));
  if (block && (phases & kForward)) launch(k_mark_pending, nmark, 256, 0, s, nready, ready);
  static std::atomic<bool> attr{false};
  if (!attr) {
    MPIR_CUDA(cudaFuncSetAttribute(k_fwd_fronts<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kFwdTri * sizeof(double))));
    MPIR_CUDA(cudaFuncSetAttribute(k_bwd_fronts<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kTri * sizeof(double))));
    attr = true;
  }
  kt.begin(kKcSolveFwd, s);
  for (int t = 0; t < nl && (phases & kForward); t++) {
    const LevelPlan &L    = P.levels[t];
    const bool       both = L.sw_count > 0 && L.sf_count > 0;
    cudaStream_t     ss   = both ? ws.side.fork(s) : s;  // warp fronts beside block fronts
    if (L.sw_count > 0)
      launch(k_fwd_small<T>, (L.sw_count + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0,
             ss, P.swarp_list.as<int32_t>() + L.sw_begin, L.sw_count, P.sfirst.as<int64_t>(),
             P.srowptr.as<int64_t>(), P.slofs.as<int64_t>(), P.child_ptr.as<int64_t>(),
             P.child_list.as<int32_t>(), P.srel.as<int32_t>(), P.zofs.as<int64_t>(), pan, x,
             zbuf);
    if (L.sf_count > 0) {
      launch(k_fwd_fronts<T>, L.fwd_items, kSolveThreads, kFwdTri * sizeof(double), s,
             P.fwd_item.as<SolveItem>() + L.fwd_map0, pan, lvt, P.gp.as<int64_t>(),
             P.gsrc.as<int64_t>(), x, zbuf, sync + 2 * t, ready, err);
    }
    if (both) ws.side.join(s);
  }
  if (phases & kDiagonal)
    launch(k_dscale, static_cast<unsigned>((S.n + 255) / 256), 256, 0, s,
           S.n, F.Dinv.as<float>(), x);
  kt.end(s);
  if (!(phases & kBackward)) return;
  MPIR_CHECK_LAUNCH();
  kt.begin(kKcSolveBwd, s);
  if (block) launch(k_mark_pending, nmark, 256, 0, s, nready, ready);
  for (int t = nl - 1; t >= 0; t--) {
    const LevelPlan &L    = P.levels[t];
    const bool       both = L.sw_count > 0 && L.sf_count > 0;
    cudaStream_t     ss   = both ? ws.side.fork(s) : s;
    if (L.sw_count > 0)
      launch(k_bwd_small<T>, (L.sw_count + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0,
             ss, P.swarp_list.as<int32_t>() + L.sw_begin, L.sw_count, P.sfirst.as<int64_t>(),
             P.srowptr.as<int64_t>(), P.srows.as<int32_t>(), P.slofs.as<int64_t>(), pan, x);
    if (L.sf_count > 0) {
      if (L.bwd_chunk_items > 0)
        launch(k_bwd_chunks<T>, L.bwd_chunk_items, kSolveThreads, 0, s, sf + L.sf_begin,
               P.chunk_map.as<int32_t>() + L.chunk_map0, pan, P.srows.as<int32_t>(),
               static_cast<const double *>(x),
               ws.part.as<double>());
      launch(k_bwd_fronts<T>, L.bwd_owner_items, kSolveThreads, kTri * sizeof(double), s,
             P.own_item.as<SolveItem>() + L.own_map0, pan,
             F.linv64t.as<double>(), x,
             static_cast<const double *>(ws.part.as<double>()), sync + 2 * t + 1, ready, err);
    }
    if (both) ws.side.join(s);
  }
  kt.end(s);
  MPIR_CHECK_LAUNCH();
}


void ldlt_solve(const Plan &P, const Numeric &F, double *x, SolveWorkspace &ws,
                cudaStream_t s, int phases) {
  switch (F.solve_prec()) {
    case 2:
      ldlt_solve_t(P, F, F.panel16.as<__nv_bfloat16>(), x, ws, s, phases);
      break;
    case 3:
      ldlt_solve_t(P, F, F.panel16.as<__half>(), x, ws, s, phases);
      break;
    default:
      ldlt_solve_t(P, F, F.panel.as<float>(), x, ws, s, phases);
  }
}


// ---------------------------------------------------------------------------
// QDLDL_solve without device allocation.
//
// For callers that cannot call cudaMalloc: processes whose device memory is
// reserved up front and handed out entirely by their own pooling allocator,
// and loops that cannot take cudaMalloc's implicit device-wide
// synchronisation.  All
// device data of this entry point (the supernodal layout of L, the factor
// values, Dinv, the fronts' update vectors and x) is packed into the one
// file-scope array below, of fixed size, that every GPU holds once this
// library is loaded.  Only factors whose supernodal fronts have at most
// kSmallFront rows are taken (the warp-per-front kernels; no diagonal-block
// inverses), and the packed data must fit the array.
namespace {
constexpr size_t kNoAllocScratchBytes = size_t{32} << 20;  // 32 MiB
constexpr int    kNoAllocMaxDevices   = 64;
}  // namespace

static __device__ __align__(256) unsigned char g_solve_scratch[kNoAllocScratchBytes];

namespace {
// Device address of g_solve_scratch on each device, looked up on the first
// call that uses that device (atomic: host threads may make their first
// calls at the same time; they store the same address).
std::atomic<void *> g_solve_scratch_addr[kNoAllocMaxDevices] = {};

// Restores the calling thread's current device on every return path.
struct DeviceRestore {
  int  saved = -1;
  DeviceRestore() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceRestore() {
    if (saved >= 0) cudaSetDevice(saved);
  }
};
}  // namespace

int qdldl_solve_noalloc(int64_t n, const int64_t *Lp, const int64_t *Li, const float *Lx,
                        const float *Dinv, double *x, int device, std::string &err) {
  if (n < 0 || device < 0 || device >= kNoAllocMaxDevices) {
    err = "invalid dimension or device";
    return kBadArgument;
  }
  if (n == 0) return kOk;
  Symbolic  S;
  const int rc = analyze_from_L(n, Lp, Li, S, err);
  if (rc != kOk) return rc;
  for (int64_t J = 0; J < S.ns; J++)
    if (S.h(J) > kSmallFront) {
      err = "a supernodal front has " + std::to_string(S.h(J)) + " rows; this entry point takes at most " +
            std::to_string(kSmallFront);
      return -7;
    }
  // Factor values in the panel layout (explicit zeros for padding).
  std::vector<float> pan(S.panel_elems, 0.0f);
  for (int64_t J = 0; J < S.ns; J++) {
    const int64_t f = S.sfirst[J], l = S.sfirst[J + 1], w = l - f, h = S.h(J);
    for (int64_t j = f; j < l; j++) {
      int64_t q = S.srowptr[J] + w;  // rows below the supernode's own columns
      for (int64_t p = Lp[j]; p < Lp[j + 1]; p++) {
        const int64_t r = Li[p];
        int64_t       lr;
        if (r < l) {
          lr = r - f;
        } else {
          while (S.srows[q] < r) q++;
          lr = w + (q - S.srowptr[J] - w);
        }
        pan[S.slofs[J] + (j - f) * h + lr] = Lx[p];
      }
    }
  }
  // Pack every region into the scratch array, 256-byte aligned.
  struct Region {
    const void *src;
    size_t      bytes;
    size_t      ofs;
  };
  std::vector<Region> reg;
  size_t              top = 0;
  auto add = [&](const void *src, size_t bytes) {
    top = (top + 255) / 256 * 256;
    reg.push_back({src, bytes, top});
    top += bytes;
    return reg.size() - 1;
  };
  const size_t r_sfirst = add(S.sfirst.data(), S.sfirst.size() * sizeof(int64_t));
  const size_t r_srowptr = add(S.srowptr.data(), S.srowptr.size() * sizeof(int64_t));
  const size_t r_srows = add(S.srows.data(), S.srows.size() * sizeof(int32_t));
  const size_t r_srel = add(S.srel.data(), S.srel.size() * sizeof(int32_t));
  const size_t r_slofs = add(S.slofs.data(), S.slofs.size() * sizeof(int64_t));
  const size_t r_cptr = add(S.child_ptr.data(), S.child_ptr.size() * sizeof(int64_t));
  const size_t r_clist = add(S.child_list.data(), S.child_list.size() * sizeof(int32_t));
  const size_t r_zofs = add(S.zofs.data(), S.zofs.size() * sizeof(int64_t));
  const size_t r_level = add(S.level_sup.data(), S.level_sup.size() * sizeof(int32_t));
  const size_t r_panel = add(pan.data(), pan.size() * sizeof(float));
  const size_t r_dinv = add(Dinv, n * sizeof(float));
  const size_t r_x = add(x, n * sizeof(double));
  const size_t r_zbuf = add(nullptr, S.z_elems * sizeof(double));  // written on the device
  if (top > kNoAllocScratchBytes) {
    err = "needs " + std::to_string(top) + " bytes of device scratch; this entry point has " +
          std::to_string(kNoAllocScratchBytes);
    return kBadArgument;
  }
  DeviceRestore restore;  // the caller's current device is left as it was
  MPIR_CUDA(cudaSetDevice(device));
  void *addr = g_solve_scratch_addr[device].load(std::memory_order_acquire);
  if (!addr) {
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_solve_scratch);
    if (e != cudaSuccess) throw CudaError(e, "cudaGetSymbolAddress(g_solve_scratch)");
    g_solve_scratch_addr[device].store(addr, std::memory_order_release);
  }
  unsigned char     *base = static_cast<unsigned char *>(addr);
  const cudaStream_t s    = cudaStreamPerThread;
  for (const Region &r : reg)
    if (r.src && r.bytes)
      MPIR_CUDA(cudaMemcpyAsync(base + r.ofs, r.src, r.bytes, cudaMemcpyHostToDevice, s));
  auto at = [&](size_t i) { return static_cast<void *>(base + reg[i].ofs); };
  const int64_t *sfirst  = static_cast<const int64_t *>(at(r_sfirst));
  const int64_t *srowptr = static_cast<const int64_t *>(at(r_srowptr));
  const int32_t *srows   = static_cast<const int32_t *>(at(r_srows));
  const int32_t *srel    = static_cast<const int32_t *>(at(r_srel));
  const int64_t *slofs   = static_cast<const int64_t *>(at(r_slofs));
  const int64_t *cptr    = static_cast<const int64_t *>(at(r_cptr));
  const int32_t *clist   = static_cast<const int32_t *>(at(r_clist));
  const int64_t *zofs    = static_cast<const int64_t *>(at(r_zofs));
  const int32_t *level   = static_cast<const int32_t *>(at(r_level));
  const float   *panel   = static_cast<const float *>(at(r_panel));
  const float   *dinv    = static_cast<const float *>(at(r_dinv));
  double        *xd      = static_cast<double *>(at(r_x));
  double        *zbuf    = static_cast<double *>(at(r_zbuf));
  const int      nl      = S.nlevels;
  for (int t = 0; t < nl; t++) {
    const int32_t cnt = static_cast<int32_t>(S.level_ptr[t + 1] - S.level_ptr[t]);
    launch(k_fwd_small<float>, (cnt + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, s,
           level + S.level_ptr[t], cnt, sfirst, srowptr, slofs, cptr, clist, srel, zofs, panel,
           xd, zbuf);
  }
  launch(k_dscale, static_cast<unsigned>((n + 255) / 256), 256, 0, s, n, dinv, xd);
  for (int t = nl - 1; t >= 0; t--) {
    const int32_t cnt = static_cast<int32_t>(S.level_ptr[t + 1] - S.level_ptr[t]);
    launch(k_bwd_small<float>, (cnt + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, s,
           level + S.level_ptr[t], cnt, sfirst, srowptr, srows, slofs, panel, xd);
  }
  MPIR_CHECK_LAUNCH();
  MPIR_CUDA(cudaMemcpyAsync(x, xd, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
  return kOk;
}

}  // namespace mpir
