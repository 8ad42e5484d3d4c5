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
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.hpp"
#include "solve.hpp"

namespace mpir {

constexpr int kWarpsPerCta = 4;
constexpr int kSmallH      = kSmallFront;

// ---------------------------------------------------------------------------
// y = Linv z for one 128-column block with 512 threads: thread (q, i) adds
// the 32 products of row i in column slice q (unrolled, independent loads);
// slices are summed in order.  Linv is lower triangular, column-major.
__device__ __forceinline__ double block_lower_apply(const double *Lv, const double *zb, int nb,
                                                    double (*part)[kNB]) {
  const int tid = threadIdx.x, i = tid % kNB, q = tid / kNB;
  double    acc = 0.0;
#pragma unroll
  for (int jj = 0; jj < kNB / 4; jj++) {
    const int j = q * (kNB / 4) + jj;
    if (j <= i && i < nb) acc += Lv[i + j * kNB] * zb[j];
  }
  part[q][i] = acc;
  __syncthreads();
  return (part[0][i] + part[1][i]) + (part[2][i] + part[3][i]);
}

// x = Linv^T v with the row-major copy Lt (Lt[i * kNB + j] = Linv[i][j]):
// thread (q, j) adds rows i >= j of slice q.
__device__ __forceinline__ double block_upper_apply(const double *Lt, const double *v, int nb,
                                                    double (*part)[kNB]) {
  const int tid = threadIdx.x, j = tid % kNB, q = tid / kNB;
  double    acc = 0.0;
#pragma unroll
  for (int ii = 0; ii < kNB / 4; ii++) {
    const int i = q * (kNB / 4) + ii;
    if (i >= j && i < nb) acc += Lt[i * kNB + j] * v[i];
  }
  part[q][j] = acc;
  __syncthreads();
  return (part[0][j] + part[1][j]) + (part[2][j] + part[3][j]);
}

// Forward
__global__ void __launch_bounds__(32 * kWarpsPerCta)
    k_fwd_small(const int32_t *list, int count, const int64_t *sfirst,
                const int64_t *srowptr, const int64_t *slofs,
                const int64_t *child_ptr, const int32_t *child_list,
                const int32_t *srel, const int64_t *zofs, const float *panel,
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
  const float *P = panel + slofs[J];
  for (int k = 0; k < w; k++) {
    const double zk = z[k];
    for (int i = k + 1 + lane; i < h; i += 32)
      z[i] -= static_cast<double>(P[i + (int64_t)k * h]) * zk;
    __syncwarp();
  }
  double *zo = zbuf + zofs[J];
  for (int i = lane; i < h; i += 32) {
    if (i < w) x[f + i] = z[i];
    zo[i] = z[i];
  }
}

// Large fronts: right-hand side plus children's update vectors, then the
// solution of the first column block, y_0 = Linv_0 z_0, stored into x.
__global__ void __launch_bounds__(kSolveThreads)
    k_fwd_gather(const int32_t *list, const int64_t *sfirst, const int64_t *srowptr,
                 const int64_t *child_ptr, const int32_t *child_list, const int32_t *srel,
                 const int64_t *zofs, const int64_t *linv_ofs, const double *linv64, double *x,
                 double *zbuf) {
  __shared__ double zb[kNB];
  __shared__ double part[4][kNB];
  const int     J = list[blockIdx.x];
  const int64_t f = sfirst[J];
  const int64_t w = sfirst[J + 1] - f;
  const int64_t h = srowptr[J + 1] - srowptr[J];
  double       *z = zbuf + zofs[J];
  for (int64_t i = threadIdx.x; i < h; i += blockDim.x) z[i] = i < w ? x[f + i] : 0.0;
  __syncthreads();
  for (int64_t c = child_ptr[J]; c < child_ptr[J + 1]; c++) {
    const int      C  = child_list[c];
    const int64_t  wc = sfirst[C + 1] - sfirst[C];
    const int64_t  rc = srowptr[C + 1] - srowptr[C] - wc;
    const int32_t *rl = srel + srowptr[C] + wc;
    const double  *zc = zbuf + zofs[C] + wc;
    for (int64_t a = threadIdx.x; a < rc; a += blockDim.x) z[rl[a]] += zc[a];
    __syncthreads();
  }
  const int nb = static_cast<int>(w < kNB ? w : kNB);
  if (threadIdx.x < nb) zb[threadIdx.x] = z[threadIdx.x];
  __syncthreads();
  const double y = block_lower_apply(linv64 + linv_ofs[J], zb, nb, part);
  if (threadIdx.x < nb) x[f + threadIdx.x] = y;
}

// One column block of the large fronts.  The block's solution y is already
// in x; each CTA updates its 128 rows below the block, z_r -= L_{r,b} y, with
// the block's columns split in four quarters over the CTA's 512 threads.
// The first CTA's rows are the next block, so once they are updated it
// solves that block, y' = Linv_{b+1} z_{b+1}, into x for the next step.
__global__ void __launch_bounds__(kSolveThreads)
    k_fwd_step(const StepDesc *descs, int ndesc, const float *panel,
               const double *linv64, double *x, double *zbuf) {
  __shared__ double y[kNB];
  __shared__ double part[4][kNB];
  const int         t  = blockIdx.x;
  int               lo = 0, hi = ndesc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (descs[mid].fsolve_tile0 <= t) lo = mid; else hi = mid - 1;
  }
  const StepDesc d     = descs[lo];
  const int      local = t - d.fsolve_tile0;
  const int      tid   = threadIdx.x;
  const int64_t  h     = d.h;
  double        *z     = zbuf + d.zofs;
  if (tid < d.nbk) y[tid] = x[(int64_t)d.col0 + d.kb + tid];
  __syncthreads();
  const int     rr = tid % kSolveRows, qq = tid / kSolveRows;
  const int64_t r  = (int64_t)d.kb + d.nbk + (int64_t)local * kSolveRows + rr;
  double        acc = 0.0;
  if (r < h) {
    const float *P  = panel + d.panel + r + (int64_t)d.kb * h;
    const int    k1 = min(d.nbk, (qq + 1) * (kNB / 4));
    for (int k = qq * (kNB / 4); k < k1; k++)
      acc += static_cast<double>(P[(int64_t)k * h]) * y[k];
  }
  part[qq][rr] = acc;
  __syncthreads();
  if (qq == 0 && r < h) z[r] -= (part[0][rr] + part[1][rr]) + (part[2][rr] + part[3][rr]);
  const int kn = d.kb + d.nbk;
  if (local == 0 && kn < d.w) {
    __syncthreads();
    const int nb = d.w - kn < kNB ? d.w - kn : kNB;
    if (tid < nb) y[tid] = z[kn + tid];  // the next block's right-hand side
    __syncthreads();
    const double yn = block_lower_apply(linv64 + d.linv + (int64_t)kNB * kNB, y, nb, part);
    if (tid < nb) x[(int64_t)d.col0 + kn + tid] = yn;
  }
}

__global__ void k_dscale(int64_t n, const float *Dinv, double *x) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) x[i] *= static_cast<double>(Dinv[i]);
}

// ---------------------------------------------------------------------------
// Backward
__global__ void __launch_bounds__(32 * kWarpsPerCta)
    k_bwd_small(const int32_t *list, int count, const int64_t *sfirst,
                const int64_t *srowptr, const int32_t *srows,
                const int64_t *slofs, const float *panel, double *x) {
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
  const float *P = panel + slofs[J];
  for (int k = w - 1; k >= 0; k--) {
    double s = 0.0;
    for (int i = k + 1 + lane; i < h; i += 32)
      s += static_cast<double>(P[i + (int64_t)k * h]) * z[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) z[k] -= s;
    __syncwarp();
  }
  for (int i = lane; i < w; i += 32) x[f + i] = z[i];
}

__global__ void k_bwd_gather(const int32_t *list, const int64_t *sfirst,
                             const int64_t *srowptr, const int32_t *srows,
                             const int64_t *zofs, const double *x,
                             double *zbuf) {
  const int      J  = list[blockIdx.x];
  const int64_t  f  = sfirst[J];
  const int64_t  w  = sfirst[J + 1] - f;
  const int64_t  h  = srowptr[J + 1] - srowptr[J];
  const int32_t *rw = srows + srowptr[J];
  double        *z  = zbuf + zofs[J];
  for (int64_t i = threadIdx.x; i < h; i += blockDim.x)
    z[i] = i < w ? x[f + i] : x[rw[i]];
}

// One column block, backward: partial sums t_k = sum_r L_{r,kb+k} z_r over a
// chunk of 128 rows below the block (each warp takes 8 of the block's
// columns); the last chunk to finish adds the partials in chunk order and
// solves x_b = Linv^T (z_b - t) with the row-major copy of the inverse.
__global__ void __launch_bounds__(kSolveThreads)
    k_bwd_step(const StepDesc *descs, int ndesc, const float *panel,
               const double *linv64t, double *x, double *zbuf, double *part,
               int32_t *counter) {
  __shared__ double zr[kSolveChunk];
  __shared__ double v[kNB];
  __shared__ double red[4][kNB];
  __shared__ int    last;
  const int         t  = blockIdx.x;
  int               lo = 0, hi = ndesc - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (descs[mid].bsolve_chunk0 <= t) lo = mid; else hi = mid - 1;
  }
  const StepDesc d     = descs[lo];
  const int      chunk = t - d.bsolve_chunk0;
  const int      tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int64_t  h   = d.h;
  double        *z   = zbuf + d.zofs;
  const int64_t  r0  = (int64_t)d.kb + d.nbk + (int64_t)chunk * kSolveChunk;
  const int64_t  r1  = min(r0 + kSolveChunk, h);
  if (tid < kSolveChunk) zr[tid] = r0 + tid < r1 ? z[r0 + tid] : 0.0;
  __syncthreads();
  const float *P  = panel + d.panel;
  double      *pp = part + d.bpart + (int64_t)chunk * kNB;
  constexpr int kWarps = kSolveThreads / 32;
  for (int k = warp; k < d.nbk; k += kWarps) {
    const float *col = P + (int64_t)(d.kb + k) * h;
    double       s   = 0.0;
    for (int64_t r = r0 + lane; r < r1; r += 32)
      s += static_cast<double>(col[r]) * zr[r - r0];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) pp[k] = s;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(counter + d.id, 1) == d.bsolve_chunks - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  {
    // Partials of column k: thread (q, k) adds chunks q, q + 4, ...; the
    // four sums are then added in order.
    const int k = tid % kNB, q = tid / kNB;
    double    s = 0.0;
    if (k < d.nbk)
      for (int c = q; c < d.bsolve_chunks; c += 4)
        s += __ldcg(part + d.bpart + (int64_t)c * kNB + k);
    red[q][k] = s;
  }
  __syncthreads();
  if (tid < d.nbk)
    v[tid] = z[d.kb + tid] - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]));
  __syncthreads();
  // Lt[i * kNB + j] = Linv[i][j]
  const double xb = block_upper_apply(linv64t + d.linv, v, d.nbk, red);
  if (tid < d.nbk) {
    z[d.kb + tid]                    = xb;
    x[(int64_t)d.col0 + d.kb + tid] = xb;
  }
}

// ---------------------------------------------------------------------------
void SolveWorkspace::allocate(const Plan &P) {
  release_graph();
  zbuf.resize(std::max<int64_t>(P.S.z_elems, 1) * sizeof(double));
  part.resize(std::max<int64_t>(P.bpart_elems, 1) * sizeof(double));
  counters.resize(std::max<int64_t>(P.ndesc, 1) * sizeof(int32_t));
  xbuf.resize(std::max<int64_t>(P.S.n, 1) * sizeof(double));
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
    const int64_t before = launch_counter();
    ldlt_solve(P, F, ws.xbuf.as<double>(), ws, capture_stream);
    MPIR_CUDA(cudaStreamEndCapture(capture_stream, &g));
    ws.graph_launches = launch_counter() - before;
    launch_counter() = before;
    MPIR_CUDA(cudaGraphInstantiate(&ws.graph, g, 0));
    cudaGraphDestroy(g);
  }
  MPIR_CUDA(cudaMemcpyAsync(ws.xbuf.as<void>(), x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  MPIR_CUDA(cudaGraphLaunch(ws.graph, s));
  launch_counter() += ws.graph_launches;
  MPIR_CUDA(cudaMemcpyAsync(x, ws.xbuf.as<void>(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

void ldlt_solve(const Plan &P, const Numeric &F, double *x, SolveWorkspace &ws,
                cudaStream_t s, int phases) {
  const Symbolic &S  = P.S;
  KernelTimer    &kt = kernel_timer();
  if (S.n == 0) return;
  const float *pan  = F.panel.as<float>();
  const double *lv  = F.linv64.as<double>();
  double      *zbuf = ws.zbuf.as<double>();
  const int    nl   = static_cast<int>(P.levels.size());
  kt.begin(kKcSolveFwd, s);
  for (int t = 0; t < nl && (phases & kForward); t++) {
    const LevelPlan &L = P.levels[t];
    if (L.small_count > 0)
      launch(k_fwd_small, (L.small_count + kWarpsPerCta - 1) / kWarpsPerCta,
                    32 * kWarpsPerCta, 0, s, 
          P.small_list.as<int32_t>() + L.small_begin, L.small_count,
          P.sfirst.as<int64_t>(), P.srowptr.as<int64_t>(), P.slofs.as<int64_t>(),
          P.child_ptr.as<int64_t>(), P.child_list.as<int32_t>(),
          P.srel.as<int32_t>(), P.zofs.as<int64_t>(), pan, x, zbuf);
    if (L.large_count > 0) {
      launch(k_fwd_gather, L.large_count, kSolveThreads, 0, s,
             P.large_list.as<int32_t>() + L.large_begin, P.sfirst.as<int64_t>(),
             P.srowptr.as<int64_t>(), P.child_ptr.as<int64_t>(),
             P.child_list.as<int32_t>(), P.srel.as<int32_t>(), P.zofs.as<int64_t>(),
             P.linv_ofs_d.as<int64_t>(), lv, x, zbuf);
      for (const auto &st : L.steps)
        launch(k_fwd_step, st.fsolve_tiles, kSolveThreads, 0, s, 
            P.steps.as<StepDesc>() + st.begin, st.count, pan, lv, x, zbuf);
    }
  }
  if (phases & kDiagonal)
    launch(k_dscale, static_cast<unsigned>((S.n + 255) / 256), 256, 0, s, 
        S.n, F.Dinv.as<float>(), x);
  kt.end(s);
  if (!(phases & kBackward)) return;
  MPIR_CHECK_LAUNCH();
  kt.begin(kKcSolveBwd, s);
  MPIR_CUDA(cudaMemsetAsync(ws.counters.as<void>(), 0,
                            std::max<int64_t>(P.ndesc, 1) * sizeof(int32_t), s));
  for (int t = nl - 1; t >= 0; t--) {
    const LevelPlan &L = P.levels[t];
    if (L.small_count > 0)
      launch(k_bwd_small, (L.small_count + kWarpsPerCta - 1) / kWarpsPerCta,
                    32 * kWarpsPerCta, 0, s, 
          P.small_list.as<int32_t>() + L.small_begin, L.small_count,
          P.sfirst.as<int64_t>(), P.srowptr.as<int64_t>(), P.srows.as<int32_t>(),
          P.slofs.as<int64_t>(), pan, x);
    if (L.large_count > 0) {
      launch(k_bwd_gather, L.large_count, 256, 0, s, 
          P.large_list.as<int32_t>() + L.large_begin, P.sfirst.as<int64_t>(),
          P.srowptr.as<int64_t>(), P.srows.as<int32_t>(), P.zofs.as<int64_t>(), x,
          zbuf);
      for (size_t q = L.steps.size(); q-- > 0;) {
        const auto &st = L.steps[q];
        launch(k_bwd_step, st.bsolve_chunks, kSolveThreads, 0, s,
               P.steps.as<StepDesc>() + st.begin, st.count, pan, F.linv64t.as<double>(), x,
               zbuf, ws.part.as<double>(), ws.counters.as<int32_t>());
      }
    }
  }
  kt.end(s);
  MPIR_CHECK_LAUNCH();
}


// ---------------------------------------------------------------------------
// QDLDL_solve without device allocation.
//
// For callers that cannot call cudaMalloc: code running while a CUDA stream
// capture is open (allocation is not allowed there), and processes whose
// device memory is handed out entirely by their own pooling allocator.  All
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
// call that uses that device.
void *g_solve_scratch_addr[kNoAllocMaxDevices] = {};
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
  MPIR_CUDA(cudaSetDevice(device));
  if (!g_solve_scratch_addr[device]) {
    void             *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_solve_scratch);
    if (e != cudaSuccess) throw CudaError(e, "cudaGetSymbolAddress(g_solve_scratch)");
    g_solve_scratch_addr[device] = p;
  }
  unsigned char     *base = static_cast<unsigned char *>(g_solve_scratch_addr[device]);
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
    launch(k_fwd_small, (cnt + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, s,
           level + S.level_ptr[t], cnt, sfirst, srowptr, slofs, cptr, clist, srel, zofs, panel,
           xd, zbuf);
  }
  launch(k_dscale, static_cast<unsigned>((n + 255) / 256), 256, 0, s, n, dinv, xd);
  for (int t = nl - 1; t >= 0; t--) {
    const int32_t cnt = static_cast<int32_t>(S.level_ptr[t + 1] - S.level_ptr[t]);
    launch(k_bwd_small, (cnt + kWarpsPerCta - 1) / kWarpsPerCta, 32 * kWarpsPerCta, 0, s,
           level + S.level_ptr[t], cnt, sfirst, srowptr, srows, slofs, panel, xd);
  }
  MPIR_CHECK_LAUNCH();
  MPIR_CUDA(cudaMemcpyAsync(x, xd, n * sizeof(double), cudaMemcpyDeviceToHost, s));
  MPIR_CUDA(cudaStreamSynchronize(s));
  return kOk;
}

}  // namespace mpir
