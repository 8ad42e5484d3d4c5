// Device-resident plan (per pattern) and numeric factor (per value set).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"
#include "symbolic.hpp"

namespace mpir {

// Device memory (memory.cu).  An allocation on the current device, usable
// from every stream once device_alloc returns; m records its device, its
// source (the stream-ordered pool, or cudaMalloc with a cache of idle
// blocks) and its capacity.  A free waits for nothing (the caller's work on
// the buffer has completed).  device_free_bytes counts what the pool and
// the cache hold idle as free; device_cache_flush returns the cache's blocks
// of a device; set_thread_pool chooses the calling thread's source.
struct DevMem {
  int    device = 0;
  bool   pooled = false;
  size_t cap    = 0;
};
void  *device_alloc(size_t bytes, DevMem *m);
void   device_free(void *p, const DevMem &m);
size_t device_free_bytes(int device);
void   device_cache_flush(int device);
// Zeroes a buffer of the current device, complete for every stream on return.
void   device_zero(void *p, size_t bytes);
void   set_thread_pool(bool pool);
// Pinned host memory with a cache of freed blocks (by size).
void  *pinned_alloc(size_t bytes);
void   pinned_free(void *p, size_t bytes);

// Owning device allocation.
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { resize(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer &)            = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), bytes_(o.bytes_), m_(o.m_) {
    o.p_     = nullptr;
    o.bytes_ = 0;
  }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
      release();
      p_       = o.p_;
      bytes_   = o.bytes_;
      m_       = o.m_;
      o.p_     = nullptr;
      o.bytes_ = 0;
    }
    return *this;
  }
  void resize(size_t bytes) {
    release();
    if (bytes) p_ = device_alloc(bytes, &m_);
    bytes_ = bytes;
  }
  void release() {
    if (p_) device_free(p_, m_);
    p_     = nullptr;
    bytes_ = 0;
  }
  template <class T>
  T *as() const {
    return static_cast<T *>(p_);
  }
  size_t bytes() const { return bytes_; }

 private:
  void  *p_     = nullptr;
  size_t bytes_ = 0;
  DevMem m_;
};

template <class T>
DeviceBuffer upload(const std::vector<T> &v, cudaStream_t s) {
  DeviceBuffer b(v.size() * sizeof(T));
  if (!v.empty())
    MPIR_CUDA(cudaMemcpyAsync(b.as<void>(), v.data(), v.size() * sizeof(T),
                              cudaMemcpyHostToDevice, s));
  return b;
}

// Launch lists of one etree level.
struct LevelPlan {
  int32_t small_begin = 0, small_count = 0;  // into small list
  int32_t large_begin = 0, large_count = 0;  // into large list
  // Extend-add CTAs (EaChunk) of the level's large parents: the columns of
  // their panels [ea_begin[0], + ea_count[0]) before the fronts are
  // factored, those of their update matrices [ea_begin[1], + ea_count[1])
  // after the products that define them.
  int32_t ea_begin[2] = {0, 0}, ea_count[2] = {0, 0};
  struct Step {
    int32_t begin, count, trsm_tiles, upd_tiles;
    // left-looking update of this block column before its diagonal block
    int32_t ll_begin, ll_count, ll_tiles, ll_rtiles, ll_convs;
  };
  std::vector<Step> steps;
  // update matrices of the level's large fronts, after their last step
  int32_t u_begin = 0, u_count = 0, u_tiles = 0, u_rtiles = 0, u_convs = 0;
  // Solve: large fronts' gather list = large list; small fronts handled by
  // one warp each; large fronts by the SolveFront launches: fronts
  // [sf_begin, sf_begin + sf_count), forward CTAs, backward chunk CTAs and
  // backward column-block CTAs.
  int32_t sf_begin = 0, sf_count = 0;
  int32_t sw_begin = 0, sw_count = 0;  // warp-solved fronts (swarp list)
  int32_t fwd_items = 0, bwd_chunk_items = 0, bwd_owner_items = 0;
  // Offsets of the level's work items (Plan::fwd_item, own_item) and of its
  // chunk -> front map (front index within the level).
  int64_t fwd_map0 = 0, chunk_map0 = 0, own_map0 = 0;
};

// Everything the kernels need about one analysed pattern.
class Plan {
 public:
  Symbolic               S;
  std::vector<LevelPlan> levels;
  int64_t                linv_elems = 0;
  int64_t                nnz_full   = 0;
  int64_t                ndesc      = 0;  // step descriptors in total
  int64_t                spart_elems = 0; // backward chunk partials (doubles)
  // Solve synchronisation words (2 tickets per level) and whether any front
  // takes the ticketed block kernels; reset before every solve.
  int64_t                nblock_fronts = 0, sync_elems = 0;
  double                 update_flops = 0, trsm_flops = 0, panel_read_bytes = 0;
  // Pattern arrays on the device.
  DeviceBuffer amap, arow, acol, diag_pos, Kp, Kj, Ksrc;
  DeviceBuffer sfirst, srowptr, srows, srel, slofs, uofs, zofs, child_ptr,
      child_list, perm;
  DeviceBuffer ea_chunks, ea_hits;  // EaChunk / EaHit, see LevelPlan::ea_begin
  DeviceBuffer small_list, large_list, steps, ea_tasks, linv_ofs_d, gemm_probs,
      solve_fronts, swarp_list, sblock_list, gp, gsrc, fwd_item, chunk_map, own_item;
  int64_t      ws_elems = 0;  // split-K partial tiles (floats)
  int64_t      bconv_elems = 0;  // converted B operands of the largest launch (floats)
  std::vector<int32_t> h_small, h_large;
  // Solve lists: fronts solved by one warp, fronts with a SolveFront entry
  // (same order as the SolveFront array).
  std::vector<int32_t> h_swarp, h_sblock;
  std::vector<int64_t> linv_ofs;  // per supernode, -1 for small fronts
  // Packed fronts (PackedFront) of the large fronts: float offsets of the
  // packed rows and of the packed pivots per supernode (-1 for small
  // fronts), and the totals.
  std::vector<int64_t> pk_ofs, pd_ofs;
  int64_t              pk_elems = 0, pd_elems = 0;

  // The host tables and, unless upload is false, their device copies.
  void build(Symbolic &&sym, cudaStream_t s, bool upload = true);
  // Device bytes upload_all() takes.
  size_t upload_bytes() const;
  // Device memory the plan holds.
  size_t device_bytes() const;
  // Frees the device arrays (the host arrays stay) / uploads them again.
  void release_device();
  void upload_all(cudaStream_t s);
  bool   on_device = false;
  double upload_ms = 0;  // host wall time of the last upload_all
  // Host copies of the launch and solve tables that build() computes.
  struct HostArrays {
    std::vector<StepDesc>   descs;
    std::vector<EaTask>     tasks;
    std::vector<EaChunk>    chunks;
    std::vector<EaHit>      hits;
    std::vector<int32_t>    chunk_map;
    std::vector<GemmProb>   probs;
    std::vector<SolveFront> sfronts;
    std::vector<int64_t>    gp, gsrc;
    std::vector<SolveItem>  fwd_item, own_item;
  } host_;
  bool is_large(int64_t J) const { return S.h(J) > kSmallFront; }
  // Packed-front geometry (PackedFront): first packed row of the
  // off-diagonal rows, K-groups per row tile, row tiles.
  int64_t pk_wt(int64_t J) const { return (S.w(J) + 127) / 128 * 128; }
  int64_t pk_groups(int64_t J) const { return (S.w(J) + 31) / 32 * 8; }
  int64_t pk_tiles(int64_t J) const { return (pk_wt(J) + S.h(J) - S.w(J) + 127) / 128; }
};

// Numeric factor of one value set on a plan.
class Numeric {
 public:
  // linv: float32 inverses of the diagonal blocks (the factor's panel solve);
  // linv64: the same inverses in float64 (the triangular solves), column-major;
  // linv64t: row-major copy of linv64 (the backward solve).
  DeviceBuffer panel, uarena, linv, linv64, linv64t, D, Dinv, status, ws;
  // Packed fronts for the tensor-core updates: rows (pack) and pivots
  // (packd: D, then sign(D) sqrt|D|, Plan::pd_elems floats each).
  DeviceBuffer pack, packd;
  // 16-bit copy of the panels for the solves of the bfloat16 / float16
  // tiers (store_prec 2 / 3; 1 = the solves read the float32 panels).
  DeviceBuffer panel16;
  int          store_prec = 1;
  int          solve_prec() const { return panel16.bytes() ? store_prec : 1; }
  // B operands converted ahead of the 3xTF32 updates (GemmProb::bc).
  DeviceBuffer bconv;
  DeviceBuffer AD, Axs, Kval, Korig, Ax;
  double       eps_uf = 0;
  bool         valid  = false;
  bool         nonfinite = false;  // a pivot of the last factor is not finite
  // Captured factorization (run_graph) and what it was captured for.
  cudaGraphExec_t graph          = nullptr;
  const double   *graph_ax       = nullptr;
  double          graph_eps      = 0;
  int             graph_mode     = -2;
  int64_t         graph_launches = 0;
  bool            ran_plain      = false;  // a plain factorization since the graph was released
  // Trailing-update engine: -1 float32 SIMT, 0 bfloat16 tensor cores,
  // 1 3xTF32 tensor cores, 2 float16 tensor cores, 3 3xBF16 tensor cores.
  // The panel solves run on the tensor cores (3xTF32) with every tensor-core
  // engine, on the SIMT units with the SIMT engine or MPIR_TRSM=simt.
  int          update_mode = -1;

  void allocate(const Plan &P);
  // The buffers only the factorization uses (update arena, packed fronts,
  // split partials, converted operands, float32 block inverses, the values):
  // trim() releases them once a factor is done (a resident factor keeps what
  // the solves read: L, the float64 block inverses, D, K), ensure_scratch()
  // brings them back before the next factorization.
  void ensure_scratch(const Plan &P);
  void trim();
  bool has_scratch = false;
  // Device memory allocate() takes for P, and what this factor holds.
  static size_t bytes_for(const Plan &P, int store_prec = 1);
  size_t        device_bytes() const;
  // Scale the caller's values (device, caller order), assemble and factor.
  void run(const Plan &P, const double *d_Ax, double eps_uf, cudaStream_t s);
  // The same, replayed from a CUDA graph captured on capture_stream at the
  // first call (and again when d_Ax, eps_uf or the update engine change); the
  // plain launches when the per-class kernel timer is on.
  void run_graph(const Plan &P, const double *d_Ax, double eps_uf, cudaStream_t s,
                 cudaStream_t capture_stream);
  void release_graph();
  // Records the whole factorization of d_Ax on capture_stream as a graph
  // (not run, not instantiated; the caller owns it); *launches receives the
  // kernel launches it holds.
  cudaGraph_t record(const Plan &P, const double *d_Ax, double eps, cudaStream_t capture_stream,
                     int64_t *launches);
  ~Numeric() { release_graph(); }
  // Reads the status; returns #positive D, -1 on a zero pivot or -5 when a
  // bounded device wait ran out.
  int64_t result(cudaStream_t s, int32_t *zero_col = nullptr,
                 bool *nonfinite = nullptr) const;
};

// Tensor-core GemmProb updates from the packed fronts (mode 0 bfloat16,
// 1 3xTF32, 2 float16).  packs = the sign(D) sqrt|D| array.
void launch_gemm_tc(int mode, const GemmProb *probs, int nprob, int tiles, const float *pack,
                    const float *packd, const float *packs, const float *bconv, float *panel,
                    float *uarena, float *ws, FactorStatus *st, cudaStream_t s);
int  tc_gemm_smem_bytes(int mode);
// Converts the B operands of a launch's problems for the 3xTF32 product.
void launch_convert_b(const GemmProb *probs, int nprob, int convs, const float *pack,
                      const float *packd, float *bconv, cudaStream_t s);
// Tensor-core GEMM CTAs resident per SM (shared-memory bound).
int  tc_ctas_per_sm();
// Panel solves of a block step on the tensor cores (3xTF32), one CTA per
// 128-row tile; the same outputs as k_step_gemm<true>.
void launch_trsm_tc(const StepDesc *descs, int ndesc, int tiles, float *panel, const float *linv,
                    const float *Dinv, float *pack, FactorStatus *st, cudaStream_t s);
// Streaming multiprocessors of a B200.
constexpr int kSMs = 148;

// Kernel-class timer used by the benchmark's roofline figures.
struct KernelTimer {
  bool                      enabled = false;
  std::vector<cudaEvent_t>  ev;
  std::vector<int>          cls;
  void                      begin(int c, cudaStream_t s);
  void                      end(cudaStream_t s);
  void                      reset();
  // Total milliseconds and launches per class (after a synchronize).
  void collect(double *ms, int64_t *count, int nclass);
};
enum KernelClass : int {
  kKcSmallFront = 0,
  kKcDiag,
  kKcTrsm,
  kKcUpdate,
  kKcExtendAdd,
  kKcZero,
  kKcScatter,
  kKcSolveFwd,
  kKcSolveBwd,
  kKcSpmv,
  kKcVec,
  kKcReduce,
  kKcCount
};
KernelTimer &kernel_timer();

}  // namespace mpir
