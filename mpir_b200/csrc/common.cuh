// Shared device-side definitions for the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace mpir {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const char *what)
      : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)),
        code(c) {}
};

#define MPIR_CUDA(call)                                             \
  do {                                                              \
    cudaError_t e__ = (call);                                       \
    if (e__ != cudaSuccess) throw ::mpir::CudaError(e__, #call);    \
  } while (0)

#define MPIR_CHECK_LAUNCH() MPIR_CUDA(cudaGetLastError())

// Host-side count of kernel launches issued by this library (read by the
// benchmark for its launch figure); safe from several host threads.  While a
// thread records a CUDA graph (LaunchCapture), its launches are counted for
// the graph instead, and each replay adds the graph's count.
int64_t launch_total();
void    launch_add(int64_t n);
class LaunchCapture {
 public:
  LaunchCapture();
  ~LaunchCapture();
  LaunchCapture(const LaunchCapture &)            = delete;
  LaunchCapture &operator=(const LaunchCapture &) = delete;
  int64_t count() const { return count_; }
  void    add(int64_t n) { count_ += n; }

 private:
  LaunchCapture *outer_;
  int64_t        count_ = 0;
};

// Launch helper: counts the launch, then issues it.
template <class... KArgs, class... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t s, Args &&...args) {
  launch_add(1);
  kernel<<<grid, block, smem, s>>>(static_cast<KArgs>(args)...);
}


// One block step of one front in the blocked dense partial factorization.
// The front's panel is h x w column-major at `panel` (floats, relative to the
// panel base); its update matrix is (h-w) x (h-w) at `uofs` (relative to the
// update arena, -1 when h == w).  The step eliminates columns
// [kb, kb + nbk) of the panel.
struct StepDesc {
  int64_t panel;
  int64_t uofs;
  int64_t linv;       // nbk x nbk inverse of the unit-lower diagonal block,
                      // column-major with leading dimension kNB
  int32_t h, w, kb, nbk;
  int32_t col0;       // permuted index of the front's first column
  int32_t trsm_tile0; // first TRSM row tile of this desc within the step
  int32_t upd_tile0;  // first update tile of this desc within the step
  int32_t upd_panel_tiles;
  // Packed copy of the front for the tensor-core updates (see PackedFront):
  // float offset of the front's packed rows and pivots, K-groups per row
  // tile, and the packed row of the first off-diagonal row.
  int64_t pk;
  int64_t pd;
  int32_t pk_g;
  int32_t pk_wt;
};

// One large front in the triangular solves.  The forward solve of a level
// runs one CTA per row block of 128 rows of each front (first the diagonal
// row blocks of all fronts, front-major, then the off-diagonal ones); the
// backward solve one CTA per 128-row chunk of the
// off-diagonal rows (partial sums for all columns) and then one CTA per
// column block (front-major, last block first).  CTAs take their work in
// ticket order, so every block they wait for belongs to an earlier ticket.
struct SolveFront {
  int64_t panel;   // panel offset (h x w, column-major)
  int64_t zofs;    // front vector in the solve workspace (h doubles)
  int64_t linv;    // float64 inverse of diagonal block 0 (block b at + b kNB^2)
  int64_t part;    // backward chunk partials (chunks x w doubles)
  int64_t rows;    // the front's row index set at srows[rows ..]
  int64_t gptr;    // row i's child contributions: zbuf[gsrc[e]] for e in
                   // gp[gptr + i] .. gp[gptr + i + 1], in child order
  int32_t h, w, nb;
  int32_t col0;    // permuted index of the front's first column
  int32_t n;       // order of the whole system (stride of the ready copies)
  int32_t chunk0, chunks;  // backward chunk CTAs
  int32_t own0;    // first backward column-block CTA
};

// One work item of the ticketed solve launches: a copy of its front's
// descriptor and its row block (forward) or column block (backward), so a CTA
// reads one record after taking its ticket.
struct SolveItem {
  SolveFront f;
  int32_t    r;
  int32_t    pad;
};

// Packed copy of a large front's L for the tensor-core updates.  Rows are
// renumbered so that the off-diagonal rows start on a 128-row boundary:
// packed row p = r for r < w, p = Wt + (r - w) for r >= w, Wt = w rounded up
// to 128.  Row tile t (packed rows 128t .. 128t+127) holds the columns in
// K-groups of 4; K-group g of row tile t is 2048 contiguous bytes at float
// offset pk + (t * G + g) * 512, in the tensor cores' K-major core-matrix
// layout without swizzle (packed row m of the tile at byte 16m, its 4 columns
// consecutive).  G = ceil(w / 32) * 8, so every stage of 16 or 32 columns is
// one contiguous, 16-byte aligned block.  Positions that hold no value of L
// (rows Wt > p >= w, rows past the last, columns >= w, the diagonal blocks)
// stay zero.  The pivots D of the front's columns are packed beside it at pd
// (G * 4 floats, zero past w), and sign(D) sqrt|D| in a second array at the
// same offsets.
struct PackedFront {
  static constexpr int kRowTile = 128;
  static constexpr int kGroupFloats = 512;  // 128 rows x 4 columns
};

// One GEMM-shaped update of a front, C -= (A D) A^T restricted to N columns:
//   C[r, c] -= sum_{k < K} A[r, k] D[k] A[c, k]   (r < M, c < N, c <= r if lower)
// A is M x K inside a panel (leading dimension lda), D the K pivots at
// D[d_ofs ...], C at c_ofs in the panels or in the update arena.  Used for
// the left-looking block updates of a front's own columns (K = columns
// eliminated so far) and for its update matrix (K = all its columns).  The
// K range may be split across CTAs whose partial tiles go to a workspace and
// are added in split order by a reduction launch.
//
// Rows are counted in the packed numbering of the front (PackedFront): local
// row m of the problem is output row m for m < gap_at, nothing for
// gap_at <= m < gap_at + gap, and output row m - gap beyond.  The columns
// (N <= gap_at) have no gap.
struct GemmProb {
  int64_t a_ofs;   // panel offset of A(0, 0)
  int64_t c_ofs;   // offset of C(0, 0)
  int64_t d_ofs;   // index of D for column 0 of A
  int64_t ws_ofs;  // float offset of the split partials, -1 when unsplit
  int64_t pa, pb;  // packed offsets of the first row tile of A and of B
  int64_t pd;      // packed offset of D for column 0
  int64_t prow;    // floats between consecutive packed row tiles
  int32_t gap_at, gap;
  int32_t lda, ldc;
  int32_t M, N, K;
  int32_t c_in_u;  // C lives in the update arena (else in the panels)
  int32_t lower;
  int32_t splits;
  int32_t ntm, ntiles;  // row tiles; tiles of the (lower) tile pattern
  int32_t tile0;   // first CTA of this problem in its GEMM launch
  int32_t rtile0;  // first CTA of this problem in its reduction launch
  // B converted ahead of the 3xTF32 product (k_convert_b): B D split into
  // tf32 high and low parts, in the packed layout, at float offsets bc (high)
  // and bc_lo (low) of the conversion buffer; btiles row tiles of bgroups
  // K-groups each (row tiles bprow floats apart); cv0 = first CTA of this
  // problem in its conversion launch.
  int64_t bc, bc_lo, bprow;
  int32_t btiles, bgroups, cv0;
};
constexpr int kConvGroups = 8;   // K-groups per conversion CTA (4 per thread)

// Extend-add: the update matrix U_C of a child C (|R_C| x |R_C|, lower
// triangle, column-major with leading dimension |R_C|) is added into its
// parent's front through the child's relative row map (increasing).
struct EaTask {
  int64_t child_u;     // U_C offset in the update arena
  int64_t rel;         // offset of the child's relative row map in srel
  int32_t rc;          // |R_C|
  int32_t pad;
};
// One extend-add CTA: parent columns [c0, c0 + nc), all in the parent's
// panel (c0 + nc <= wp) or all in its update matrix (c0 >= wp), and the
// children that add to them, hits [hit0, hit1) in child order.
struct EaChunk {
  int64_t parent_panel;
  int64_t parent_u;    // -1 when the parent has no update matrix
  int32_t hp, wp;      // parent front height and width
  int32_t c0, nc;
  int32_t hit0, hit1;
};
// Columns [ulo, uhi) of task `task`'s U_C land in the chunk (at most
// kEaChunk of them).
struct EaHit {
  int32_t task, ulo, uhi, pad;
};


// Output row of local packed row m of a problem, -1 inside its gap.
__host__ __device__ __forceinline__ int gemm_out_row(const GemmProb &pb, int m) {
  return m < pb.gap_at ? m : (m < pb.gap_at + pb.gap ? -1 : m - pb.gap);
}

// Device status of one numeric factorization.
struct FactorStatus {
  int32_t zero_pivot;  // smallest column (permuted) with D == 0, or INT_MAX
  int32_t npos;        // number of positive D entries
  int32_t nonfinite;   // 1 if a non-finite D was produced
  int32_t timeout;     // 1 if a bounded device wait ran out
};

constexpr int kSmallThreads = 256;
constexpr int kDiagThreads  = 512;
constexpr int kGemmThreads  = 256;
constexpr int kEaChunk      = 8;     // parent columns per extend-add CTA
constexpr int kSolveRows = 128;        // rows per forward-solve CTA
constexpr int kSolveChunk = 128;       // rows per backward-solve CTA
constexpr int kSolveThreads = 512;     // 4 column quarters x 128 rows
// Fronts of at most this width and height are solved by one warp each
// (column by column); larger ones by the SolveFront launches.
constexpr int kWarpSolveW = 32;
constexpr int kWarpSolveH = 256;

}  // namespace mpir
