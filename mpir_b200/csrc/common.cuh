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
// benchmark for its launch figure).
int64_t &launch_counter();
#define MPIR_COUNT(n) (::mpir::launch_counter() += (n))

// Launch helper: counts the launch, then issues it.
template <class... KArgs, class... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t s, Args &&...args) {
  ++launch_counter();
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
  // Solve fields: the front's vector at zofs (h doubles) in the solve
  // workspace; forward row tiles and backward row chunks of this desc within
  // the step; backward partial sums at bpart (chunks x kNB doubles); the
  // desc's global index (for its completion counter).
  int64_t zofs;
  int64_t bpart;
  int32_t fsolve_tile0;
  int32_t bsolve_chunk0;
  int32_t bsolve_chunks;
  int32_t id;
};

// One GEMM-shaped update of a front, C -= (A D) A^T restricted to N columns:
//   C[r, c] -= sum_{k < K} A[r, k] D[k] A[c, k]   (r < M, c < N, c <= r if lower)
// A is M x K inside a panel (leading dimension lda), D the K pivots at
// D[d_ofs ...], C at c_ofs in the panels or in the update arena.  Used for
// the left-looking block updates of a front's own columns (K = columns
// eliminated so far) and for its update matrix (K = all its columns).  The
// K range may be split across CTAs whose partial tiles go to a workspace and
// are added in split order by a reduction launch.
struct GemmProb {
  int64_t a_ofs;   // panel offset of A(0, 0)
  int64_t c_ofs;   // offset of C(0, 0)
  int64_t d_ofs;   // index of D for column 0 of A
  int64_t ws_ofs;  // float offset of the split partials, -1 when unsplit
  int32_t lda, ldc;
  int32_t M, N, K;
  int32_t c_in_u;  // C lives in the update arena (else in the panels)
  int32_t lower;
  int32_t splits;
  int32_t ntm, ntiles;  // row tiles; tiles of the (lower) tile pattern
  int32_t tile0;   // first CTA of this problem in its GEMM launch
  int32_t rtile0;  // first CTA of this problem in its reduction launch
};

// Extend-add task: add the lower triangle of child C's update matrix into
// its parent's front, CTA-chunked by columns of U_C.
struct EaTask {
  int64_t child_u;     // U_C offset in the update arena
  int64_t parent_panel;
  int64_t parent_u;    // -1 when the parent has no update matrix
  int64_t rel;         // offset of the child's relative row map in srel
  int32_t rc;          // |R_C|
  int32_t hp, wp;      // parent front height and width
  int32_t chunk0;      // first column chunk of this task within the launch
};

// Zero-fill segment (float offset into the update arena, length).
struct Segment {
  int64_t ofs, len;
  int64_t chunk0;  // first chunk of this segment within the launch
};

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
constexpr int kEaChunk      = 8;     // U_C columns per extend-add CTA
constexpr int64_t kZeroChunk = 16384;  // floats per zero-fill CTA
constexpr int kSolveRows = 128;        // rows per forward-solve CTA
constexpr int kSolveChunk = 128;       // rows per backward-solve CTA
constexpr int kSolveThreads = 512;     // 4 column quarters x 128 rows

}  // namespace mpir
