// Triangular-solve workspace and entry point (solve.cu).
#pragma once
#include <string>
#include <utility>

#include "engine.hpp"

namespace mpir {

// A second stream and two events, created on first use on the current
// device: a level's warp-solved fronts run on it beside the same level's
// block fronts (neither reads what the other writes), inside a recorded
// graph as a parallel branch.
class SideStream {
 public:
  SideStream() = default;
  SideStream(const SideStream &)            = delete;
  SideStream &operator=(const SideStream &) = delete;
  SideStream(SideStream &&o) noexcept { swap(o); }
  SideStream &operator=(SideStream &&o) noexcept {
    if (this != &o) {
      reset();
      swap(o);
    }
    return *this;
  }
  ~SideStream() { reset(); }
  // The side stream, after everything issued to s so far.
  cudaStream_t fork(cudaStream_t s);
  // Work issued to s from here on runs after everything issued to the side.
  void join(cudaStream_t s);

 private:
  void swap(SideStream &o) {
    std::swap(st_, o.st_);
    std::swap(fork_, o.fork_);
    std::swap(join_, o.join_);
  }
  void         reset();
  cudaStream_t st_   = nullptr;
  cudaEvent_t  fork_ = nullptr, join_ = nullptr;
};

struct SolveWorkspace {
  DeviceBuffer zbuf;      // front vectors, zofs layout (doubles)
  DeviceBuffer part;      // backward chunk partial sums (doubles)
  DeviceBuffer sync;      // tickets (Plan::sync_elems int32)
  DeviceBuffer ready;     // block results for the CTAs that wait on them (n
                          // doubles, the pending marker until written)
  DeviceBuffer err;       // SolveCtl: err = 1 when a bounded wait gave up, then
                          // the test controls of the waits (solve_dev.cuh)
  DeviceBuffer xbuf;      // fixed vector the captured solve works on
  cudaGraphExec_t graph = nullptr;  // captured L D L^T solve (all phases)
  int64_t graph_launches = 0;       // kernels one replay runs
  SideStream side;
  void allocate(const Plan &P);
  void release_graph();
  ~SolveWorkspace() { release_graph(); }
};

// Phases of the solve, combinable as bits.
enum SolvePhase : int { kForward = 1, kDiagonal = 2, kBackward = 4, kAllPhases = 7 };

// x (permuted order, float64, device) <- (L D L^T)^{-1} x, or the phases
// selected: (L+I)^{-1} x, Dinv .* x, (L+I)^{-T} x (qdldl.hpp:362-432).
void ldlt_solve(const Plan &P, const Numeric &F, double *x, SolveWorkspace &ws,
                cudaStream_t s, int phases = kAllPhases);

// The same full solve replayed from a CUDA graph captured on first use on
// `capture_stream` (a non-default stream) and launched on `s`; x is copied
// into and out of the workspace vector the graph was captured on.
void ldlt_solve_graph(const Plan &P, const Numeric &F, double *x, SolveWorkspace &ws,
                      cudaStream_t s, cudaStream_t capture_stream);

// Workspace of the several-vector solves (solve_multi.cu) for one width.
// An instantiated CUDA graph, destroyed with its owner (movable).
struct GraphExec {
  cudaGraphExec_t g = nullptr;
  GraphExec()       = default;
  GraphExec(const GraphExec &) = delete;
  GraphExec &operator=(const GraphExec &) = delete;
  GraphExec(GraphExec &&o) noexcept : g(o.g) { o.g = nullptr; }
  GraphExec &operator=(GraphExec &&o) noexcept {
    if (this != &o) {
      reset();
      g   = o.g;
      o.g = nullptr;
    }
    return *this;
  }
  ~GraphExec() { reset(); }
  void reset() {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
};

struct MultiSolveWorkspace {
  int          nr = 0;  // vectors per application (4, 8 or 16)
  DeviceBuffer zbuf, part, sync, ready, err;
  // The application recorded as a graph on the fixed block xbuf (n x nr).
  DeviceBuffer xbuf;
  GraphExec    graph;
  int64_t      graph_launches = 0;
  SideStream   side;
  void         allocate(const Plan &P, int width);
  static size_t bytes_for(const Plan &P, int width);
};

// Vectors per several-vector application for nrhs right-hand sides (the
// kernels are instantiated for 4, 8 and 16; unused columns are zero).
int multi_width(int nrhs);

// X (n x width, column-major, leading dimension n, permuted order, float64,
// device) <- (L D L^T)^{-1} X, or the phases selected, for all width columns
// at once (solve_multi.cu).
void ldlt_solve_multi(const Plan &P, const Numeric &F, double *X, int width,
                      MultiSolveWorkspace &ws, cudaStream_t s, int phases = kAllPhases);
// The same full application replayed from a graph recorded on first use on
// capture_stream (X copied into and out of the workspace block): one launch
// instead of a few per level, which is most of an application's cost for
// small systems.  The plain launches while the per-class kernel timer is on.
void ldlt_solve_multi_graph(const Plan &P, const Numeric &F, double *X, int width,
                            MultiSolveWorkspace &ws, cudaStream_t s,
                            cudaStream_t capture_stream);

// QDLDL_solve (float32 factor, float64 x, host arrays) whose device data
// lives in a fixed file-scope array instead of allocated memory; see
// mpir_qdldl_solve_noalloc in include/mpir_b200.h.  Returns a status and a
// message in err.
int qdldl_solve_noalloc(int64_t n, const int64_t *Lp, const int64_t *Li, const float *Lx,
                        const float *Dinv, double *x, int device, std::string &err);

}  // namespace mpir
