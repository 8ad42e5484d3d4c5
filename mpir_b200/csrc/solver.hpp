// GMRES-IR solver object behind the C ABI: one analysed pattern, one numeric
// factor, the GMRES basis and the refinement vectors, all on one device.
#pragma once
#include <memory>
#include <string>
#include <vector>
#include <stdexcept>

#include "engine.hpp"
#include "solve.hpp"
#include "vec.hpp"

namespace mpir {

enum Prec : int { kF64 = 0, kF32 = 1, kBF16 = 2, kF16 = 3, kDD = 4 };
// Trailing-update engines a float32 factor may take (mpir_solver_set_update).
enum UpdateEngine : int { kUpdateDefault = 0, kUpdateTF32x3 = 1, kUpdateBF16x3 = 2 };

// A bounded device wait of the triangular solves ran out (status -5).
struct WaitTimeout : std::runtime_error {
  WaitTimeout() : std::runtime_error("a bounded device wait of the triangular solves ran out") {}
};

struct Report {
  int32_t status           = 0;
  int32_t ir_iterations    = 0;
  int32_t gmres_iterations = 0;
  int32_t precond_applies  = 0;
  int32_t spmv_count       = 0;
  int32_t reorth_count     = 0;
  int32_t stop_reason      = 0;  // 0 max iterations, 1 small update,
                                 // 2 stagnation, 3 exact residual
  int32_t factor_prec      = 0;  // type the factor is stored and applied in
  double  residual_norm    = 0;
  double  backward_error   = 0;
  double  factor_ms        = 0;
  double  solve_ms         = 0;
};

// One refinement step and one solve in the solver log (the fields of the
// reference's VERBOSE log, gmres_ir.hpp:539-632).
struct IrIter {
  int64_t iteration;
  double  residual, d_norm, timestamp_ms, inner_time_ms;
};
struct IrEvent {
  double              initial_residual = 0;
  std::vector<IrIter> iterations;
  int                 stop_reason      = 0;
  int64_t             total_iterations = 0;
  double              total_time_ms    = 0;
};

class Solver {
 public:
  Solver(int uf, int uw, int ur, int device);
  ~Solver();

  int  device;
  int  uf, uw, ur;
  int64_t ir_iter    = 10;    // gmres_ir.hpp:113-114
  int64_t gmres_iter = 10;    // gmres_ir.hpp:115-116 (clamped to n on use)
  double  tol        = 1e-10; // gmres_ir.hpp:117
  int     update_engine = kUpdateDefault;  // see set_update_engine
  // Trailing-update engine of a float32 factor (UpdateEngine); takes effect
  // at the next factorization.
  void set_update_engine(int engine);

  // Host entry points (caller arrays on the host, caller order).
  int analyze(int64_t n, const int64_t *Ap, const int64_t *Ai, const double *Ax,
              int ordering);
  // Take an analysed pattern built elsewhere (shared with other solvers of
  // the same pattern) and allocate this solver's factor and workspaces.
  void adopt(std::shared_ptr<Plan> P);
  std::shared_ptr<Plan> shared_plan() const { return plan_; }
  // Device memory this solver holds beyond its plan, and what adopt() plus
  // one batch of `width` right-hand sides would take for plan P.
  size_t device_bytes() const;
  // Device bytes that solving `width` right-hand sides in lockstep would add
  // to what this solver holds (0 if its batch buffers already fit).
  size_t batch_growth(int width) const;
  static size_t bytes_for(const Plan &P, int64_t gmres_iter, int width, int uf = kF32);
  int factor(const double *Ax);
  int solve(const double *b, double *x, Report *rep);
  // Device entry points (caller arrays already on this device).
  int factor_device(const double *d_Ax);
  int solve_device(const double *d_b, double *d_x, Report *rep);
  // nrhs GMRES-IR solves in lockstep (gmres_batch.cu): B and X hold nrhs
  // vectors of length n (column-major, caller order, device); every
  // preconditioner application takes all of them at once.  reps: nrhs
  // reports (NULL allowed).  nrhs <= kMaxBatch.
  int solve_batch_device(int nrhs, const double *d_B, double *d_X, Report *reps);
  int solve_batch(int nrhs, const double *B, double *X, Report *reps);
  // X (n x nrhs, column-major, the solver's permuted and scaled order,
  // device) <- (L D L^T)^{-1} X with the current factor: one vector by the
  // single-vector kernels, several by the several-vector kernels.
  void precond_device(int nrhs, double *d_X);
  static constexpr int kMaxBatch = 16;
  // The type the factor is computed and applied in (a double factor type is
  // served by the float32 factor).
  int applied_prec() const { return uf == kF64 ? kF32 : uf; }
  // Plain iterative refinement with the factor (LUIR_QDLDL); host and
  // device vectors.
  int luir(const double *b, double *x, int maxiter, Report *rep);
  // r = b - A x on the original matrix (caller order, host vectors), in
  // float64 or, with dd, in double-double rounded to float64; returns
  // max|r|.  Needs the values of a successful factorization.
  double residual(const double *b, const double *x, double *r, bool dd);
  int luir_device(const double *d_b, double *d_x, int maxiter, Report *rep);
  // The log of the solves since the last call, as JSON (GmresLDLIR::DumpLog).
  std::string dump_log();

  void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
  // Test controls of the bounded waits (SolveCtl): 2^poll_log2 polls per
  // wait (0: the default), and the work item of the forward block solves
  // whose result is not published (-1: none).  For failure tests only.
  void set_wait_controls(int poll_log2, int withhold_item);
  cudaStream_t stream() const { return stream_; }

  bool analyzed() const { return plan_ != nullptr; }
  const Plan &plan() const {
    if (!plan_) throw std::logic_error("no analysed pattern");
    return *plan_;
  }
  const Numeric &numeric() const { return num_; }
  // Release the factorization-only buffers of the current factor (see
  // Numeric::trim); the next factor() allocates them again.
  void trim() { num_.trim(); }
  // Factor groups (group.cu): the factorization of the values in this
  // solver's own value buffer recorded as a graph (scratch allocated first),
  // and the status check after a launch that ran it.
  cudaGraph_t record_factor(int64_t *launches);
  double     *values_device();
  int         finish_recorded_factor(double ms);
  double last_factor_ms = 0;
  int64_t last_npos     = 0;

 private:
  void precond_gmres(const double *b, double *res, Report &st);
  void ensure_vectors();
  // Batched GMRES (gmres_batch.cu): vectors of the batch k*n apart inside
  // blocks of width bw_ (n * bw_ doubles per block).
  void ensure_batch(int width);
  void precond_gmres_batch(int nb, const double *b, double *res, std::vector<Report> &st,
                           const std::vector<int32_t> &active);
  void multi_apply(double *block);

  cudaStream_t          own_stream_ = nullptr, stream_ = nullptr;
  std::shared_ptr<Plan> plan_;
  Numeric               num_;
  SolveWorkspace        ws_;
  VecOps                vec_;
  DeviceBuffer          V_, bs_, bp_, ADp_, x_, r_, t_, d_, hd_, y_, hb_, hx_;
  int64_t               vec_m_ = -1;
  // Batch state: width, basis and vectors, host staging of the per-vector
  // scalars (pinned), the several-vector solve workspace.
  int                   bw_ = 0;
  int64_t               bm_ = -1;
  VecOps                vecb_;
  MultiSolveWorkspace   mws_;
  DeviceBuffer          bV_, bbs_, bbp_, bx_, br_, bt_, bd_, bhd_, by_, bfac_, bact_, bkq_, bin_,
                        bout_, bpre_;
  double               *hpin_ = nullptr;  // pinned host scalars (fac, y, act, kq)
  size_t                hpin_bytes_ = 0;
  static constexpr int  kStageSlots = 16;
  int                   stage_next_ = 0;
  // The next staging slot (2 * bw_ doubles) for an upload of per-vector
  // scalars; slots are reused after kStageSlots uploads, and the batched
  // solve synchronises its stream at least once in fewer uploads than that.
  double *stage_slot() {
    double *p   = hpin_ + static_cast<size_t>(stage_next_) * 2 * bw_;
    stage_next_ = (stage_next_ + 1) % kStageSlots;
    return p;
  }
  int32_t               wait_ctl_[2] = {0, 0};  // SolveCtl words 1-2 (set_wait_controls)
  cudaEvent_t           ev0_ = nullptr, ev1_ = nullptr;
  std::vector<IrEvent>  log_;
};

double eps_of(int prec);

}  // namespace mpir
