// Serving engine behind mpir_server_* (server.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <string>

#include "solver.hpp"

namespace mpir {

struct ServerConfig {
  int     device     = 0;
  int     uf         = kF32;  // factor type of every resident factor
  int     ur         = kF64;  // residual type
  int     workers    = 4;     // concurrent jobs (host threads, one stream each)
  int     max_batch  = 16;    // right-hand sides solved in lockstep
  int     update     = kUpdateDefault;  // trailing-update engine (float32 factors)
  int64_t budget_bytes = int64_t{150} * 1000000000;  // 150 GB
  int64_t max_ir_iterations    = 10;
  int64_t max_gmres_iterations = 10;
  double  tolerance            = 1e-10;
};

// One request: the system (pattern and values, upper CSC, caller order) and
// its right-hand side; every array must stay valid until the request is
// done.  pattern_key names (n, Ap, Ai), values_key the values Ax on it.
struct ServerRequest {
  uint64_t      pattern_key = 0, values_key = 0;
  int64_t       n  = 0;
  const int64_t *Ap = nullptr, *Ai = nullptr;
  const double  *Ax = nullptr, *b = nullptr;
  double        *x  = nullptr;
  int64_t        id = 0;        // set by submit
  double         t_submit = 0;  // set by submit
};

struct ServerResult {
  int64_t     id = 0;
  int         status = 0;
  int         path   = 0;  // 0 resident factor, 1 refactorization, 2 new pattern
  int         batch  = 1;  // right-hand sides solved together with this one
  double      latency_ms = 0, queue_ms = 0, service_ms = 0;
  Report      report{};
  std::string message;
};

struct ServerStats {
  int64_t submitted = 0, completed = 0, failed = 0, refused = 0;
  int64_t analyses = 0, factorizations = 0, solves = 0, batched_solves = 0, batched_rhs = 0;
  int64_t evictions = 0, resident_factors = 0, resident_patterns = 0, queued = 0;
  int64_t bytes_in_use = 0, peak_bytes = 0;
  int64_t analysis_reuses = 0;  // plans rebuilt from a cached host analysis
  int64_t plan_uploads    = 0;  // evicted plans uploaded again from their host tables
  // Worker time (host wall clock, summed over workers) in the host analysis,
  // the plan build and upload, the factorizations (allocation included) and
  // the solves.
  double analysis_ms = 0, plan_ms = 0, factor_ms = 0, solve_ms = 0;
  // Device time (CUDA events) of the factorizations and of the solves.
  double factor_device_ms = 0, solve_device_ms = 0;
  // Parts of factor_ms: a new factor's setup (solver, resident buffers) and
  // the release of its factorization scratch afterwards.
  double setup_ms = 0, trim_ms = 0;
  // Part of plan_ms: copying plans' arrays to the device (builds and uploads).
  double plan_upload_ms = 0;
};

class Server {
 public:
  explicit Server(const ServerConfig &cfg);
  ~Server();
  int64_t     submit(ServerRequest r);
  bool        wait(int64_t id, ServerResult *out);
  void        drain();
  ServerStats stats();

 private:
  struct Impl;
  std::unique_ptr<Impl> impl_;
};

}  // namespace mpir
