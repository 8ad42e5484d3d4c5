// Factor groups (group.cu): several value sets on one analysed pattern,
// refactorized by one graph launch.
#pragma once
#include <memory>
#include <vector>

#include "solver.hpp"

namespace mpir {

class FactorGroup {
 public:
  FactorGroup(Solver &base, int k);
  ~FactorGroup();
  FactorGroup(const FactorGroup &)            = delete;
  FactorGroup &operator=(const FactorGroup &) = delete;
  int     size() const { return static_cast<int>(members_.size()); }
  Solver &member(int i) { return *members_.at(i); }
  // Values of member i at Ax_host + i * stride (host); one launch for all.
  // npos (NULL or size() entries): each factor's positive pivots or status.
  int    factor(const double *Ax_host, int64_t stride, int64_t *npos);
  double last_ms() const { return last_ms_; }

 private:
  void                                 record();
  int                                  device_;
  std::vector<std::unique_ptr<Solver>> members_;
  cudaStream_t                         stream_ = nullptr;
  cudaGraphExec_t                      exec_   = nullptr;
  cudaEvent_t                          ev0_ = nullptr, ev1_ = nullptr;
  int64_t                              launches_ = 0;
  double                               last_ms_  = 0;
};

}  // namespace mpir
