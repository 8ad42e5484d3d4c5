// Drop-in Stats for the reference's include/qdldl-luir/stats.hpp: the fields
// LUIR_QDLDL fills (stats.hpp:10-31), filled by the GPU implementation.
#pragma once
#ifndef MPIR_B200_LUIR_STATS_HPP
#define MPIR_B200_LUIR_STATS_HPP

#include <cstdio>
#include <string>

class Stats {
 public:
  Stats() { init(); }
  void init() {
    fact_prec_ = work_prec_ = res_prec_ = "";
    n_ = 0;
    nnz_ = 0;
    time_sym_ = time_num_fact_ = time_solve_ = time_ref_ = 0.0;
    num_refinement_steps_ = 0;
    Lnz_ = 0;
    relative_residual_ = 0.0;
  }
  double get_total_time() { return time_sym_ + time_num_fact_ + time_solve_ + time_ref_; }
  double get_time_num_fact() { return time_num_fact_; }
  int    get_num_refinement_steps() { return num_refinement_steps_; }
  double get_residual() { return relative_residual_; }

  std::string   fact_prec_, work_prec_, res_prec_;
  int           n_;
  long int      nnz_;
  double        time_sym_, time_num_fact_, time_solve_, time_ref_;
  int           num_refinement_steps_;
  unsigned long Lnz_;
  double        relative_residual_;

  void print(const char *str = 0) {
    if (str) std::printf("%s\n", str);
    std::printf("%-20s: %d\n%-20s: %ld\n%-20s: %d\n%-20s: %.2e\n", "n", n_, "nnz", nnz_,
                "refinement steps", num_refinement_steps_, "relative residual",
                relative_residual_);
  }
};

#endif
