// Drop-in GmresLDLIR<UF, UW, UR> for the reference's
// include/MPIR/gmres_ir.hpp:90-315: the same public interface (Compute,
// Solve, SetMaxIRIterations, SetMaxGmresIterations, SetTolerance, defaults
// 10 / 10 / 1e-10), running GMRES-IR preconditioned by a supernodal LDL^T
// factor on the GPU through libmpir_b200 (device from the environment
// variable MPIR_DEVICE, default 0).
//
// Differences a caller can see:
//  * Compute builds a complete LDL^T factor (fill-reducing order, float32
//    factor) where the reference's shipped Compute builds an FGPILU factor;
//    the FGPILU template parameters and ILU_k are accepted and unused.
//  * Compute throws std::runtime_error on invalid input or a zero pivot (the
//    reference's Compute has no error path); Solve returns an empty vector on
//    a size mismatch, as the reference does (gmres_ir.hpp:639-642), and throws
//    on a device error.
//  * Provided precisions: UF = double, float, std::bfloat16_t or
//    std::float16_t; UW = double; UR = double or a double-double type
//    (mpir::double_double, or the QD library's dd_real with MPIR_USE_QD).
//    UF = double (the reference example's instantiation) scales with
//    eps(double) as the reference's Compute does and preconditions with the
//    float32 factor (LastReport().factor_prec = MPIR_F32); the 16-bit types
//    keep L in that type for the solves.  Other combinations throw from
//    Compute.
//  * LastReport() gives the iteration counts and the backward error.
//  * DumpLogText() returns the solver log as JSON text (the schema of the
//    reference's DumpLog, gmres_ir.hpp:305-313); with VERBOSE defined and
//    nlohmann/json available, DumpLog() returns it parsed, as the reference.
#pragma once
#ifndef MPIR_B200_GMRES_IR_HPP
#define MPIR_B200_GMRES_IR_HPP

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#if defined(VERBOSE) && __has_include(<nlohmann/json.hpp>)
#include <nlohmann/json.hpp>
#define MPIR_DROPIN_HAS_JSON 1
#endif

#include "../mpir_b200.h"
#include "fp_concepts.hpp"
#include "ops.hpp"
#include "qdldl.hpp"

namespace mpir_dropin {
template <class T>
constexpr int real_prec() {
  if constexpr (std::is_same_v<T, mpir::double_double>) return MPIR_DD;
#ifdef MPIR_USE_QD
  else if constexpr (std::is_same_v<T, dd_real>) return MPIR_DD;
#endif
  else return prec_of<T>();
}
}  // namespace mpir_dropin

template <typename UF, typename UW, typename UR>
  requires Refinable<UF, UW, UR>
class GmresLDLIR {
  mpir_solver h_          = nullptr;
  std::size_t n_          = 0;
  std::size_t ir_iter_    = 10;
  std::size_t gmres_iter_ = 10;
  double      tol_        = 1e-10;
  mpir_report last_{};

  static void check(int rc, const char *what) {
    if (rc < 0)
      throw std::runtime_error(std::string("GmresLDLIR ") + what + ": " + mpir_last_error());
  }
  void release() {
    if (h_) mpir_solver_destroy(h_);
    h_ = nullptr;
  }

 public:
  GmresLDLIR() = default;
  ~GmresLDLIR() { release(); }
  GmresLDLIR(const GmresLDLIR &)            = delete;
  GmresLDLIR &operator=(const GmresLDLIR &) = delete;
  GmresLDLIR(GmresLDLIR &&o) noexcept { *this = std::move(o); }
  GmresLDLIR &operator=(GmresLDLIR &&o) noexcept {
    if (this != &o) {
      release();
      h_ = o.h_, n_ = o.n_, ir_iter_ = o.ir_iter_, gmres_iter_ = o.gmres_iter_;
      tol_ = o.tol_, last_ = o.last_;
      o.h_ = nullptr;
    }
    return *this;
  }

  template <typename TAx, std::size_t MAX_MATRIX_SIZE = 1 << 21,
            std::size_t MAX_SWEEPS = 10, std::size_t BATCH_SIZE = 4096>
  void Compute(std::vector<std::size_t> Ap, std::vector<std::size_t> Ai,
               std::vector<TAx> Ax, std::size_t /*ILU_k*/) {
    release();
    n_ = Ap.empty() ? 0 : Ap.size() - 1;
    check(mpir_solver_create(&h_, mpir_dropin::prec_of<UF>(), mpir_dropin::prec_of<UW>(),
                             mpir_dropin::real_prec<UR>(), mpir_dropin::device()),
          "create");
    check(mpir_solver_set_max_ir_iterations(h_, static_cast<int64_t>(ir_iter_)), "settings");
    check(mpir_solver_set_max_gmres_iterations(h_, static_cast<int64_t>(gmres_iter_)), "settings");
    check(mpir_solver_set_tolerance(h_, tol_), "settings");
    std::vector<int64_t> ap(Ap.begin(), Ap.end()), ai(Ai.begin(), Ai.end());
    std::vector<double>  ax(Ax.size());
    for (std::size_t i = 0; i < Ax.size(); i++) ax[i] = static_cast<double>(Ax[i]);
    check(mpir_solver_compute(h_, static_cast<int64_t>(n_), ap.data(), ai.data(), ax.data()),
          "Compute");
  }

  std::vector<UW> Solve(const std::vector<UW> &b) {
    if (!h_ || b.size() != n_) return {};
    std::vector<double> bd(b.begin(), b.end()), xd(n_);
    check(mpir_solver_solve(h_, bd.data(), xd.data(), &last_), "Solve");
    return std::vector<UW>(xd.begin(), xd.end());
  }

  void SetMaxIRIterations(std::size_t n) {
    ir_iter_ = n;
    if (h_) check(mpir_solver_set_max_ir_iterations(h_, static_cast<int64_t>(n)), "settings");
  }
  void SetMaxGmresIterations(std::size_t n) {
    gmres_iter_ = n;
    if (h_) check(mpir_solver_set_max_gmres_iterations(h_, static_cast<int64_t>(n)), "settings");
  }
  void SetTolerance(UR tol) {
    tol_ = static_cast<double>(tol);
    if (h_) check(mpir_solver_set_tolerance(h_, tol_), "settings");
  }

  const mpir_report &LastReport() const { return last_; }

  // The log of the solves since the previous call, as JSON text; clears it.
  std::string DumpLogText() {
    if (!h_) return "{}";
    int64_t len = 0;
    check(mpir_solver_dump_log(h_, nullptr, 0, &len), "DumpLog");
    std::string out(static_cast<size_t>(len), '\0');
    check(mpir_solver_dump_log(h_, out.data(), len, &len), "DumpLog");
    out.resize(static_cast<size_t>(len > 0 ? len - 1 : 0));
    return out;
  }
#ifdef MPIR_DROPIN_HAS_JSON
  nlohmann::json DumpLog() { return nlohmann::json::parse(DumpLogText()); }
#endif
};

#endif
