// Drop-in LUIR_QDLDL for the reference's include/qdldl-luir/luir.hpp:33-241:
// the same template and arguments; the factorization and the plain
// iterative refinement run on the GPU through libmpir_b200
// (mpir_luir_qdldl; device from MPIR_DEVICE, default 0).
//
// Provided: FACTPREC = float, std::bfloat16_t or std::float16_t (the factor
// is computed with float32 accumulation and rounded to FACTPREC where the
// reference stores FACTPREC), RESPREC = WORKPREC = XPREC = double.  The
// reference prints a message and calls exit(-1) on an input that is not
// upper triangular; this version throws std::runtime_error with the
// library's message instead, for that and for any device error.
#pragma once
#ifndef MPIR_B200_LUIR_HPP
#define MPIR_B200_LUIR_HPP

#include <stdexcept>
#include <string>
#include <type_traits>
#include <typeinfo>

#include "../MPIR/qdldl.hpp"
#include "stats.hpp"

template <typename FACTPREC, typename RESPREC, typename WORKPREC, typename XPREC,
          typename INT>
void LUIR_QDLDL(INT n, const INT *Ap, const INT *Ai, const WORKPREC *Ax, const WORKPREC *b,
                XPREC *x, Stats *stats, int maxiter = 10) {
  static_assert(std::is_same_v<WORKPREC, double> && std::is_same_v<XPREC, double> &&
                    std::is_same_v<RESPREC, double>,
                "provided: RESPREC = WORKPREC = XPREC = double");
  constexpr int fp = mpir_dropin::prec_of<FACTPREC>();
  static_assert(fp == MPIR_F32 || fp == MPIR_BF16 || fp == MPIR_F16,
                "provided: FACTPREC = float, std::bfloat16_t, std::float16_t");
  const int64_t                     nnz = static_cast<int64_t>(Ap[n] - Ap[0]);
  mpir_dropin::I64View<INT>         p(Ap, static_cast<int64_t>(n) + 1), i(Ai, nnz);
  mpir_report                       rep{};
  const int rc = mpir_luir_qdldl(static_cast<int64_t>(n), p.p, i.p, Ax, b, x, fp, maxiter, &rep,
                                 mpir_dropin::device());
  if (rc != MPIR_OK) throw std::runtime_error(std::string("LUIR_QDLDL: ") + mpir_last_error());
  stats->fact_prec_            = typeid(FACTPREC).name();
  stats->work_prec_            = typeid(WORKPREC).name();
  stats->res_prec_             = typeid(RESPREC).name();
  stats->n_                    = static_cast<int>(n);
  stats->nnz_                  = static_cast<long int>(nnz);
  stats->num_refinement_steps_ = rep.ir_iterations;
  stats->relative_residual_    = rep.residual_norm;
  stats->time_num_fact_        = rep.factor_ms * 1e-3;
  stats->time_ref_             = rep.solve_ms * 1e-3;
}

#endif
