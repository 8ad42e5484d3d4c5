// Drop-in QDLDL for the reference's include/MPIR/qdldl.hpp: the same
// templates and return codes, computed by libmpir_b200 (the numeric factor
// and the solves on the GPU, device from the environment variable
// MPIR_DEVICE, default 0).
//
//   QDLDL_etree   qdldl.hpp:48-105   host; returns sum(Lnz), -1 or -2
//   QDLDL_factor  qdldl.hpp:172-345  returns #positive D, -1 on zero pivot
//   QDLDL_Lsolve  qdldl.hpp:362-372
//   QDLDL_Ltsolve qdldl.hpp:389-400
//   QDLDL_solve   qdldl.hpp:417-432
//
// All buffers stay caller-allocated ("does not use MALLOC" in the
// reference); the work arrays bwork/iwork/fwork are accepted and unused.  The
// factor is computed in float32 and stored in PREC (float, or
// std::bfloat16_t / std::float16_t rounded from float32); PREC = double is
// not provided and QDLDL_factor then returns MPIR_ERR_UNSUPPORTED (-7).  The
// void solves throw std::runtime_error when the device reports an error.
#pragma once
#ifndef MPIR_B200_QDLDL_HPP
#define MPIR_B200_QDLDL_HPP

#include <cstdint>
#include <cstdlib>
#include <limits>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>
#if __has_include(<stdfloat>)
#include <stdfloat>
#endif

#include "../mpir_b200.h"

namespace mpir_dropin {

inline int device() {
  const char *e = std::getenv("MPIR_DEVICE");
  return e ? std::atoi(e) : 0;
}

template <class T>
constexpr int prec_of() {
  if constexpr (std::is_same_v<T, double>) return MPIR_F64;
  else if constexpr (std::is_same_v<T, float>) return MPIR_F32;
#if defined(__STDCPP_BFLOAT16_T__)
  else if constexpr (std::is_same_v<T, std::bfloat16_t>) return MPIR_BF16;
#endif
#if defined(__STDCPP_FLOAT16_T__)
  else if constexpr (std::is_same_v<T, std::float16_t>) return MPIR_F16;
#endif
  else return -1;
}

// int64 views of caller index arrays (copies when INT is not int64_t).
template <class INT>
struct I64View {
  std::vector<int64_t> buf;
  const int64_t       *p = nullptr;
  I64View(const INT *src, int64_t len) {
    if constexpr (std::is_same_v<INT, int64_t>) {
      p = src;
    } else {
      buf.assign(src, src + len);
      p = buf.data();
    }
  }
};

template <class INT>
void copy_out(const std::vector<int64_t> &src, INT *dst) {
  for (size_t i = 0; i < src.size(); i++) dst[i] = static_cast<INT>(src[i]);
}

inline void throw_on(int rc, const char *what) {
  if (rc < 0)
    throw std::runtime_error(std::string(what) + ": " + mpir_last_error());
}

template <typename INT, typename FACTPREC, typename XPREC>
void solve_phases(INT n, const INT *Lp, const INT *Li, const FACTPREC *Lx,
                  const FACTPREC *Dinv, XPREC *x, int which) {
  static_assert(prec_of<FACTPREC>() > 0, "factor type: float, bfloat16_t or float16_t");
  I64View<INT> lp(Lp, n + 1), li(Li, n > 0 ? static_cast<int64_t>(Lp[n]) : 0);
  constexpr bool native = std::is_same_v<XPREC, double> || std::is_same_v<XPREC, float>;
  std::vector<double> xd;
  void               *xp = x;
  int                 xprec;
  if constexpr (native) {
    xprec = prec_of<XPREC>();
  } else {
    xd.assign(x, x + n);
    xp    = xd.data();
    xprec = MPIR_F64;
  }
  int rc;
  if (which == 0)
    rc = mpir_qdldl_solve(n, lp.p, li.p, Lx, Dinv, prec_of<FACTPREC>(), xp, xprec, device());
  else if (which == 1)
    rc = mpir_qdldl_lsolve(n, lp.p, li.p, Lx, prec_of<FACTPREC>(), xp, xprec, device());
  else
    rc = mpir_qdldl_ltsolve(n, lp.p, li.p, Lx, prec_of<FACTPREC>(), xp, xprec, device());
  throw_on(rc, "QDLDL solve");
  if constexpr (!native)
    for (INT i = 0; i < n; i++) x[i] = static_cast<XPREC>(xd[i]);
}

}  // namespace mpir_dropin

template <typename INT>
INT QDLDL_etree(const INT n, const INT *Ap, const INT *Ai, INT *work, INT *Lnz,
                INT *etree) {
  using namespace mpir_dropin;
  I64View<INT> ap(Ap, n + 1), ai(Ai, n > 0 ? static_cast<int64_t>(Ap[n]) : 0);
  std::vector<int64_t> lnz(n), et(n), wk(n);
  const int64_t        r = mpir_qdldl_etree(n, ap.p, ai.p, wk.data(), lnz.data(), et.data());
  copy_out(lnz, Lnz);
  copy_out(et, etree);
  copy_out(wk, work);
  if (r >= 0 && r > static_cast<int64_t>(std::numeric_limits<INT>::max())) return -2;
  return static_cast<INT>(r);
}

template <typename INT, typename PREC>
INT QDLDL_factor(INT n, const INT *Ap, const INT *Ai, const PREC *Ax, INT *Lp,
                 INT *Li, PREC *Lx, PREC *D, PREC *Dinv, const INT *Lnz,
                 const INT *etree, bool * /*bwork*/, INT * /*iwork*/,
                 PREC * /*fwork*/) {
  using namespace mpir_dropin;
  constexpr int prec = prec_of<PREC>();
  if constexpr (prec != MPIR_F32 && prec != MPIR_BF16 && prec != MPIR_F16) {
    return static_cast<INT>(MPIR_ERR_UNSUPPORTED);
  } else {
    const int64_t        nnz = n > 0 ? static_cast<int64_t>(Ap[n]) : 0;
    I64View<INT>         ap(Ap, n + 1), ai(Ai, nnz), lnz(Lnz, n), et(etree, n);
    std::vector<double>  ax(Ax, Ax + nnz);
    int64_t              nl = 0;
    for (INT i = 0; i < n; i++) nl += static_cast<int64_t>(Lnz[i]);
    std::vector<int64_t> lp(n + 1), li(nl);
    const int64_t        r = mpir_qdldl_factor(n, ap.p, ai.p, ax.data(), lp.data(), li.data(), Lx,
                                               D, Dinv, prec, lnz.p, et.p, device());
    if (r >= -1) {
      copy_out(lp, Lp);
      copy_out(li, Li);
    }
    return static_cast<INT>(r);
  }
}

template <typename INT, typename FACTPREC, typename XPREC>
void QDLDL_Lsolve(INT n, const INT *Lp, const INT *Li, const FACTPREC *Lx, XPREC *x) {
  mpir_dropin::solve_phases(n, Lp, Li, Lx, static_cast<const FACTPREC *>(nullptr), x, 1);
}

template <typename INT, typename FACTPREC, typename XPREC>
void QDLDL_Ltsolve(INT n, const INT *Lp, const INT *Li, const FACTPREC *Lx, XPREC *x) {
  mpir_dropin::solve_phases(n, Lp, Li, Lx, static_cast<const FACTPREC *>(nullptr), x, 2);
}

template <typename INT, typename FACTPREC, typename XPREC>
void QDLDL_solve(const INT n, const INT *Lp, const INT *Li, const FACTPREC *Lx,
                 const FACTPREC *Dinv, XPREC *x) {
  mpir_dropin::solve_phases(n, Lp, Li, Lx, Dinv, x, 0);
}

#endif
