// Host vector helpers with the signatures of the reference's
// include/MPIR/ops.hpp (MatrixMultiply :25-45, VectorAdd :54-61,
// VectorSubtract :88-96, VectorMultiply :123-131, VectorScale :160-168,
// VectorDot :195-200, Dnrm2 :231-287, InfNrm :324-329), for callers that
// build right-hand sides or check results on the host, as the reference's
// example driver does.  The solver's own products, norms and dot products
// run on the GPU inside libmpir_b200; these helpers are not on that path.
#pragma once
#ifndef MPIR_B200_OPS_HPP
#define MPIR_B200_OPS_HPP

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <numeric>
#include <span>
#include <vector>

#include "fp_concepts.hpp"

// y = K x for K given by its upper triangle in CSC; products in Top, stored in T.
template <typename T, typename Top = T, typename Ta, typename Tx>
  requires Refinable<T, Top>
std::vector<T> MatrixMultiply(const std::vector<std::size_t> &Ap,
                              const std::vector<std::size_t> &Ai,
                              const std::vector<Ta> &Ax, const std::vector<Tx> &x) {
  std::vector<T>    y(x.size(), static_cast<T>(0));
  const std::size_t n = Ap.size() - 1;
  for (std::size_t c = 0; c < n; c++)
    for (std::size_t p = Ap[c]; p < Ap[c + 1]; p++) {
      const std::size_t r = Ai[p];
      const Top         a = static_cast<Top>(Ax[p]);
      y[c] += static_cast<T>(a * static_cast<Top>(x[r]));
      if (r < c) y[r] += static_cast<T>(a * static_cast<Top>(x[c]));
    }
  return y;
}

template <typename T, typename Ta, typename Tb>
std::vector<T> VectorAdd(const std::vector<Ta> &a, const std::vector<Tb> &b) {
  std::vector<T> r(a.size());
  for (std::size_t i = 0; i < a.size(); i++) r[i] = static_cast<T>(a[i]) + static_cast<T>(b[i]);
  return r;
}

template <typename T, typename Ta, typename Tb>
std::vector<T> VectorSubtract(const std::vector<Ta> &a, const std::vector<Tb> &b) {
  std::vector<T> r(a.size());
  for (std::size_t i = 0; i < a.size(); i++) r[i] = static_cast<T>(a[i]) - static_cast<T>(b[i]);
  return r;
}

template <typename T, typename Ta, typename Tb>
std::vector<T> VectorMultiply(const std::vector<Ta> &a, const std::vector<Tb> &b) {
  std::vector<T> r(a.size());
  for (std::size_t i = 0; i < a.size(); i++) r[i] = static_cast<T>(a[i]) * static_cast<T>(b[i]);
  return r;
}

template <typename T, typename Ta, typename Tb, typename Top = T>
  requires Refinable<T, Top>
std::vector<T> VectorScale(const std::vector<Ta> &a, Tb b) {
  std::vector<T> r(a.size());
  for (std::size_t i = 0; i < a.size(); i++)
    r[i] = static_cast<T>(static_cast<Top>(a[i]) * static_cast<Top>(b));
  return r;
}

template <typename T, typename Ta, typename Tb>
T VectorDot(const std::vector<Ta> &a, const std::vector<Tb> &b) {
  T s = static_cast<T>(0);
  for (std::size_t i = 0; i < a.size(); i++) s += static_cast<T>(a[i] * b[i]);
  return s;
}

// Two-norm with a running scale (no overflow for large entries).
template <typename T, typename Tx>
T Dnrm2(std::span<const Tx> x) {
  using std::abs;
  using std::sqrt;
  if (x.empty()) return static_cast<T>(0);
  if (x.size() == 1) return abs(static_cast<T>(x[0]));
  T scale = static_cast<T>(0), ssq = static_cast<T>(1);
  for (std::size_t i = x.size(); i-- > 0;) {
    const T v = static_cast<T>(x[i]);
    if (v == static_cast<T>(0)) continue;
    const T a = abs(v);
    if (scale < a) {
      ssq   = static_cast<T>(1) + ssq * ((scale / a) * (scale / a));
      scale = a;
    } else {
      ssq += (a / scale) * (a / scale);
    }
  }
  return scale * sqrt(ssq);
}

template <typename T, typename Tx>
T Dnrm2(const std::vector<Tx> &x) {
  return Dnrm2<T, Tx>(std::span<const Tx>(x.data(), x.size()));
}

template <typename T>
T InfNrm(const std::vector<T> &x) {
  using std::abs;
  T m = static_cast<T>(0);
  for (const T &v : x) m = std::max(m, static_cast<T>(abs(v)));
  return m;
}

#endif
