// Precision concepts of the drop-in API, with the meaning of the reference's
// include/MPIR/fp_concepts.hpp:28-125: a list of types is Refinable when each
// is floating-point-like and their machine epsilons do not increase along
// the list (factor >= working >= residual precision).
//
// Besides the standard floating-point types (including std::bfloat16_t and
// std::float16_t), the residual precision may be double-double: the QD
// library's dd_real when MPIR_USE_QD is defined, or mpir::double_double,
// a tag type that selects the device's double-double residual.
#pragma once
#ifndef MPIR_B200_FP_CONCEPTS_HPP
#define MPIR_B200_FP_CONCEPTS_HPP

#include <concepts>
#include <limits>
#include <type_traits>

#ifdef MPIR_USE_QD
#include <qd/dd_real.h>
#include <qd/qd_real.h>
#endif

namespace mpir {
// Tag type for a double-double residual precision (epsilon 2^-104).
struct double_double {
  double hi = 0.0, lo = 0.0;
  constexpr double_double() = default;
  constexpr double_double(double v) : hi(v) {}  // NOLINT: implicit like dd_real
  constexpr operator double() const { return hi + lo; }
};

template <class T>
struct is_extended_real : std::false_type {};
template <>
struct is_extended_real<double_double> : std::true_type {};
#ifdef MPIR_USE_QD
template <>
struct is_extended_real<dd_real> : std::true_type {};
template <>
struct is_extended_real<qd_real> : std::true_type {};
#endif

template <class T>
constexpr double epsilon_of() {
  if constexpr (std::is_same_v<T, double_double>) {
    return 4.93038065763132e-32;  // 2^-104
  } else {
    return static_cast<double>(std::numeric_limits<T>::epsilon());
  }
}
}  // namespace mpir

template <typename T, typename... Ts>
constexpr bool is_all_floating_point_v =
    is_all_floating_point_v<T> && is_all_floating_point_v<Ts...>;
template <typename T>
constexpr bool is_all_floating_point_v<T> =
    std::floating_point<T> || mpir::is_extended_real<T>::value;

template <typename... Ts>
concept FloatingPoint = is_all_floating_point_v<Ts...>;

template <typename T, typename... Ts>
constexpr bool is_partial_ordered_v =
    ((mpir::epsilon_of<T>() >= mpir::epsilon_of<Ts>()) && ...) &&
    is_partial_ordered_v<Ts...>;
template <typename T>
constexpr bool is_partial_ordered_v<T> = true;

template <typename... Ts>
concept PartialOrdered = is_partial_ordered_v<Ts...>;

template <typename... Ts>
concept Refinable = FloatingPoint<Ts...> && PartialOrdered<Ts...>;

static_assert(Refinable<double>);
static_assert(Refinable<float, double, double>);
static_assert(Refinable<float, double, mpir::double_double>);
static_assert(!Refinable<double, float, double>);
static_assert(!Refinable<int>);

#endif
