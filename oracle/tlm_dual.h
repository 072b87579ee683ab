// Forward-mode dual number for the tangent-linear FP64 build of the
// reference path (oracle/ref_tlm.cpp).  TEST INFRASTRUCTURE ONLY: it checks
// the GPU adjoint; nothing in the product includes it.
//
// A Dual holds a value and kDirs directional derivatives.  Every operation
// computes the value with exactly the double operation the plain build
// performs (so the primal trajectory is the reference's own, bit for bit when
// both builds contract no multiply-add), and the derivatives by the chain
// rule.  Piecewise-constant functions (floor, ceil, round, comparisons) have
// zero derivative; min / max / abs follow the selected branch.
#pragma once

#include <cmath>
#include <cstddef>
#include <limits>
#include <ostream>
#include <type_traits>

namespace octlb_tlm {

constexpr int kDirs = 10;

struct Dual {
  double v = 0.0;
  double d[kDirs] = {};

  constexpr Dual() = default;
  template <class A, class = std::enable_if_t<std::is_arithmetic_v<A>>>
  constexpr Dual(A x) : v(static_cast<double>(x)), d{} {}  // NOLINT: implicit, like a double
  template <class A, class = std::enable_if_t<std::is_arithmetic_v<A>>>
  explicit constexpr operator A() const { return static_cast<A>(v); }

  constexpr Dual& operator+=(const Dual& b) {
    v += b.v;
    for (int k = 0; k < kDirs; ++k) d[k] += b.d[k];
    return *this;
  }
  constexpr Dual& operator-=(const Dual& b) {
    v -= b.v;
    for (int k = 0; k < kDirs; ++k) d[k] -= b.d[k];
    return *this;
  }
  constexpr Dual& operator*=(const Dual& b) {
    for (int k = 0; k < kDirs; ++k) d[k] = d[k] * b.v + v * b.d[k];
    v *= b.v;
    return *this;
  }
  constexpr Dual& operator/=(const Dual& b) {
    const double q = v / b.v;
    for (int k = 0; k < kDirs; ++k) d[k] = (d[k] - q * b.d[k]) / b.v;
    v = q;
    return *this;
  }
};

constexpr Dual operator+(const Dual& a) { return a; }
constexpr Dual operator-(const Dual& a) {
  Dual r;
  r.v = -a.v;
  for (int k = 0; k < kDirs; ++k) r.d[k] = -a.d[k];
  return r;
}
constexpr Dual operator+(Dual a, const Dual& b) { return a += b; }
constexpr Dual operator-(Dual a, const Dual& b) { return a -= b; }
constexpr Dual operator*(Dual a, const Dual& b) { return a *= b; }
constexpr Dual operator/(Dual a, const Dual& b) { return a /= b; }

constexpr bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
constexpr bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
constexpr bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
constexpr bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
constexpr bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
constexpr bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }

inline Dual sqrt(const Dual& a) {
  Dual r;
  r.v = std::sqrt(a.v);
  for (int k = 0; k < kDirs; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}
inline Dual abs(const Dual& a) { return a.v < 0.0 ? -a : a; }
inline Dual fabs(const Dual& a) { return abs(a); }
inline Dual exp(const Dual& a) {
  Dual r;
  r.v = std::exp(a.v);
  for (int k = 0; k < kDirs; ++k) r.d[k] = r.v * a.d[k];
  return r;
}
inline Dual log(const Dual& a) {
  Dual r;
  r.v = std::log(a.v);
  for (int k = 0; k < kDirs; ++k) r.d[k] = a.d[k] / a.v;
  return r;
}
inline Dual pow(const Dual& a, double p) {
  Dual r;
  r.v = std::pow(a.v, p);
  const double g = p * std::pow(a.v, p - 1.0);
  for (int k = 0; k < kDirs; ++k) r.d[k] = g * a.d[k];
  return r;
}
inline Dual floor(const Dual& a) { return Dual(std::floor(a.v)); }
inline Dual ceil(const Dual& a) { return Dual(std::ceil(a.v)); }
inline Dual round(const Dual& a) { return Dual(std::round(a.v)); }
inline Dual min(const Dual& a, const Dual& b) { return b.v < a.v ? b : a; }
inline Dual max(const Dual& a, const Dual& b) { return a.v < b.v ? b : a; }
inline bool isfinite(const Dual& a) { return std::isfinite(a.v); }
inline bool isnan(const Dual& a) { return std::isnan(a.v); }
inline bool isinf(const Dual& a) { return std::isinf(a.v); }

inline std::ostream& operator<<(std::ostream& os, const Dual& a) { return os << a.v; }

}  // namespace octlb_tlm

// Qualified calls (std::sqrt(x), std::max(x, 0.0)) in the differentiated
// sources resolve to the Dual forms.
namespace std {
using octlb_tlm::abs;
using octlb_tlm::ceil;
using octlb_tlm::exp;
using octlb_tlm::fabs;
using octlb_tlm::floor;
using octlb_tlm::isfinite;
using octlb_tlm::isinf;
using octlb_tlm::isnan;
using octlb_tlm::log;
using octlb_tlm::pow;
using octlb_tlm::round;
using octlb_tlm::sqrt;
inline octlb_tlm::Dual max(const octlb_tlm::Dual& a, double b) { return octlb_tlm::max(a, octlb_tlm::Dual(b)); }
inline octlb_tlm::Dual max(double a, const octlb_tlm::Dual& b) { return octlb_tlm::max(octlb_tlm::Dual(a), b); }
inline octlb_tlm::Dual min(const octlb_tlm::Dual& a, double b) { return octlb_tlm::min(a, octlb_tlm::Dual(b)); }
inline octlb_tlm::Dual min(double a, const octlb_tlm::Dual& b) { return octlb_tlm::min(octlb_tlm::Dual(a), b); }

template <>
class numeric_limits<octlb_tlm::Dual> : public numeric_limits<double> {
 public:
  static constexpr octlb_tlm::Dual min() noexcept { return numeric_limits<double>::min(); }
  static constexpr octlb_tlm::Dual max() noexcept { return numeric_limits<double>::max(); }
  static constexpr octlb_tlm::Dual lowest() noexcept { return numeric_limits<double>::lowest(); }
  static constexpr octlb_tlm::Dual epsilon() noexcept { return numeric_limits<double>::epsilon(); }
  static constexpr octlb_tlm::Dual infinity() noexcept { return numeric_limits<double>::infinity(); }
  static constexpr octlb_tlm::Dual quiet_NaN() noexcept { return numeric_limits<double>::quiet_NaN(); }
};
}  // namespace std
