// Tangent (forward-mode) build of the oracle -- test infrastructure only.
//
// Force-included ahead of ugks_oracle.c when the oracle is compiled as C++ (oracle/Makefile target
// `tangent`): every FP64 value of the oracle becomes a uo_dual (value, derivative along one
// direction), whose arithmetic propagates the derivative exactly (to rounding).  Seeding the
// derivative of the state h, b, W or of a parameter (mu_ref, wall speed, wall temperature) and running
// the oracle's own steps gives the Jacobian-vector product of those steps: the forward-mode check that
// the device adjoint (a vector-Jacobian product) is tested against, <J v, u> = <v, J^T u>.
//
// Branches (fabs, fmax, fmin, comparisons, the Newton loop's accept / stop tests) follow the values,
// so the product is that of the branch the oracle takes; where the oracle's function is not
// differentiable (a tie in fmax, |x| at 0) the one-sided derivative of the branch taken is used.
// The ABI of this build passes uo_dual arrays (value, derivative interleaved) wherever the plain
// oracle passes double arrays; oracle/tangent.py wraps it.
#pragma once
#include <cmath>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <pthread.h>
#include <stdatomic.h>
#include <unistd.h>
#include <cstddef>
#include <type_traits>

using uo_f64 = decltype(0.0);

struct uo_dual {
    uo_f64 v, d;
    uo_dual() = default;
    constexpr uo_dual(uo_f64 x) : v(x), d(0.0) {}
    constexpr uo_dual(uo_f64 x, uo_f64 dx) : v(x), d(dx) {}
    template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
    constexpr uo_dual(T x) : v(static_cast<uo_f64>(x)), d(0.0) {}
    template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
    explicit constexpr operator T() const { return static_cast<T>(v); }
    uo_dual& operator+=(uo_dual o) { v += o.v; d += o.d; return *this; }
    uo_dual& operator-=(uo_dual o) { v -= o.v; d -= o.d; return *this; }
    uo_dual& operator*=(uo_dual o) { d = d * o.v + v * o.d; v *= o.v; return *this; }
    uo_dual& operator/=(uo_dual o) { const uo_f64 q = v / o.v; d = (d - q * o.d) / o.v; v = q; return *this; }
};
static_assert(sizeof(uo_dual) == 16 && std::is_trivially_copyable_v<uo_dual>, "value and derivative");

inline uo_dual operator+(uo_dual a, uo_dual b) { return {a.v + b.v, a.d + b.d}; }
inline uo_dual operator-(uo_dual a, uo_dual b) { return {a.v - b.v, a.d - b.d}; }
inline uo_dual operator*(uo_dual a, uo_dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline uo_dual operator/(uo_dual a, uo_dual b) {
    const uo_f64 q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
inline uo_dual operator-(uo_dual a) { return {-a.v, -a.d}; }
inline uo_dual operator+(uo_dual a) { return a; }
inline bool operator<(uo_dual a, uo_dual b) { return a.v < b.v; }
inline bool operator>(uo_dual a, uo_dual b) { return a.v > b.v; }
inline bool operator<=(uo_dual a, uo_dual b) { return a.v <= b.v; }
inline bool operator>=(uo_dual a, uo_dual b) { return a.v >= b.v; }
inline bool operator==(uo_dual a, uo_dual b) { return a.v == b.v; }
inline bool operator!=(uo_dual a, uo_dual b) { return a.v != b.v; }

inline uo_dual sqrt(uo_dual a) {
    const uo_f64 s = std::sqrt(a.v);
    return {s, a.d / (2.0 * s)};
}
inline uo_dual exp(uo_dual a) {
    const uo_f64 e = std::exp(a.v);
    return {e, e * a.d};
}
// d erfc(x)/dx = -2/sqrt(pi) exp(-x^2)
inline uo_dual erfc(uo_dual a) {
    return {std::erfc(a.v), -1.1283791670955125739 * std::exp(-a.v * a.v) * a.d};
}
inline uo_dual pow(uo_dual a, uo_dual b) {
    const uo_f64 p = std::pow(a.v, b.v);
    uo_f64 d = 0.0;
    if (a.d != 0.0) d += b.v * std::pow(a.v, b.v - 1.0) * a.d;
    if (b.d != 0.0) d += p * std::log(a.v) * b.d;
    return {p, d};
}
inline uo_dual acos(uo_dual a) { return {std::acos(a.v), -a.d / std::sqrt(1.0 - a.v * a.v)}; }
inline uo_dual fabs(uo_dual a) { return a.v < 0.0 ? -a : a; }
inline uo_dual fmax(uo_dual a, uo_dual b) { return (a.v >= b.v || std::isnan(b.v)) ? a : b; }
inline uo_dual fmin(uo_dual a, uo_dual b) { return (a.v <= b.v || std::isnan(b.v)) ? a : b; }
inline uo_dual copysign(uo_dual a, uo_dual b) {
    const uo_f64 r = std::copysign(a.v, b.v);
    return {r, (std::signbit(r) == std::signbit(a.v)) ? a.d : -a.d};
}
inline uo_dual ldexp(uo_dual a, int e) { return {std::ldexp(a.v, e), std::ldexp(a.d, e)}; }
inline bool isfinite(uo_dual a) { return std::isfinite(a.v); }   // the oracle's gates see the values only
inline bool isnan(uo_dual a) { return std::isnan(a.v); }

// malloc / calloc return a pointer that converts to any object pointer, as void* does in C
struct uo_any_ptr {
    void* p;
    template <class T> operator T*() const { return static_cast<T*>(p); }
};
inline uo_any_ptr uo_malloc(size_t n) { return {std::malloc(n)}; }
inline uo_any_ptr uo_calloc(size_t n, size_t s) { return {std::calloc(n, s)}; }

#define double uo_dual
#define malloc(n) uo_malloc(n)
#define calloc(n, s) uo_calloc(n, s)
