// Op-counting build of the oracle (test and measurement infrastructure only).
//
// Force-included ahead of ugks_oracle.c when the oracle is compiled as C++ (oracle/Makefile target
// `flops`): every FP64 value of the oracle becomes a uo_real, whose arithmetic counts itself.  The
// counts give the algorithmic FP64 operations per cell-velocity update of each method, which turn
// the measured throughput into a fraction of the FP64 peak.
//   add  : + and - (binary and compound)        mul : *        div : /
//   sqrt, exp, erfc, pow, acos : calls, counted apart from the arithmetic
// Comparisons, fabs / fmax / fmin / copysign, negation and conversions are not counted.
// The counters are plain globals: run the counting build on one thread.
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

enum { UO_ADD, UO_MUL, UO_DIV, UO_SQRT, UO_EXP, UO_ERFC, UO_POW, UO_ACOS, UO_NCOUNT };
inline unsigned long long uo_count[UO_NCOUNT];

struct uo_real {
    uo_f64 v;
    uo_real() = default;
    constexpr uo_real(uo_f64 x) : v(x) {}
    template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
    constexpr uo_real(T x) : v(static_cast<uo_f64>(x)) {}
    template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
    explicit constexpr operator T() const { return static_cast<T>(v); }
    uo_real& operator+=(uo_real o) { ++uo_count[UO_ADD]; v += o.v; return *this; }
    uo_real& operator-=(uo_real o) { ++uo_count[UO_ADD]; v -= o.v; return *this; }
    uo_real& operator*=(uo_real o) { ++uo_count[UO_MUL]; v *= o.v; return *this; }
    uo_real& operator/=(uo_real o) { ++uo_count[UO_DIV]; v /= o.v; return *this; }
};
static_assert(sizeof(uo_real) == 8 && std::is_trivially_copyable_v<uo_real>, "layout of a double");

inline uo_real operator+(uo_real a, uo_real b) { ++uo_count[UO_ADD]; return a.v + b.v; }
inline uo_real operator-(uo_real a, uo_real b) { ++uo_count[UO_ADD]; return a.v - b.v; }
inline uo_real operator*(uo_real a, uo_real b) { ++uo_count[UO_MUL]; return a.v * b.v; }
inline uo_real operator/(uo_real a, uo_real b) { ++uo_count[UO_DIV]; return a.v / b.v; }
inline uo_real operator-(uo_real a) { return -a.v; }
inline uo_real operator+(uo_real a) { return a; }
inline bool operator<(uo_real a, uo_real b) { return a.v < b.v; }
inline bool operator>(uo_real a, uo_real b) { return a.v > b.v; }
inline bool operator<=(uo_real a, uo_real b) { return a.v <= b.v; }
inline bool operator>=(uo_real a, uo_real b) { return a.v >= b.v; }
inline bool operator==(uo_real a, uo_real b) { return a.v == b.v; }
inline bool operator!=(uo_real a, uo_real b) { return a.v != b.v; }

inline uo_real sqrt(uo_real a) { ++uo_count[UO_SQRT]; return std::sqrt(a.v); }
inline uo_real exp(uo_real a) { ++uo_count[UO_EXP]; return std::exp(a.v); }
inline uo_real erfc(uo_real a) { ++uo_count[UO_ERFC]; return std::erfc(a.v); }
inline uo_real pow(uo_real a, uo_real b) { ++uo_count[UO_POW]; return std::pow(a.v, b.v); }
inline uo_real acos(uo_real a) { ++uo_count[UO_ACOS]; return std::acos(a.v); }
inline uo_real fabs(uo_real a) { return std::fabs(a.v); }
inline uo_real fmax(uo_real a, uo_real b) { return std::fmax(a.v, b.v); }
inline uo_real fmin(uo_real a, uo_real b) { return std::fmin(a.v, b.v); }
inline uo_real copysign(uo_real a, uo_real b) { return std::copysign(a.v, b.v); }
inline bool isfinite(uo_real a) { return std::isfinite(a.v); }
inline bool isnan(uo_real a) { return std::isnan(a.v); }

// malloc / calloc return a pointer that converts to any object pointer, as void* does in C
struct uo_any_ptr {
    void* p;
    template <class T> operator T*() const { return static_cast<T*>(p); }
};
inline uo_any_ptr uo_malloc(size_t n) { return {std::malloc(n)}; }
inline uo_any_ptr uo_calloc(size_t n, size_t s) { return {std::calloc(n, s)}; }

extern "C" void uo_flops_reset(void) {
    for (int i = 0; i < UO_NCOUNT; ++i) uo_count[i] = 0;
}
extern "C" void uo_flops_read(unsigned long long* out) {
    for (int i = 0; i < UO_NCOUNT; ++i) out[i] = uo_count[i];
}

#define double uo_real
#define malloc(n) uo_malloc(n)
#define calloc(n, s) uo_calloc(n, s)
