// Op-counting FP32 scalar for the algorithmic flop count of the raymarch -- TEST INFRASTRUCTURE ONLY.
//
// CountF holds a float and behaves like one, and every arithmetic operation on it adds to per-thread tallies:
// additions/subtractions, multiplications, divisions, square roots, comparisons, min/max/abs, and calls of each
// transcendental function.  oracle/opcount/core/numerics/precision.hpp makes it the `scalar` of the reference's
// FP32 build, so that the reference's own per-pixel code (core/render/pixel.hpp) is counted as written.
#pragma once

#include <cmath>
#include <cstdint>
#include <type_traits>

namespace phx_opcount {

enum Op {
  kAdd, kMul, kDiv, kSqrt, kCmp, kMinMaxAbs,
  kExp, kLog, kSin, kCos, kPow, kCbrt, kAcos, kExpm1, kTanh, kSinh, kCosh, kAcosh, kFmod, kFloor,
  kNumOps
};

inline const char* op_name(int k) {
  static const char* names[kNumOps] = {"add", "mul", "div", "sqrt", "cmp", "minmaxabs", "exp", "log", "sin", "cos",
                                       "pow", "cbrt", "acos", "expm1", "tanh", "sinh", "cosh", "acosh", "fmod",
                                       "floor"};
  return names[k];
}

struct Tally {
  unsigned long long n[kNumOps];
};

inline Tally& tally() {
  static thread_local Tally t{};
  return t;
}

inline void bump(Op k) { tally().n[k]++; }

struct CountF {
  float v;
  CountF() = default;
  constexpr CountF(float x) : v(x) {}
  constexpr CountF(double x) : v((float)x) {}
  constexpr CountF(int x) : v((float)x) {}
  constexpr CountF(long x) : v((float)x) {}
  constexpr CountF(long long x) : v((float)x) {}
  constexpr CountF(unsigned x) : v((float)x) {}
  constexpr CountF(unsigned long x) : v((float)x) {}
  template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
  constexpr explicit operator T() const {
    return (T)v;
  }
  CountF& operator+=(CountF b) { bump(kAdd); v += b.v; return *this; }
  CountF& operator-=(CountF b) { bump(kAdd); v -= b.v; return *this; }
  CountF& operator*=(CountF b) { bump(kMul); v *= b.v; return *this; }
  CountF& operator/=(CountF b) { bump(kDiv); v /= b.v; return *this; }
};
static_assert(sizeof(CountF) == sizeof(float), "CountF must have float's layout");

inline CountF operator-(CountF a) { return CountF(-a.v); }
inline CountF operator+(CountF a) { return a; }

#define PHX_OPC_BIN(OP, KIND)                                                                       \
  inline CountF operator OP(CountF a, CountF b) { bump(KIND); return CountF(a.v OP b.v); }          \
  template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>                             \
  inline CountF operator OP(CountF a, T b) { bump(KIND); return CountF(a.v OP (float)b); }          \
  template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>                             \
  inline CountF operator OP(T a, CountF b) { bump(KIND); return CountF((float)a OP b.v); }
PHX_OPC_BIN(+, kAdd)
PHX_OPC_BIN(-, kAdd)
PHX_OPC_BIN(*, kMul)
PHX_OPC_BIN(/, kDiv)
#undef PHX_OPC_BIN

#define PHX_OPC_CMP(OP)                                                                             \
  inline bool operator OP(CountF a, CountF b) { bump(kCmp); return a.v OP b.v; }                    \
  template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>                             \
  inline bool operator OP(CountF a, T b) { bump(kCmp); return a.v OP (float)b; }                    \
  template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>                             \
  inline bool operator OP(T a, CountF b) { bump(kCmp); return (float)a OP b.v; }
PHX_OPC_CMP(<)
PHX_OPC_CMP(>)
PHX_OPC_CMP(<=)
PHX_OPC_CMP(>=)
PHX_OPC_CMP(==)
PHX_OPC_CMP(!=)
#undef PHX_OPC_CMP

#define PHX_OPC_FN1(NAME, KIND)                                                                     \
  inline CountF NAME(CountF a) { bump(KIND); return CountF(std::NAME(a.v)); }
PHX_OPC_FN1(sqrt, kSqrt)
PHX_OPC_FN1(exp, kExp)
PHX_OPC_FN1(log, kLog)
PHX_OPC_FN1(sin, kSin)
PHX_OPC_FN1(cos, kCos)
PHX_OPC_FN1(cbrt, kCbrt)
PHX_OPC_FN1(acos, kAcos)
PHX_OPC_FN1(expm1, kExpm1)
PHX_OPC_FN1(tanh, kTanh)
PHX_OPC_FN1(sinh, kSinh)
PHX_OPC_FN1(cosh, kCosh)
PHX_OPC_FN1(acosh, kAcosh)
PHX_OPC_FN1(floor, kFloor)
PHX_OPC_FN1(fabs, kMinMaxAbs)
#undef PHX_OPC_FN1
inline CountF abs(CountF a) { return fabs(a); }
inline CountF pow(CountF a, CountF b) { bump(kPow); return CountF(std::pow(a.v, b.v)); }
inline CountF fmod(CountF a, CountF b) { bump(kFmod); return CountF(std::fmod(a.v, b.v)); }
inline CountF fmin(CountF a, CountF b) { bump(kMinMaxAbs); return CountF(std::fmin(a.v, b.v)); }
inline CountF fmax(CountF a, CountF b) { bump(kMinMaxAbs); return CountF(std::fmax(a.v, b.v)); }
inline bool isfinite(CountF a) { return std::isfinite(a.v); }
inline bool isnan(CountF a) { return std::isnan(a.v); }

}  // namespace phx_opcount

// The reference calls most math functions as std::name(x): the same overloads in namespace std.
namespace std {
using phx_opcount::abs;
using phx_opcount::acos;
using phx_opcount::acosh;
using phx_opcount::cbrt;
using phx_opcount::cos;
using phx_opcount::cosh;
using phx_opcount::exp;
using phx_opcount::expm1;
using phx_opcount::fabs;
using phx_opcount::floor;
using phx_opcount::fmax;
using phx_opcount::fmin;
using phx_opcount::fmod;
using phx_opcount::isfinite;
using phx_opcount::isnan;
using phx_opcount::log;
using phx_opcount::pow;
using phx_opcount::sin;
using phx_opcount::sinh;
using phx_opcount::sqrt;
using phx_opcount::tanh;
}  // namespace std

using phx_opcount::abs;
using phx_opcount::acos;
using phx_opcount::acosh;
using phx_opcount::cbrt;
using phx_opcount::cos;
using phx_opcount::cosh;
using phx_opcount::exp;
using phx_opcount::expm1;
using phx_opcount::fabs;
using phx_opcount::floor;
using phx_opcount::fmax;
using phx_opcount::fmin;
using phx_opcount::fmod;
using phx_opcount::isfinite;
using phx_opcount::isnan;
using phx_opcount::log;
using phx_opcount::pow;
using phx_opcount::sin;
using phx_opcount::sinh;
using phx_opcount::sqrt;
using phx_opcount::tanh;
