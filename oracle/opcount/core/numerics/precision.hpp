// Stand-in for the reference's core/numerics/precision.hpp in the op-counting build -- TEST INFRASTRUCTURE ONLY.
//
// oracle/opcount/count_ops.cpp is compiled with this directory ahead of the reference's src/ on the include path, so
// that the reference's headers, which include "core/numerics/precision.hpp", get this file: it declares the same
// names (scalar, IS_FP32, limits<>, accuracy_name, core::precision::comp_add) with `scalar` = the op-counting FP32
// type and the FP32 thresholds of the reference's FP32 build.  Everything else is the reference's own code.
#pragma once

#include <type_traits>

#include "core/numerics/macros.hpp"
#include "opcount.hpp"

enum accuracy_mode { FP64, FP32 };

using scalar = phx_opcount::CountF;
inline constexpr bool IS_FP32 = true;

static inline const char* accuracy_name(void) { return "FP32 (op-counting)"; }

template <class T>
struct limits;

template <>
struct limits<phx_opcount::CountF> {
  static constexpr float step_tiny = 1e-30f;
  static constexpr float step_big = 1e30f;
  static constexpr float tol_series = 1e-9f;
  static constexpr float tol_asym = 1e-8f;
};

// sincos_t / fmod_t of the reference's macros.hpp for the counting type (host forms: sin and cos, fmod)
static inline void sincos_t(scalar x, scalar* s, scalar* c) {
  *s = std::sin(x);
  *c = std::cos(x);
}
static inline scalar fmod_t(scalar x, scalar y) { return std::fmod(x, y); }

namespace core {
namespace precision {
// hi + lo += d, compensated: the error of hi + d (TwoSum) folds into lo, then (hi, lo) is renormalised.
static inline void comp_add(scalar* hi, scalar* lo, scalar d) {
  const scalar sum = *hi + d;
  const scalar d_part = sum - *hi;
  const scalar err = (*hi - (sum - d_part)) + (d - d_part);
  *lo += err;
  const scalar renorm = sum + *lo;
  *lo = *lo - (renorm - sum);
  *hi = renorm;
}
}  // namespace precision
}  // namespace core
