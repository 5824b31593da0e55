// Shared definitions for the PHOENIX-B200 raymarch path: host/device qualifiers, constants and a few math helpers
// that have a cheaper device form.  The same headers are compiled by nvcc (device kernels, host set-up) and by g++
// (host tools such as the snapshot generator and the dump reader).
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define PHX_HD __host__ __device__ __forceinline__
#define PHX_D __device__ __forceinline__
#define PHX_HD_OUTLINE __host__ __device__ __noinline__
#else
#define PHX_HD inline
#define PHX_D inline
#define PHX_HD_OUTLINE __attribute__((noinline))
#endif

namespace phx {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kTwoPi = 2.0 * kPi;
constexpr double kHalfPi = 0.5 * kPi;

// CGS constants.  These are the CODATA-era values the reference renderer uses (core/numerics/constants.hpp:22-52);
// the flux of an image scales with them, so they have to be the same numbers for results to agree.
namespace cgs {
constexpr double m_proton = 1.6726219e-24;
constexpr double m_electron = 9.1093829e-28;
constexpr double q_electron = 4.80320425e-10;
constexpr double k_boltzmann = 1.3806488e-16;
constexpr double c_light = 2.99792458e10;
constexpr double h_planck = 6.62606885e-27;
constexpr double g_newton = 6.674e-8;
constexpr double m_sun = 1.989e33;
constexpr double kpc = 3.086e21;
constexpr double jansky = 1e23;
}  // namespace cgs

// Maximum number of AMR levels a snapshot may carry (the level table of the reference model is 16 deep).
constexpr int kMaxLevels = 16;
// Maximum number of observing frequencies in one render (the reference's CPU default for PHX_MAX_FREQS).
constexpr int kMaxFreqs = 32;
// Primitive slots of one cell, RAPTOR order: rho, u, u^1..3 (Lorentz factor times 3-velocity), B^1..3.
enum Prim { kRho = 0, kUU = 1, kU1 = 2, kU2 = 3, kU3 = 4, kB1 = 5, kB2 = 6, kB3 = 7, kNPrim = 8 };

template <class T>
PHX_HD void sincos_t(T x, T* s, T* c) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4) {
    sincosf(x, s, c);
  } else {
    sincos(x, s, c);
  }
#else
  *s = std::sin(x);
  *c = std::cos(x);
#endif
}

// x mod y for y > 0 and |x / y| < 2^40, bit-identical to fmod: the truncated quotient n makes x - n y exactly
// representable, so one FMA with n returns it exactly.  The quotient estimate q = trunc(x * (1/y)) is off by at most
// one; the sign of the remainder (or |r| >= y) shows which, and the FMA is redone with n.
PHX_HD double fmod_exact(double x, double y) {
  const double q = trunc(x * (1.0 / y));
  double r = fma(-q, y, x);
  if (x >= 0.0) {
    if (r < 0.0) r = fma(-(q - 1.0), y, x);
    else if (r >= y) r = fma(-(q + 1.0), y, x);
  } else {
    if (r > 0.0) r = fma(-(q + 1.0), y, x);
    else if (r <= -y) r = fma(-(q - 1.0), y, x);
  }
  return r == 0.0 ? copysign(0.0, x) : r;  // fmod's zero carries the sign of x
}

// x mod y for y > 0 (sign of x kept).  On the device the float form is a truncated-quotient FMA, which is what the
// reference's device build does (core/numerics/macros.hpp:41), exact for the |x| < 4 pi that occur here; the double
// form is fmod_exact (the library fmod's bits at a fraction of its cost).
template <class T>
PHX_HD T fmod_t(T x, T y) {
#if defined(__CUDA_ARCH__)
  if constexpr (sizeof(T) == 4) {
    return fmaf(-truncf(x * (1.0f / y)), y, x);
  } else {
    return fmod_exact(x, y);
  }
#else
  return std::fmod(x, y);
#endif
}

template <class T>
PHX_HD T sq(T x) {
  return x * x;
}

// Precision-generic wrappers: float arguments go to the float routines on both host and device, double to double.
#define PHX_MATH1(name)                             \
  PHX_HD float name##_t(float x) { return std::name(x); } \
  PHX_HD double name##_t(double x) { return std::name(x); }
#if defined(__CUDA_ARCH__)
#undef PHX_MATH1

#define PHX_MATH1(name)                             \
  PHX_HD float name##_t(float x) { return name##f(x); } \
  PHX_HD double name##_t(double x) { return name(x); }
#endif
PHX_MATH1(exp)
PHX_MATH1(log)
PHX_MATH1(sqrt)
PHX_MATH1(cbrt)
PHX_MATH1(expm1)
PHX_MATH1(tanh)
PHX_MATH1(acos)
PHX_MATH1(cos)
PHX_MATH1(sin)
PHX_MATH1(fabs)
PHX_MATH1(floor)
PHX_MATH1(sinh)
PHX_MATH1(log1p)
#undef PHX_MATH1

#if defined(__CUDA_ARCH__)
PHX_HD float fmin_t(float x, float y) { return fminf(x, y); }
PHX_HD double fmin_t(double x, double y) { return fmin(x, y); }
PHX_HD float fmax_t(float x, float y) { return fmaxf(x, y); }
PHX_HD double fmax_t(double x, double y) { return fmax(x, y); }
#else
PHX_HD float fmin_t(float x, float y) { return std::fmin(x, y); }
PHX_HD double fmin_t(double x, double y) { return std::fmin(x, y); }
PHX_HD float fmax_t(float x, float y) { return std::fmax(x, y); }
PHX_HD double fmax_t(double x, double y) { return std::fmax(x, y); }
#endif

// Hardware-approximate forms for the FP32 emission coefficients (special-function-unit exp / log, approximate
// reciprocal and division: ~1e-6 relative at worst, far below the transfer's error budget).  The double overloads are
// the accurate routines, so FP64 renders are unaffected.
namespace fastm {
#if defined(__CUDA_ARCH__)
PHX_D float exp(float x) { return __expf(x); }
PHX_D float log(float x) { return __logf(x); }
PHX_D float div(float a, float b) { return __fdividef(a, b); }
PHX_D float rcp(float x) { return __fdividef(1.0f, x); }
// sqrt from the hardware reciprocal square root (about 2 ulp): NaN for x < 0 like sqrtf (a bad sample stays bad),
// 0 at x = 0 (where x * rsqrt(x) would be 0 * inf)
PHX_D float sqrt(float x) { return x == 0.0f ? 0.0f : x * rsqrtf(x); }
PHX_D float rsqrt(float x) { return rsqrtf(x); }
PHX_D float tanh(float x) { return 1.0f - __fdividef(2.0f, __expf(2.0f * x) + 1.0f); }
PHX_D float cos(float x) { return __cosf(x); }
#else
inline float exp(float x) { return std::exp(x); }
inline float log(float x) { return std::log(x); }
inline float div(float a, float b) { return a / b; }
inline float rcp(float x) { return 1.0f / x; }
inline float sqrt(float x) { return std::sqrt(x); }
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float tanh(float x) { return std::tanh(x); }
inline float cos(float x) { return std::cos(x); }
#endif
// 1/x for the FP64 geodesic of the mixed mode: a single-precision reciprocal refined by two Newton-Raphson steps
// r <- r + r (1 - x r) in FP64 (each squares the relative error: ~1e-7 -> ~1e-14 -> rounding), about 1 ulp and fewer
// instructions than an IEEE division.  Arguments outside float's normal range take the division.
PHX_HD double rcp_nr(double x) {
  const double ax = x < 0.0 ? -x : x;
  if (!(ax > 1e-30 && ax < 1e30)) return 1.0 / x;
#if defined(__CUDA_ARCH__)
  double r = (double)__fdividef(1.0f, (float)x);
#else
  double r = (double)(1.0f / (float)x);
#endif
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
PHX_HD double exp(double x) { return exp_t(x); }
PHX_HD double log(double x) { return log_t(x); }
PHX_HD double div(double a, double b) { return a / b; }
PHX_HD double rcp(double x) { return 1.0 / x; }
PHX_HD double sqrt(double x) { return sqrt_t(x); }
PHX_HD double rsqrt(double x) { return 1.0 / sqrt_t(x); }
PHX_HD double tanh(double x) { return tanh_t(x); }
PHX_HD double cos(double x) { return cos_t(x); }
}  // namespace fastm

}  // namespace phx
