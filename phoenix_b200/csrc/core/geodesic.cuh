// Geodesic state and RK4 integrator of the raymarch.
//
// The state is (x^mu, k^mu, F^mu): position, wave vector and the parallel-transported camera polarization vector
// (NS = 12), or (x^mu, k^mu) alone (NS = 8) when the polarization comes from the Walker-Penrose constant (kerr.cuh).
// At FP32 it is carried as hi + lo float pairs updated by compensated (TwoSum) addition, and a ray in the southern
// hemisphere is integrated in the mirror coordinate pi - x2 so that x2 keeps its precision next to the south pole
// (the same device the reference's FP32 build uses, core/geometry/geodesic.hpp:200-256).  At FP64 the lo half is
// unused.  The right-hand side is phx::geodesic_accel (kerr.cuh).  The step-size rule is RAPTOR's, capped at a
// quarter of the current AMR cell (geodesic.hpp:267-292).
#pragma once

#include "defs.cuh"
#include "kerr.cuh"

namespace phx {

// Knuth TwoSum of hi + d folded into (hi, lo), then renormalised (fast two-sum).
template <class R>
PHX_HD void comp_add(R& hi, R& lo, R d) {
  const R s = hi + d;
  const R bb = s - hi;
  const R err = (hi - (s - bb)) + (d - bb);
  lo += err;
  const R s2 = s + lo;
  lo = lo - (s2 - s);
  hi = s2;
}

template <class R, int NS = 12>
struct GeoState {
  R hi[NS];  // x[0..3], k[4..7], F[8..11] (NS = 12)
  R lo[NS];  // compensation (FP32 only)
};

// Initial state from the FP64 camera photon and polarization vector (F unused when NS = 8).
template <class R, bool kComp, int NS>
PHX_HD void geo_init(GeoState<R, NS>& g, const double ph[8], const double F[4]) {
  double v[12];
  for (int i = 0; i < 8; i++) v[i] = ph[i];
  for (int i = 0; i < 4; i++) v[8 + i] = F[i];
  for (int i = 0; i < NS; i++) {
    g.hi[i] = R(v[i]);
    g.lo[i] = kComp ? R(v[i] - (double)g.hi[i]) : R(0);
  }
}

template <class R, bool kComp, int NS>
PHX_HD R geo_get(const GeoState<R, NS>& g, int i) {
  return kComp ? g.hi[i] + g.lo[i] : g.hi[i];
}

// x2 measured from the nearer pole where the integrator folds (FP32), else x2 itself.
template <class R, bool kComp, int NS>
PHX_HD R pole_x2(const GeoState<R, NS>& g) {
  if (kComp && g.hi[2] > R(kHalfPi)) {
    const R pi_hi = R(kPi), pi_lo = R(kPi - (double)R(kPi));
    return (pi_hi - g.hi[2]) + (pi_lo - g.lo[2]);
  }
  return g.hi[2] + (kComp ? g.lo[2] : R(0));
}

// exp(d) by its Taylor series to d^N in Horner form: N = 11 for |d| <= 0.1 (truncation below 3e-21 relative), N = 7
// for |d| <= 0.025 (below 4e-18).
template <class T, int N = 11>
PHX_HD T exp_small(T d) {
  if constexpr (N == 7) {
    // Estrin's form: three levels of independent products instead of a seven-deep Horner chain
    const T d2 = d * d, d4 = d2 * d2;
    const T q0 = (T(1) + d) + d2 * (T(1.0 / 2.0) + d * T(1.0 / 6.0));
    const T q1 = (T(1.0 / 24.0) + d * T(1.0 / 120.0)) + d2 * (T(1.0 / 720.0) + d * T(1.0 / 5040.0));
    return q0 + d4 * q1;
  } else {
    T e = T(1);
#pragma unroll
    for (int n = N; n >= 1; n--) e = T(1) + d * T(1.0 / n) * e;
    return e;
  }
}

// Largest stage offset in x1 and x2 that the shifted stages take by the short series (exp_small<7>, sincos_tiny).
// A step changes x1 and x2 by at most about `stepsize` = 0.01 (the step-size rule), so the bound leaves 2.5x margin;
// a larger offset (or |hslope| > 0.5, where the theta shift could exceed sincos_tiny's range) evaluates the point
// directly.
constexpr double kShiftMax = 0.025;

// One stage's derivatives with the point evaluated directly (exp and sincos of the stage's own x1, x2): the shifted
// stages' fallback for offsets beyond kShiftMax.  Out of line (arguments and results by value): the shifted form covers
// nearly every stage, so this second copy of the metric, its exp and its sincos stays out of the march loop (measured on
// B200: the same step time as inlined, two registers fewer at the 168-register cap).
template <class R>
struct StagePoint {
  R a, hs, x1, x2, k[4], F[4];
};
template <class R>
struct StageDeriv {
  R dk[4], dF[4];
};

template <class R, bool kF>
PHX_HD_OUTLINE StageDeriv<R> geodesic_accel_direct(StagePoint<R> p) {
  StageDeriv<R> o;
#pragma unroll
  for (int i = 0; i < 4; i++) o.dF[i] = R(0);
  geodesic_accel<R, kF>(p.a, p.hs, p.x1, p.x2, p.k, p.F, o.dk, o.dF);
  return o;
}

// One classical RK4 step of length dt.  Stage sums are kept as (d0 + d3) and (d1 + d2) so that the update
// ((d0 + d3) + 2 (d1 + d2)) dt/6 needs two 12-vectors instead of four (kShift: one running sum).  The stage loop is deliberately not unrolled:
// one copy of the stage body (metric, derivatives, both Christoffel contractions) keeps the march loop small enough
// for the instruction cache, which four unrolled copies overflow.
// kShift (uncompensated state only; the mixed mode's FP64 geodesic): each stage's exp(x1) and sincos(x2) come from the
// step's starting point and short series of the stage offset (exp_small<7>, sincos_tiny: exact to rounding for
// offsets up to kShiftMax), one exp and one sincos per step instead of four, and the geometry's reciprocals are the
// Newton-refined FP64 ones (fastm::rcp_nr); a stage whose offset is larger evaluates the point directly.
template <class R, bool kComp, int NS, bool kShift = false>
PHX_HD void rk4_step(R a, R hs, GeoState<R, NS>& g, R dt) {
  constexpr bool kF = NS == 12;
  static_assert(!(kShift && kComp), "the shifted stages need an uncompensated state");
  const R pi_hi = R(kPi), pi_lo = R(kPi - (double)R(kPi));
  const bool south = kComp && g.hi[2] > R(kHalfPi);
  R e0 = R(0), sx0 = R(0), cx0 = R(0), s2x0 = R(0), st0 = R(0), ct0 = R(0);
  if constexpr (kShift) {
    e0 = exp_t(g.hi[1]);
    sincos_t(g.hi[2], &sx0, &cx0);
    // theta at the start, theta0 = x2 + (h/2) sin 2x2: each stage's theta follows from a small shift of it
    s2x0 = R(2) * sx0 * cx0;
    sincos_t(g.hi[2] + R(0.5) * hs * s2x0, &st0, &ct0);
  }
  R inc[NS], s03[NS], s12[NS];
#pragma unroll
  for (int i = 0; i < NS; i++) inc[i] = R(0);
#pragma unroll 1
  for (int q = 0; q < 4; q++) {
    R y[12];
#pragma unroll
    for (int i = 0; i < NS; i++) y[i] = kComp ? g.hi[i] + (g.lo[i] + inc[i]) : g.hi[i] + inc[i];
    if (south) {
      y[2] = (pi_hi - g.hi[2]) + ((pi_lo - g.lo[2]) - inc[2]);
      y[6] = -y[6];
      if constexpr (kF) y[10] = -y[10];
    }
    R d[12];
    d[0] = y[4];
    d[1] = y[5];
    d[2] = y[6];
    d[3] = y[7];
    if constexpr (kShift) {
      const R d1 = inc[1], d2 = inc[2];
      if (fabs_t(d1) <= R(kShiftMax) && fabs_t(d2) <= R(kShiftMax) && fabs_t(hs) <= R(0.5)) {
        R sd, cd;
        sincos_tiny(d2, &sd, &cd);
        const R sx = sx0 * cd + cx0 * sd, cx = cx0 * cd - sx0 * sd;
        const R s2x = R(2) * sx * cx, c2x = (cx - sx) * (cx + sx);
        // theta - theta0 = d2 + (h/2)(sin 2x2 - sin 2x2_0): |.| <= (1 + |h|) kShiftMax <= 0.0375
        R sdt, cdt;
        sincos_tiny(d2 + R(0.5) * hs * (s2x - s2x0), &sdt, &cdt);
        const KerrPt<R> p = kerr_point_theta<R, true>(a, hs, e0 * exp_small<R, 7>(d1), s2x, c2x,
                                                      st0 * cdt + ct0 * sdt, ct0 * cdt - st0 * sdt);
        geodesic_accel_at<R, kF, true>(a, p, y + 4, y + 8, d + 4, d + 8);
      } else {
        StagePoint<R> sp;
        sp.a = a;
        sp.hs = hs;
        sp.x1 = y[1];
        sp.x2 = y[2];
#pragma unroll
        for (int i = 0; i < 4; i++) {
          sp.k[i] = y[4 + i];
          sp.F[i] = kF ? y[8 + i] : R(0);
        }
        const StageDeriv<R> sd = geodesic_accel_direct<R, kF>(sp);
#pragma unroll
        for (int i = 0; i < 4; i++) {
          d[4 + i] = sd.dk[i];
          if constexpr (kF) d[8 + i] = sd.dF[i];
        }
      }
    } else {
      geodesic_accel<R, kF>(a, hs, y[1], y[2], y + 4, y + 8, d + 4, d + 8);
    }
    if (south) {
      d[2] = -d[2];
      d[6] = -d[6];
      if constexpr (kF) d[10] = -d[10];
    }
    if constexpr (kShift) {
      // one running sum d0 + 2 d1 + 2 d2 + d3 (one 8-vector of doubles fewer live through the stages)
#pragma unroll
      for (int i = 0; i < NS; i++) s03[i] = (q == 0 ? R(0) : s03[i]) + (q == 1 || q == 2 ? R(2) : R(1)) * d[i];
    } else {
#pragma unroll
      for (int i = 0; i < NS; i++) {
        if (q == 0) s03[i] = d[i];
        if (q == 1) s12[i] = d[i];
        if (q == 2) s12[i] += d[i];
        if (q == 3) s03[i] += d[i];
      }
    }
    if (q < 3) {
      const R wdt = (q == 2 ? R(1) : R(0.5)) * dt;
#pragma unroll
      for (int i = 0; i < NS; i++) inc[i] = wdt * d[i];
    }
  }
  const R dt6 = dt / R(6);
#pragma unroll
  for (int i = 0; i < NS; i++) {
    const R du = (kShift ? s03[i] : s03[i] + R(2) * s12[i]) * dt6;
    if (kComp) {
      comp_add(g.hi[i], g.lo[i], du);
    } else {
      g.hi[i] += du;
    }
  }
}

// RAPTOR step size (negative: the ray runs backwards from the camera), capped by a quarter of the AMR cell.
// dxc == nullptr means no cap.
template <class R>
PHX_HD R step_size(R stepsize, R x2, const R k[4], const R* dxc, R tiny, R big) {
  const R dlx1 = stepsize / (fabs_t(k[1]) + tiny);
  const R dlx2 = stepsize * fmin_t(x2, R(kPi) - x2) / (fabs_t(k[2]) + tiny);
  const R dlx3 = stepsize / (fabs_t(k[3]) + tiny);
  const R i1 = R(1) / (fabs_t(dlx1) + tiny);
  const R i2 = R(1) / (fabs_t(dlx2) + tiny);
  const R i3 = R(1) / (fabs_t(dlx3) + tiny);
  R grid = big;
  if (dxc) {
    const R s1 = dxc[0] / (fabs_t(k[1]) + tiny);
    const R s2 = dxc[1] / (fabs_t(k[2]) + tiny);
    const R s3 = dxc[2] / (fabs_t(k[3]) + tiny);
    const R is1 = R(1) / (fabs_t(s1) + tiny);
    const R is2 = R(1) / (fabs_t(s2) + tiny);
    const R is3 = R(1) / (fabs_t(s3) + tiny);
    grid = R(1) / (is1 + is2 + is3) / R(4);
  }
  return -fmin_t(R(1) / (i1 + i2 + i3), grid);
}

// The same rule with the reciprocals folded (FP32 paths): 1 / (stepsize / |k| + tiny) -> |k| / stepsize and
// 1 / (dxc / |k| + tiny) -> |k| / dxc with the leaf's inverse cell sizes idxc, so that two divisions remain instead of
// twelve.  Equal to step_size up to rounding; the pole term keeps the reference's 1 / tiny limit at x2 = 0.
// kNR: the mixed mode's FP64 reciprocals (geo_rcp, geo_div).
template <class R, bool kNR = false>
PHX_HD R step_size_fast(R stepsize, R inv_stepsize, R x2, const R k[4], const R* idxc, R tiny, R big) {
  const R a1 = fabs_t(k[1]) + tiny, a2 = fabs_t(k[2]) + tiny, a3 = fabs_t(k[3]) + tiny;
  const R m = fmin_t(x2, R(kPi) - x2);
  const R i2 = fmin_t(geo_div<R, kNR>(a2, stepsize * m), R(1) / tiny);  // m = 0: the reference's 1 / tiny
  const R sum = (a1 + a3) * inv_stepsize + i2;
  R grid = big;
  if (idxc) grid = geo_div<R, kNR>(R(0.25), a1 * idxc[0] + a2 * idxc[1] + a3 * idxc[2]);
  return -fmin_t(geo_rcp<R, kNR>(sum), grid);
}

// Re-solve k^t from the spatial components so that g_{mu nu} k^mu k^nu = 0 (the larger root), as the reference
// does for each plasma sample (geodesic.hpp:297-306, called from core/render/pixel.hpp:69-71).
template <class R>
PHX_HD void normalize_null(const Cov<R>& g, R k[4]) {
  const R aa = g.tt;
  const R beta = -(g.t1 * k[1] + g.t3 * k[3]) / aa;
  const R gam = -(g.x11 * k[1] * k[1] + R(2) * g.x13 * k[1] * k[3] + g.x22 * k[2] * k[2] + g.x33 * k[3] * k[3]) / aa;
  k[0] = beta + sqrt_t(beta * beta + gam);
}

}  // namespace phx
