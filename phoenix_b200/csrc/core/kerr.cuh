// Kerr spacetime in modified Kerr-Schild coordinates of the BHAC flavour (MKS-BHAC):
//   x0 = t,  x1 = ln r,  x2 with theta = x2 + (h/2) sin(2 x2),  x3 = phi.
// The reference renderer evaluates the same metric (core/geometry/metric.hpp:26-221) and the geodesic equation in a
// closed-form Christoffel contraction (core/geometry/geodesic.hpp:81-195).  Here the metric is kept as its seven
// non-zero covariant components and six non-zero contravariant ones, and the geodesic right-hand side is formed from
// the analytic first derivatives d g_{mu nu} / d x1 and d g_{mu nu} / d x2 (the metric depends on x1, x2 only):
//   Gamma^mu(U, V) = g^{mu nu} a_nu,
//   a_nu = 1/2 [ (U^1 D1 + U^2 D2)_{nu b} V^b + (V^1 D1 + V^2 D2)_{nu b} U^b - delta_{nu 1} U.D1.V - delta_{nu 2} U.D2.V ]
// which is the textbook Gamma_{nu ab} = (d_a g_{nu b} + d_b g_{nu a} - d_nu g_{ab}) / 2 with the vanishing t- and
// phi-derivatives dropped.  Everything lives in registers: ~60 flops of geometry and ~110 FMAs of contraction for the
// two accelerations (k.k and k.F) an RK4 stage needs.
#pragma once

#include "defs.cuh"

namespace phx {

// Geometry of one point: everything the metric, its inverse and its derivatives share.
template <class T>
struct KerrPt {
  T r;    // exp(x1)
  T s;    // sin(theta)
  T c;    // cos(theta)
  T s2;   // sin^2(theta)
  T tp;   // d theta / d x2
  T tpp;  // d^2 theta / d x2^2
  T sig;   // Sigma = r^2 + a^2 cos^2(theta)
  T isig;  // 1 / Sigma
  T q;     // 2 r / Sigma
};

// Non-zero covariant components g_{mu nu} (symmetric).
template <class T>
struct Cov {
  T tt, t1, t3, x11, x13, x22, x33;
};

// Non-zero contravariant components g^{mu nu} (symmetric; g^{t3} = g^{t2} = 0).
template <class T>
struct Contra {
  T tt, t1, x11, x13, x22, x33;
};

// sin d and cos d for |d| <= 0.5 from their Taylor series in Horner form, truncated where the next term is below the
// type's rounding (FP32: 5 terms each, error < 3e-10; FP64: 8 terms each, error < 1e-18).
template <class T>
PHX_HD void sincos_small(T d, T* sn, T* cs) {
  const T z = d * d;
  T s, c;
  if constexpr (sizeof(T) == 4) {
    s = T(1) - z * T(1.0 / 72.0);
    s = T(1) - z * T(1.0 / 42.0) * s;
    s = T(1) - z * T(1.0 / 20.0) * s;
    s = T(1) - z * T(1.0 / 6.0) * s;
    c = T(1) - z * T(1.0 / 56.0);
    c = T(1) - z * T(1.0 / 30.0) * c;
    c = T(1) - z * T(1.0 / 12.0) * c;
    c = T(1) - z * T(1.0 / 2.0) * c;
  } else {
    s = T(1) - z * T(1.0 / 210.0);
    s = T(1) - z * T(1.0 / 156.0) * s;
    s = T(1) - z * T(1.0 / 110.0) * s;
    s = T(1) - z * T(1.0 / 72.0) * s;
    s = T(1) - z * T(1.0 / 42.0) * s;
    s = T(1) - z * T(1.0 / 20.0) * s;
    s = T(1) - z * T(1.0 / 6.0) * s;
    c = T(1) - z * T(1.0 / 182.0);
    c = T(1) - z * T(1.0 / 132.0) * c;
    c = T(1) - z * T(1.0 / 90.0) * c;
    c = T(1) - z * T(1.0 / 56.0) * c;
    c = T(1) - z * T(1.0 / 30.0) * c;
    c = T(1) - z * T(1.0 / 12.0) * c;
    c = T(1) - z * T(1.0 / 2.0) * c;
  }
  *sn = d * s;
  *cs = c;
}

// Reciprocal and quotient of the geometry code: the type's fast form (FP32: hardware reciprocal; FP64: exact division),
// or with kNR (the mixed mode's FP64 geodesic) the Newton-refined FP64 reciprocal.
template <class T, bool kNR>
PHX_HD T geo_rcp(T x) {
  if constexpr (kNR && sizeof(T) == 8) {
    return fastm::rcp_nr(x);
  } else {
    return fastm::rcp(x);
  }
}

template <class T, bool kNR>
PHX_HD T geo_div(T a, T b) {
  if constexpr (kNR && sizeof(T) == 8) {
    return a * fastm::rcp_nr(b);
  } else {
    return fastm::div(a, b);
  }
}

// sin d and cos d for |d| <= 0.0375 in FP64: four Taylor terms each (truncation below 2e-17 and 1e-16 relative),
// summed in Estrin's form (two levels of independent products instead of a three-deep Horner chain).
template <class T>
PHX_HD void sincos_tiny(T d, T* sn, T* cs) {
  const T z = d * d, z2 = z * z;
  const T s = (T(1) - z * T(1.0 / 6.0)) + z2 * (T(1.0 / 120.0) - z * T(1.0 / 5040.0));
  const T c = (T(1) - z * T(1.0 / 2.0)) + z2 * (T(1.0 / 24.0) - z * T(1.0 / 720.0));
  *sn = d * s;
  *cs = c;
}

// The rest of the geometry once r, sin 2x2, cos 2x2 and sin, cos of theta are known.
template <class T, bool kNR = false>
PHX_HD KerrPt<T> kerr_point_theta(T a, T hs, T r, T s2x, T c2x, T st, T ct) {
  KerrPt<T> p;
  p.r = r;
  p.tp = T(1) + hs * c2x;
  p.tpp = T(-2) * hs * s2x;
  p.s = st;
  p.c = ct;
  p.s2 = p.s * p.s;
  p.sig = p.r * p.r + a * a * p.c * p.c;
  p.isig = geo_rcp<T, kNR>(p.sig);  // FP32: hardware reciprocal (2 ulp), FP64: exact division or Newton-refined
  p.q = T(2) * p.r * p.isig;
  return p;
}

// Geometry at (r, x2) when r = exp(x1) and sin x2, cos x2 are already known.
template <class T, bool kNR = false>
PHX_HD KerrPt<T> kerr_point_rsc(T a, T hs, T r, T x2, T sx, T cx) {
  // sin 2x2, cos 2x2 from sin x2, cos x2 (double-angle identities)
  const T s2x = T(2) * sx * cx, c2x = (cx - sx) * (cx + sx);
  const T d = T(0.5) * hs * s2x;  // theta = x2 + d
  T st, ct;
  if (fabs_t(hs) <= T(1)) {
    // sin, cos of theta by angle addition: |d| <= |hs| / 2 <= 0.5 needs no second sincos
    T sd, cd;
    sincos_small(d, &sd, &cd);
    st = sx * cd + cx * sd;
    ct = cx * cd - sx * sd;
  } else {
    sincos_t(x2 + d, &st, &ct);
  }
  return kerr_point_theta<T, kNR>(a, hs, r, s2x, c2x, st, ct);
}

// Geometry at (r, x2) when r = exp(x1) is already known.
template <class T>
PHX_HD KerrPt<T> kerr_point_r(T a, T hs, T r, T x2) {
  T sx, cx;
  sincos_t(x2, &sx, &cx);
  return kerr_point_rsc(a, hs, r, x2, sx, cx);
}

template <class T>
PHX_HD KerrPt<T> kerr_point(T a, T hs, T x1, T x2) {
  return kerr_point_r(a, hs, exp_t(x1), x2);
}

template <class T>
PHX_HD Cov<T> cov_metric(const KerrPt<T>& p, T a) {
  Cov<T> g;
  const T opq = T(1) + p.q;
  g.tt = p.q - T(1);
  g.t1 = p.q * p.r;
  g.t3 = -a * p.s2 * p.q;
  g.x11 = opq * p.r * p.r;
  g.x13 = -a * p.s2 * opq * p.r;
  g.x22 = p.sig * p.tp * p.tp;
  g.x33 = p.s2 * (p.sig + a * a * p.s2 * opq);
  return g;
}

template <class T, bool kNR = false>
PHX_HD Contra<T> contra_metric(const KerrPt<T>& p, T a) {
  Contra<T> u;
  const T isig = p.isig;
  const T ir = geo_rcp<T, kNR>(p.r);
  const T tp2 = p.tp * p.tp;
  const T iprod = isig * geo_rcp<T, kNR>(tp2 * p.s2);  // one reciprocal for both 1 / theta'^2 and 1 / sin^2
  u.tt = -(T(1) + p.q);
  u.t1 = T(2) * isig;
  u.x11 = isig * ((p.r - T(2)) * p.r + a * a) * ir * ir;
  u.x13 = a * isig * ir;
  u.x22 = iprod * p.s2;
  u.x33 = iprod * tp2;
  return u;
}

// Inner product of a lowered vector with a vector.
template <class T>
PHX_HD T dot4(const T Ud[4], const T V[4]) {
  return Ud[0] * V[0] + Ud[1] * V[1] + Ud[2] * V[2] + Ud[3] * V[3];
}

// g_{mu nu} U^mu V^nu
template <class T>
PHX_HD T dot(const Cov<T>& g, const T U[4], const T V[4]) {
  return g.tt * U[0] * V[0] + g.t1 * (U[0] * V[1] + U[1] * V[0]) + g.t3 * (U[0] * V[3] + U[3] * V[0]) +
         g.x11 * U[1] * V[1] + g.x13 * (U[1] * V[3] + U[3] * V[1]) + g.x22 * U[2] * V[2] + g.x33 * U[3] * V[3];
}

// out = M V for a symmetric matrix with the metric's sparsity pattern (works for Cov and the derivative sets).
template <class T, class M>
PHX_HD void symv(const M& m, const T V[4], T out[4]) {
  out[0] = m.tt * V[0] + m.t1 * V[1] + m.t3 * V[3];
  out[1] = m.t1 * V[0] + m.x11 * V[1] + m.x13 * V[3];
  out[2] = m.x22 * V[2];
  out[3] = m.t3 * V[0] + m.x13 * V[1] + m.x33 * V[3];
}

template <class T>
PHX_HD void raise(const Contra<T>& u, const T Vd[4], T out[4]) {
  out[0] = u.tt * Vd[0] + u.t1 * Vd[1];
  out[1] = u.t1 * Vd[0] + u.x11 * Vd[1] + u.x13 * Vd[3];
  out[2] = u.x22 * Vd[2];
  out[3] = u.x13 * Vd[1] + u.x33 * Vd[3];
}

// Full 4x4 covariant metric (host-side tools and the decode path; the render path uses Cov directly).
template <class T>
PHX_HD void metric_dd_full(T a, T hs, T x1, T x2, T g[4][4]) {
  const KerrPt<T> p = kerr_point(a, hs, x1, x2);
  const Cov<T> c = cov_metric(p, a);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) g[i][j] = T(0);
  g[0][0] = c.tt;
  g[0][1] = g[1][0] = c.t1;
  g[0][3] = g[3][0] = c.t3;
  g[1][1] = c.x11;
  g[1][3] = g[3][1] = c.x13;
  g[2][2] = c.x22;
  g[3][3] = c.x33;
}

template <class T>
PHX_HD void metric_uu_full(T a, T hs, T x1, T x2, T g[4][4]) {
  const KerrPt<T> p = kerr_point(a, hs, x1, x2);
  const Contra<T> c = contra_metric(p, a);
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++) g[i][j] = T(0);
  g[0][0] = c.tt;
  g[0][1] = g[1][0] = c.t1;
  g[1][1] = c.x11;
  g[1][3] = g[3][1] = c.x13;
  g[2][2] = c.x22;
  g[3][3] = c.x33;
}

// First derivatives of the covariant metric with respect to x1 (D1) and x2 (D2).
template <class T>
PHX_HD void cov_derivs(const KerrPt<T>& p, T a, Cov<T>* D1, Cov<T>* D2) {
  const T a2 = a * a, r = p.r, r2 = r * r, q = p.q, opq = T(1) + q;
  // x1: dr/dx1 = r, dSigma/dx1 = 2 r^2, dq/dx1 = q (1 - 2 r^2 / Sigma)
  const T q1 = q * (T(1) - T(2) * r2 * p.isig);
  D1->tt = q1;
  D1->t1 = (q1 + q) * r;
  D1->t3 = -a * p.s2 * q1;
  D1->x11 = (q1 + T(2) * opq) * r2;
  D1->x13 = -a * p.s2 * (q1 + opq) * r;
  D1->x22 = T(2) * r2 * p.tp * p.tp;
  D1->x33 = p.s2 * (T(2) * r2 + a2 * p.s2 * q1);
  // x2: d(sin^2)/dx2 = 2 s c theta', dSigma/dx2 = -2 a^2 s c theta', dq/dx2 = -q dSigma / Sigma
  const T sc2 = T(2) * p.s * p.c * p.tp;
  const T sig2 = -a2 * sc2;
  const T q2 = -q * sig2 * p.isig;
  D2->tt = q2;
  D2->t1 = q2 * r;
  D2->t3 = -a * (sc2 * q + p.s2 * q2);
  D2->x11 = q2 * r2;
  D2->x13 = -a * r * (sc2 * opq + p.s2 * q2);
  D2->x22 = sig2 * p.tp * p.tp + T(2) * p.sig * p.tp * p.tpp;
  D2->x33 = sc2 * (p.sig + a2 * p.s2 * opq) + p.s2 * (sig2 + a2 * (sc2 * opq + p.s2 * q2));
}

// Right-hand side of the geodesic equation and of the parallel transport of a polarization vector F:
//   dk^mu/dl = -Gamma^mu_ab k^a k^b,   dF^mu/dl = -Gamma^mu_ab k^a F^b.
// kF = false: k only (F and dF are not touched; the polarization then comes from the Walker-Penrose constant).
template <class T, bool kF = true, bool kNR = false>
PHX_HD void geodesic_accel_at(T a, const KerrPt<T>& p, const T k[4], const T F[4], T dk[4], T dF[4]) {
  Cov<T> D1, D2;
  cov_derivs(p, a, &D1, &D2);
  const Contra<T> u = contra_metric<T, kNR>(p, a);
  T Pk[4], Qk[4];
  symv(D1, k, Pk);  // D1 k
  symv(D2, k, Qk);  // D2 k
  const T kD1k = Pk[0] * k[0] + Pk[1] * k[1] + Pk[2] * k[2] + Pk[3] * k[3];
  const T kD2k = Qk[0] * k[0] + Qk[1] * k[1] + Qk[2] * k[2] + Qk[3] * k[3];
  T ak[4];
  for (int n = 0; n < 4; n++) ak[n] = k[1] * Pk[n] + k[2] * Qk[n];
  ak[1] -= T(0.5) * kD1k;
  ak[2] -= T(0.5) * kD2k;
  T gk[4];
  raise(u, ak, gk);
  for (int n = 0; n < 4; n++) dk[n] = -gk[n];
  if constexpr (kF) {
    T PF[4], QF[4];
    symv(D1, F, PF);  // D1 F
    symv(D2, F, QF);  // D2 F
    const T kD1F = Pk[0] * F[0] + Pk[1] * F[1] + Pk[2] * F[2] + Pk[3] * F[3];
    const T kD2F = Qk[0] * F[0] + Qk[1] * F[1] + Qk[2] * F[2] + Qk[3] * F[3];
    T aF[4];
    for (int n = 0; n < 4; n++) aF[n] = T(0.5) * (k[1] * PF[n] + k[2] * QF[n] + F[1] * Pk[n] + F[2] * Qk[n]);
    aF[1] -= T(0.5) * kD1F;
    aF[2] -= T(0.5) * kD2F;
    T gF[4];
    raise(u, aF, gF);
    for (int n = 0; n < 4; n++) dF[n] = -gF[n];
  }
}

template <class T, bool kF = true>
PHX_HD void geodesic_accel(T a, T hs, T x1, T x2, const T k[4], const T F[4], T dk[4], T dF[4]) {
  geodesic_accel_at<T, kF>(a, kerr_point(a, hs, x1, x2), k, F, dk, dF);
}

// Walker-Penrose constant of a null geodesic k with a polarization vector f (k.f = 0), in the MKS-BHAC coordinates of
// this file (Kerr-Schild t and phi, r = exp(x1), theta(x2)):
//   kappa = (r + i a cos(theta)) (sin(theta) B - i A),
//   A = R(k) E(f) - R(f) E(k),   B = T(k) P(f) - T(f) P(k),
//   R(v) = dr(v) = r v^1,   T(v) = dtheta(v) = theta' v^2,   E(v) = v^t - a sin^2(theta) v^phi,
//   P(v) = (r^2 + a^2) v^phi - a v^t - a dr(v).
// Y(k, f) = Re kappa and h(k, f) = -Im kappa are the contractions of k and f with Kerr's Killing-Yano 2-form
// Y = a cos(theta) dr ^ (dt - a sin^2 dphi) + r sin(theta) dtheta ^ ((r^2 + a^2) dphi - a dt) and its Hodge dual, the
// closed conformal Killing-Yano form h = db, b = [(r^2 + a^2 sin^2) dt - a sin^2 (r^2 + a^2) dphi] / 2 (Boyer-Lindquist
// forms; the Kerr-Schild change of t and phi adds the -a dr in P).  Both are constant along the geodesic when f is
// parallel-transported (Walker & Penrose 1970; Chandrasekhar 1983 sec. 63), so kappa taken once at the camera fixes
// the transported polarization direction at every later point.
template <class T>
struct WPForms {
  T A, B;
};

template <class T>
PHX_HD WPForms<T> wp_forms(T a, const KerrPt<T>& p, const T k[4], const T f[4]) {
  const T rr = p.r * p.r + a * a;
  const T Rk = p.r * k[1], Rf = p.r * f[1];
  const T Tk = p.tp * k[2], Tf = p.tp * f[2];
  const T Ek = k[0] - a * p.s2 * k[3], Ef = f[0] - a * p.s2 * f[3];
  const T Pk = rr * k[3] - a * k[0] - a * Rk, Pf = rr * f[3] - a * f[0] - a * Rf;
  return {Rk * Ef - Rf * Ek, Tk * Pf - Tf * Pk};
}

template <class T>
PHX_HD void walker_penrose(T a, const KerrPt<T>& p, const T k[4], const T f[4], T kappa[2]) {
  const WPForms<T> w = wp_forms(a, p, k, f);
  const T wre = p.s * w.B, wim = -w.A, ac = a * p.c;
  kappa[0] = p.r * wre - ac * wim;
  kappa[1] = p.r * wim + ac * wre;
}

// Components (C, S), up to one common factor, of the transported polarization vector on an orthonormal screen pair
// (perp, para) orthogonal to k at point p, from the Walker-Penrose constant: f = C perp + S para + alpha k, A and B are
// linear in f with A(k) = B(k) = 0, and kappa (r - i a cos) = (r^2 + a^2 cos^2) (sin B(f) - i A(f)), a 2x2 system in
// (C, S) solved by Cramer's rule without the division (cos 2 chi and sin 2 chi need only the ratio).
template <class T>
PHX_HD void wp_components(T a, const KerrPt<T>& p, const T k[4], const T perp[4], const T para[4], const T kappa[2],
                          T* C, T* S) {
  const WPForms<T> fp = wp_forms(a, p, k, perp), fq = wp_forms(a, p, k, para);
  const T ac = a * p.c;
  const T wre = kappa[0] * p.r + kappa[1] * ac, wim = kappa[1] * p.r - kappa[0] * ac;
  *C = -wre * fq.A - p.s * fq.B * wim;
  *S = p.s * fp.B * wim + fp.A * wre;
}

}  // namespace phx
