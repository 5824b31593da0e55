// Block-AMR sampler: which leaf holds a point, and the plasma state there.
//
// Device layout of a snapshot (built once per snapshot, resident in HBM):
//   lb, dxc   [nleafs][3]              block origin and cell size per leaf (in the render precision)
//   prim      [nleafs][cells][8]       primitives per cell, 32 B per cell in FP32: a trilinear corner is two 128-bit
//                                      loads, and the i / i+1 corners of a row share one 64-B segment
//   fmap      [fd0][fd1][fd2] int32    leaf id per finest-level block slot: the per-level maps of the reference
//                                      (core/model/sampler.hpp:55-82, host/io/bhac_io.hpp:257-309) flattened so that a
//                                      lookup is one load instead of up to nlevels dependent loads; slot (i,j,k) holds
//                                      the first leaf met walking levels coarse -> fine, exactly the map walk's answer.
// Semantics follow the reference sampler (core/model/sampler.hpp:29-427): coordinate wrap with its -1e-6 shift of
// x2, half-open leaf test with a +-1e-9 nudge away from the equator, inclusive cache test, linear-scan fallback,
// block-local trilinear interpolation clamped at block faces, and the fluid derivation with the R_high/R_low
// temperature prescription and emission cuts.
#pragma once

#include "defs.cuh"
#include "kerr.cuh"

namespace phx {

template <class R, class PT>
struct SnapView {
  const R* lb;
  const R* dxc;
  const PT* prim;
  const int32_t* fmap;
  int32_t fd[3];
  int32_t nleafs, nlevels, cells;
  int32_t nx[3];
  R x_lo[4], x_hi[4];
  R w0[3];  // base-level block widths
  R iw0up[3];  // finest-level slots per unit of x: 2^(nlevels-1) / w0
  R a, hs, gam;
  // FP64 leaf geometry and spacetime constants, used by the mixed-precision path (FP64 geodesic, FP32 plasma stage)
  const double* lbd;
  const double* dxcd;
  double xlo_d[4], xhi_d[4], w0_d[3];
  double a_d, hs_d;

  PHX_HD SnapView<double, PT> fp64_view() const {
    SnapView<double, PT> v;
    v.lb = lbd;
    v.dxc = dxcd;
    v.prim = prim;
    v.fmap = fmap;
    for (int d = 0; d < 3; d++) {
      v.fd[d] = fd[d];
      v.nx[d] = nx[d];
      v.w0[d] = w0_d[d];
      v.iw0up[d] = double(1 << (nlevels - 1)) / w0_d[d];
    }
    for (int d = 0; d < 4; d++) {
      v.x_lo[d] = xlo_d[d];
      v.x_hi[d] = xhi_d[d];
    }
    v.nleafs = nleafs;
    v.nlevels = nlevels;
    v.cells = cells;
    v.a = a_d;
    v.hs = hs_d;
    v.gam = gam;
    v.lbd = lbd;
    v.dxcd = dxcd;
    v.a_d = a_d;
    v.hs_d = hs_d;
    return v;
  }
};

// Per-render plasma constants.
template <class R>
struct PlasmaView {
  R Ne, Bu, rhigh, rlow, ibc;
  R sigma_cut, thetae_min, thetae_max, rt_outer;
};

template <class R>
struct Fluid {
  R U[4], B[4];
  R n_e, Bmag, theta_e;
};

template <class R>
PHX_HD void wrap_coords(R x[4]) {
  const R TP = R(kTwoPi), PI = R(kPi);
  x[3] = fmod_t(x[3], TP);
  x[2] = fmod_t(x[2], PI) - R(1e-6);
  if (x[3] < R(0)) x[3] = TP + x[3];
  if (x[2] < R(0)) {
    x[2] = -x[2];
    x[3] = PI + x[3];
  }
}

template <class R, class PT>
PHX_HD bool outside_domain(const SnapView<R, PT>& s, const R x[4]) {
  return x[1] > s.x_hi[1] || x[1] < s.x_lo[1] || x[2] < s.x_lo[2] || x[2] > s.x_hi[2] || x[3] < s.x_lo[3] ||
         x[3] > s.x_hi[3];
}

template <class R>
PHX_HD R leaf_nudge(const R x[4]) {
  return x[2] > R(kHalfPi) ? R(-1e-9) : R(1e-9);
}

// fast: slot coordinates from the precomputed scale instead of the divisions (FP32; the caller verifies the
// candidate and retries with the divisions, so the leaf found is the same)
template <class R, class PT>
PHX_HD int find_leaf_map(const SnapView<R, PT>& s, const R x[4], R small, bool fast = false) {
  const R up = R(1 << (s.nlevels - 1));
  R fi, fj, fk;
  if (fast) {
    fi = (x[1] + small - s.x_lo[1]) * s.iw0up[0];
    fj = (x[2] + small - s.x_lo[2]) * s.iw0up[1];
    fk = (x[3] + small - s.x_lo[3]) * s.iw0up[2];
  } else {
    fi = (x[1] + small - s.x_lo[1]) / s.w0[0] * up;
    fj = (x[2] + small - s.x_lo[2]) / s.w0[1] * up;
    fk = (x[3] + small - s.x_lo[3]) / s.w0[2] * up;
  }
  if (fi < R(0) || fj < R(0) || fk < R(0)) return -1;
  const int i = (int)fi, j = (int)fj, k = (int)fk;
  if (i >= s.fd[0] || j >= s.fd[1] || k >= s.fd[2]) return -1;
#if defined(__CUDA_ARCH__)
  return __ldg(s.fmap + ((size_t)i * s.fd[1] + j) * s.fd[2] + k);
#else
  return s.fmap[((size_t)i * s.fd[1] + j) * s.fd[2] + k];
#endif
}

template <class T>
PHX_HD T ldg(const T* p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}

template <class R, class PT>
PHX_HD bool inside_leaf(const SnapView<R, PT>& s, int leaf, const R x[4], R small) {
  bool in = true;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const R lo = ldg(s.lb + 3 * leaf + d);
    const R hi = lo + R(s.nx[d]) * ldg(s.dxc + 3 * leaf + d);
    in = in && !(x[1 + d] + small < lo || x[1 + d] + small >= hi);
  }
  return in;
}

template <class R, class PT>
PHX_HD bool inside_cached(const SnapView<R, PT>& s, int leaf, const R x[4]) {
  bool in = true;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const R lo = ldg(s.lb + 3 * leaf + d);
    const R hi = lo + R(s.nx[d]) * ldg(s.dxc + 3 * leaf + d);
    in = in && !(x[1 + d] < lo || x[1 + d] > hi);
  }
  return in;
}

// Linear scan in leaf order: the first leaf whose half-open box holds the nudged point.  The rare fallback of
// find_leaf, kept out of line so that it costs the march loop no instruction-cache space.
template <class R, class PT>
PHX_HD_OUTLINE int find_leaf_scan(const SnapView<R, PT>& s, R x1, R x2, R x3, R small) {
  const R x[4] = {R(0), x1, x2, x3};
  for (int leaf = 0; leaf < s.nleafs; leaf++)
    if (inside_leaf(s, leaf, x, small)) return leaf;
  return -1;
}

// Counts of the rare slow path, for diagnostics (incremented by the caller when `scanned` is set).
template <class R, class PT>
PHX_HD int find_leaf(const SnapView<R, PT>& s, const R x[4], bool* scanned) {
  const R small = leaf_nudge(x);
  int cand = find_leaf_map(s, x, small, sizeof(R) == 4);
  if (cand >= 0 && inside_leaf(s, cand, x, small)) return cand;
  if constexpr (sizeof(R) == 4) {
    cand = find_leaf_map(s, x, small);
    if (cand >= 0 && inside_leaf(s, cand, x, small)) return cand;
  }
  const R eps = R(1e-6);
  if (cand < 0 && (x[1] < s.x_lo[1] - eps || x[1] > s.x_hi[1] + eps || x[2] < s.x_lo[2] - eps ||
                   x[2] > s.x_hi[2] + eps || x[3] < s.x_lo[3] - eps || x[3] > s.x_hi[3] + eps))
    return -1;
  *scanned = true;
  return find_leaf_scan(s, x[1], x[2], x[3], small);
}

// Cell and trilinear weights of point x inside one leaf: weights measured from the block's lower corner and clamped at
// the block faces (no ghost cells).  c: the lower corner cell (clamped into the block), del: weights of the upper
// corners.
template <class R, class PT, bool kFloorBy1000>
PHX_HD void cell_weights(const SnapView<R, PT>& s, int leaf, const R x[4], int c[3], R del[3]) {
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const R lb = ldg(s.lb + 3 * leaf + d), dx = ldg(s.dxc + 3 * leaf + d);
    // FP32: one reciprocal per axis (rounding-level difference; the interpolant is continuous across cells)
    const R idx = sizeof(R) == 4 ? fastm::rcp(dx) : R(0);
    const R u = sizeof(R) == 4 ? (x[1 + d] - lb) * idx : (x[1 + d] - lb) / dx;
    c[d] = (int)u;
    if (c[d] >= s.nx[d]) c[d] = s.nx[d] - 1;
    if (c[d] < 0) c[d] = 0;  // unreachable for finite points of the leaf; keeps every gather inside the block
    const int ix = kFloorBy1000 ? (int)(u + R(1000)) - 1000 : (int)floor_t(u);
    const R off = x[1 + d] - (R(ix) * dx + lb);
    del[d] = (ix < 0) ? R(0) : (ix > s.nx[d] - 2) ? R(1) : (sizeof(R) == 4 ? off * idx : off / dx);
  }
}

// Weighted sum of the 8 primitives over the 2x2x2 corners from cell c (corners past the block's last cell reuse it).
template <class R, class PT>
PHX_HD void gather_prims(const PT* prim, int cells, const int nx[3], int leaf, const int c[3], const R del[3],
                         R q[kNPrim]) {
  const int nx0 = nx[0], nx01 = nx[0] * nx[1];
  const int cip = c[0] + 1 < nx[0] ? c[0] + 1 : c[0];
  const int cjp = c[1] + 1 < nx[1] ? c[1] + 1 : c[1];
  const int ckp = c[2] + 1 < nx[2] ? c[2] + 1 : c[2];
  const R b1 = R(1) - del[0], b2 = R(1) - del[1], b3 = R(1) - del[2];
  const int ci[4] = {c[0], c[0], cip, cip};
  const int cj[4] = {c[1], cjp, c[1], cjp};
  const R wq[4] = {b1 * b2, b1 * del[1], del[0] * b2, del[0] * del[1]};
  const PT* base = prim + (size_t)leaf * cells * kNPrim;
#pragma unroll
  for (int a = 0; a < kNPrim; a++) q[a] = R(0);
#pragma unroll
  for (int z = 0; z < 2; z++) {
    const int ck = z ? ckp : c[2];
    const R wz = z ? del[2] : b3;
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const PT* p = base + (size_t)(ci[n] + cj[n] * nx0 + ck * nx01) * kNPrim;
      R v[kNPrim];
#if defined(__CUDA_ARCH__)
      if constexpr (sizeof(PT) == 4) {
        const float4 lo4 = __ldg(reinterpret_cast<const float4*>(p));
        const float4 hi4 = __ldg(reinterpret_cast<const float4*>(p) + 1);
        v[0] = lo4.x; v[1] = lo4.y; v[2] = lo4.z; v[3] = lo4.w;
        v[4] = hi4.x; v[5] = hi4.y; v[6] = hi4.z; v[7] = hi4.w;
      } else {
        const double2* p2 = reinterpret_cast<const double2*>(p);
#pragma unroll
        for (int h = 0; h < 4; h++) {
          const double2 t = __ldg(p2 + h);
          v[2 * h] = R(t.x);
          v[2 * h + 1] = R(t.y);
        }
      }
#else
      for (int a = 0; a < kNPrim; a++) v[a] = R(p[a]);
#endif
      const R w = wq[n] * wz;
#pragma unroll
      for (int a = 0; a < kNPrim; a++) q[a] += v[a] * w;
    }
  }
}

// Trilinear interpolation of the 8 primitives inside one leaf (sampler.hpp:211-291).
template <class R, class PT, bool kFloorBy1000>
PHX_HD void interp_prims(const SnapView<R, PT>& s, int leaf, const R x[4], R q[kNPrim]) {
  int c[3];
  R del[3];
  cell_weights<R, PT, kFloorBy1000>(s, leaf, x, c, del);
  gather_prims<R, PT>(s.prim, s.cells, s.nx, leaf, c, del, q);
}

// Fluid 4-velocity, magnetic 4-vector, |B| [G], n_e and Theta_e from the interpolated primitives; returns whether
// the point emits (sampler.hpp:305-376).  g / u: metric at x.
template <class R>
PHX_HD bool derive_fluid(const PlasmaView<R>& pv, R gam, R r, const Cov<R>& g, const Contra<R>& u, const R q[kNPrim],
                         Fluid<R>* fl) {
  const R smalll = R(1e-6);
  const R rho = q[kRho], uu = q[kUU];
  fl->n_e = rho * pv.Ne + smalll;
  // lapse alpha = 1 / sqrt(-g^tt), shift^1 = alpha^2 g^t1; the divisions are folded into reciprocals
  const R ialpha = fastm::sqrt(-u.tt);
  const R alpha = fastm::rcp(ialpha);  // FP32: hardware reciprocals and quotients here (2 ulp); FP64: exact
  const R shift1 = u.t1 * alpha * alpha;
  const R gv1 = q[kU1], gv2 = q[kU2], gv3 = q[kU3];
  const R gvv = g.x11 * gv1 * gv1 + R(2) * g.x13 * gv1 * gv3 + g.x22 * gv2 * gv2 + g.x33 * gv3 * gv3;
  const R lfac = fastm::sqrt(gvv + R(1));
  const R ilfac = fastm::rcp(lfac);
  const R V1 = gv1 * ilfac, V2 = gv2 * ilfac, V3 = gv3 * ilfac;
  const R ut = lfac * ialpha;
  fl->U[0] = ut;
  fl->U[1] = V1 * lfac - shift1 * ut;
  fl->U[2] = V2 * lfac;
  fl->U[3] = V3 * lfac;
  const R Bp1 = q[kB1], Bp2 = q[kB2], Bp3 = q[kB3];
  // B^t = lfac (gamma_ij Bp^i V^j) / alpha
  const R BV = Bp1 * (g.x11 * V1 + g.x13 * V3) + Bp2 * (g.x22 * V2) + Bp3 * (g.x13 * V1 + g.x33 * V3);
  fl->B[0] = lfac * BV * ialpha;
  fl->B[1] = (Bp1 + alpha * fl->B[0] * fl->U[1]) * ilfac;
  fl->B[2] = (Bp2 + alpha * fl->B[0] * fl->U[2]) * ilfac;
  fl->B[3] = (Bp3 + alpha * fl->B[0] * fl->U[3]) * ilfac;
  const R Bsq = fabs_t(dot(g, fl->B, fl->B)) + smalll;
  fl->Bmag = fastm::sqrt(Bsq) * pv.Bu;
  const R beta = fastm::div(uu * (gam - R(1)), R(0.5) * (Bsq + smalll));
  const R bb = beta * pv.ibc;
  const R b2 = bb * bb;
  const R ib2 = fastm::rcp(R(1) + b2);
  const R trat = (pv.rhigh * b2 + pv.rlow) * ib2;
  const R te_unit = fastm::div(R(1.0 / 3.0 * (cgs::m_proton / cgs::m_electron)), trat + R(1));
  fl->theta_e = fastm::div(uu, rho) * te_unit;
  if ((fastm::div(Bsq, rho + R(1e-20)) > pv.sigma_cut) || r > pv.rt_outer || fl->theta_e > pv.thetae_max ||
      fl->theta_e < pv.thetae_min) {
    fl->n_e = R(0);
    return false;
  }
  return true;
}

}  // namespace phx
