// One ray of the raymarch as a resumable state machine.
//
// Ray::advance() performs one pass of the reference's per-pixel loop (core/render/pixel.hpp:179-211): view the
// state -> liveness test -> leaf lookup -> a plasma sample -> theta turning points -> grid-capped step size -> RK4
// step.  FP64 processes the previous point's sample, as the reference does; the FP32 and mixed paths process this
// point's (see advance() for why both give the same samples).
// Because the state is explicit, a warp can retire a finished ray and start a new one in the same lane while its
// neighbours keep marching (the kernels' partial refill, refill_lanes < 32), as well as refill all its lanes at once.
//
// Each mode has two precisions: G of the geodesic (state, RK4, step size, leaf placement) and R of the plasma stage
// (interpolated fluid, synchrotron coefficients, transfer operator).
//   FP32   G = R = float after the FP64 camera set-up; compensated (hi, lo) geodesic state with south-pole folding;
//          deviation-form transfer operator.
//   FP64   G = R = double.
//   Mixed  G = double, R = float, plus FP64 islands of the plasma stage: the null-condition renormalisation of each
//          sample's wave vector, the segment operator where h max|K| > tau_fp64 (large optical / Faraday depth per
//          segment) and Kahan summation of the Stokes vector.  The geodesic is FP64 because the reference's
//          interpolation is block-local (no ghost cells): the sampled fluid jumps where a ray crosses a block face, so a
//          sample that the FP32 trajectory error (1e-7 .. 1e-6 in x after thousands of steps) carries across a face
//          picks up the neighbour block's values.  With an FP64 trajectory and FP64 step sizes the samples sit where
//          the FP64 oracle's do.
#pragma once

#include <type_traits>

#include "camera.cuh"
#include "defs.cuh"
#include "geodesic.cuh"
#include "kerr.cuh"
#include "sampler.cuh"
#include "synchro.cuh"
#include "transfer.cuh"

namespace phx {

enum class Mode : int { kFP32 = 0, kFP64 = 1, kMixed = 2 };

template <Mode M>
struct Policy;
// R: plasma-stage precision; G: geodesic precision; kComp: compensated (hi, lo) geodesic state; kShift: RK4 stages
// take exp(x1) and sincos(x2) from the step's start point and short series of the stage offset.
template <>
struct Policy<Mode::kFP32> {
  using R = float;
  using G = float;
  static constexpr bool kComp = true, kMixed = false, kShift = false;
};
template <>
struct Policy<Mode::kFP64> {
  using R = double;
  using G = double;
  static constexpr bool kComp = false, kMixed = false, kShift = false;
};
template <>
struct Policy<Mode::kMixed> {
  using R = float;
  using G = double;
  static constexpr bool kComp = false, kMixed = true, kShift = true;
};

// Integration limits and step-size constants in the precision G of a geodesic.
template <class G>
struct StepConsts {
  G stepsize, inv_stepsize, r_out, cut_in, rt_outer, tiny, big;
};

// Render-wide constants (one image: camera, integration, plasma and frequencies).
template <class R>
struct RenderConsts {
  int32_t W, H, nfreqs, max_steps, max_order;
  double fov_x, fov_y, cos_pa, sin_pa;
  CameraSpec cam;
  StepConsts<R> step;         // geodesics in the render precision (FP32, FP64)
  StepConsts<double> step_d;  // the mixed mode's FP64 geodesic
  R tau_fp64;
  PlasmaView<R> pv;
  R freq[kMaxFreqs], hconst[kMaxFreqs], jscale[kMaxFreqs];

  template <class G>
  PHX_HD const StepConsts<G>& steps_in() const {
    if constexpr (sizeof(G) == sizeof(R)) {
      return step;
    } else {
      return step_d;
    }
  }
};

// The camera set-up of one pixel in FP64: initial photon state (x, k), polarization vector F1, its Walker-Penrose
// constant kappa and the sign of the impact parameter beta.
struct RayStart {
  double ph[8], F1[4], kappa[2];
  int bsign;
};

// Kept out of line: it runs once per ray, and its FP64 code (impact parameters, the Newton solve for x2, the camera
// tetrad) inlined into the march loop would crowd the loop's instruction cache and register allocation.
// G: the precision of the camera tetrad's arithmetic (the geodesic precision, as in the reference's builds).
template <class G, class R>
PHX_HD_OUTLINE RayStart ray_start(const RenderConsts<R>& rc, G a, G hs, int32_t pixel) {
  RayStart st;
  const int i = pixel / rc.H, j = pixel % rc.H;
  double alpha, beta;
  pixel_impact(i, j, rc.W, rc.H, rc.fov_x, rc.fov_y, rc.cos_pa, rc.sin_pa, &alpha, &beta);
  camera_photon(rc.cam, alpha, beta, st.ph);
  camera_pol<G>(a, hs, st.ph, st.F1);
  const KerrPt<double> pc = kerr_point<double>(a, hs, st.ph[1], st.ph[2]);
  walker_penrose<double>(a, pc, st.ph + 4, st.F1, st.kappa);
  st.bsign = beta < 0.0 ? -1 : (beta > 0.0 ? 1 : 0);
  return st;
}

// Diagnostic counters a ray adds to.
struct RayCounters {
  uint32_t steps, nplasma, bad, scans, fp64_steps, fp64_ops;
};

template <Mode M, class PT, int NF>
struct Ray {
  using Pol = Policy<M>;
  using R = typename Pol::R;
  using G = typename Pol::G;
  static constexpr bool kComp = Pol::kComp, kMixed = Pol::kMixed, kShift = Pol::kShift;
  static constexpr bool kLate = M == Mode::kFP64;  // the reference's one-pass-late sample order (see advance())
  // FP32 and mixed: the polarization direction at a sample comes from the Walker-Penrose constant taken at the camera
  // (exact for parallel transport), so the geodesic state is (x, k) only; FP64 transports F1 with the state as the
  // reference does, and follows it bit for bit
  static constexpr bool kWP = !kLate;
  static constexpr int kNS = kWP ? 8 : 12;

  GeoState<G, kNS> geo;
  R kappa[2];   // Walker-Penrose constant of (k, F1) (kWP)
  G px[4], pk[4], pF[4], pdl;  // FP64 (kLate): the pending sample's point and the length of the step to it
  bool pvalid, terminate;
  int steps, turns, bsign, nplasma, bad;
  G thdot_prev, dl_prev;
  G pr;         // radius of the pending sample (exp of px[1], from the step that made it)
  int32_t pix;
  int leaf;     // leaf of the last step-size lookup (-1: none), tested before the leaf map
  G idxc[3];    // its inverse cell sizes (FP32 and mixed step-size cap)
  // transfer records (4x4 operator, Stokes sums, optical depths) per frequency slot: the kernels of 4 slots and the
  // mixed and FP64 kernels of 1 keep them in the block's dynamic shared memory (kSmemPerThread bytes per thread), the
  // FP32 one-slot and all 32-slot kernels in registers.  Measured on B200: mixed 3-frequency renders 14% faster,
  // FP64 3-5%, FP32 3-frequency 3-6% (no spills at 128 registers); FP32 with one slot 3% slower, so it keeps
  // registers.
  // Host builds (g++: tools and the host tests of this code) have no shared memory and keep the records in the object.
#if defined(__CUDACC__)
  static constexpr bool kAccShared = (kMixed || M == Mode::kFP64 || NF > 1) && NF <= 4;
#else
  static constexpr bool kAccShared = false;
#endif
  using AccStore = std::conditional_t<kAccShared, AccShared<R, kMixed, NF>, AccRegs<R, kMixed, NF>>;
  static constexpr size_t kSmemPerThread = AccStore::kSmemPerThread;
  AccStore acc;

  // The snapshot in the geodesic's precision: the plasma-stage view itself (FP32, FP64) or the FP64 view sd (mixed).
  // Both live in kernel parameter space or in the item table, so no copy is made for the out-of-line callees that
  // take the view by reference.
  PHX_HD static const SnapView<G, PT>& geo_view(const SnapView<R, PT>& s, const SnapView<double, PT>& sd) {
    if constexpr (sizeof(G) == sizeof(R)) {
      return s;
    } else {
      return sd;
    }
  }

  PHX_HD void init(const SnapView<R, PT>& s, const SnapView<double, PT>& sd, const RenderConsts<R>& rc,
                   int32_t pixel) {
    const SnapView<G, PT>& sg = geo_view(s, sd);
    init_from(ray_start<G>(rc, sg.a, sg.hs, pixel), pixel);
  }

  // Starts the ray from its camera set-up (ray_start), computed here or beforehand by the ray-setup kernel: the same
  // out-of-line function either way, so the ray is bit-identical.
  PHX_HD void init_from(const RayStart& st, int32_t pixel) {
    pix = pixel;
    geo_init<G, kComp>(geo, st.ph, st.F1);
    kappa[0] = R(st.kappa[0]);
    kappa[1] = R(st.kappa[1]);
#pragma unroll
    for (int f = 0; f < NF; f++) acc_reset<R, kMixed>(acc, f);
    pvalid = false;
    terminate = false;
    steps = turns = nplasma = bad = 0;
    bsign = st.bsign;
    thdot_prev = dl_prev = G(0);
    pr = G(0);
    leaf = -1;
    idxc[0] = idxc[1] = idxc[2] = G(0);
  }

  // The leaf of the wrapped point xw (the last one first: a ray stays tens of steps in one leaf, and since the
  // leaves tile the domain a point inside it has no other leaf); -1 outside the domain.  Also keeps the leaf's
  // inverse cell sizes for the step-size cap of the FP32 and mixed paths.
  PHX_HD int lookup(const SnapView<G, PT>& s, const G xw[4], RayCounters& ctr) {
    if (leaf >= 0 && inside_leaf(s, leaf, xw, leaf_nudge(xw))) return leaf;
    bool scanned = false;
    const int L = find_leaf(s, xw, &scanned);
    ctr.scans += scanned;
    if constexpr (!kLate) {
      if (L >= 0 && L != leaf) {
#pragma unroll
        for (int d = 0; d < 3; d++) idxc[d] = geo_rcp<G, kShift>(ldg(s.dxc + 3 * L + d));  // feeds only the step cap
      }
    }
    leaf = L;
    return L;
  }

  // One pass of the march loop; false once the ray has ended.
  //
  // The reference processes each point's plasma sample one pass late (core/render/pixel.hpp:179-211), after the
  // next point's leaf lookup, whose leaf then seeds the sampler's cache check.  FP64 keeps that order, so that it
  // follows the reference bit for bit.  The FP32 and mixed paths process each sample at its own point, before the
  // step, seeded by its own leaf (found for the step-size cap anyway): the samples, their order and their segment
  // lengths are the same (points 1.. of the live path inside rt_outer, each with the length of the step that led to
  // it), no copy of the previous point's state is carried (fewer registers), and the leaf found differs only for
  // points within the sampler's 1e-9 nudge of a block face.
  PHX_HD bool advance(const SnapView<R, PT>& s, const SnapView<double, PT>& sd, const RenderConsts<R>& rc,
                      RayCounters& ctr) {
    const SnapView<G, PT>& sg = geo_view(s, sd);
    const StepConsts<G>& sc = rc.template steps_in<G>();
    G cx[4], ck[4], cF[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      cx[i] = geo_get<G, kComp>(geo, i);
      ck[i] = geo_get<G, kComp>(geo, 4 + i);
      if constexpr (kWP) {
        cF[i] = G(0);  // unused: the sample takes the polarization from kappa
      } else {
        cF[i] = geo_get<G, kComp>(geo, 8 + i);
      }
    }
    const G r = exp_t(cx[1]);
    const bool alive = r < sc.r_out && r > sc.cut_in && steps < rc.max_steps && !terminate;
    // beyond rt_outer the reference keeps no sample (derive_fluid and process_sample both require r < rt_outer) and
    // caps no step by the grid
    const bool inner = alive && r < sc.rt_outer;
    int L = -1;
    if constexpr (kLate) {
      const bool pend_plasma = pvalid && pr < sc.rt_outer;
      const bool need_leaf = pend_plasma && alive;
      int right = -1;
      if (need_leaf || inner) {
        G xw[4] = {cx[0], cx[1], cx[2], cx[3]};
        wrap_coords(xw);
        L = lookup(sg, xw, ctr);
        if (need_leaf) right = (r < G(1) || outside_domain(sg, xw)) ? -1 : L;  // wrapping keeps x1: exp(xw[1]) = r
      }
      if (pend_plasma) process_sample(s, sg, rc, px, pk, pF, pr, pdl, right, ctr);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        px[i] = cx[i];
        pk[i] = ck[i];
        pF[i] = cF[i];
      }
      pr = r;
      pdl = dl_prev;
      pvalid = steps >= 1;
      if (!alive) return false;
    } else {
      if (!alive) return false;
      if (inner) {
        G xw[4] = {cx[0], cx[1], cx[2], cx[3]};
        wrap_coords(xw);
        L = lookup(sg, xw, ctr);
        if (steps >= 1) {
          const int right = (r < G(1) || outside_domain(sg, xw)) ? -1 : L;  // wrapping keeps x1: exp(xw[1]) = r
          process_sample(s, sg, rc, cx, ck, cF, r, dl_prev, right, ctr);
        }
      }
    }

    if (thdot_prev * ck[2] < G(0) && steps > 2) turns++;
    thdot_prev = ck[2];
    if ((bsign < 0 && turns > rc.max_order) || (bsign > 0 && turns > rc.max_order + 1)) terminate = true;

    const bool cap = inner && L >= 0;
    const G x2 = pole_x2<G, kComp>(geo);
    G dl;
    if constexpr (!kLate) {
      // FP32 and mixed: the reciprocals folded (two divisions instead of twelve; the same rule up to rounding)
      dl = step_size_fast<G, kShift>(sc.stepsize, sc.inv_stepsize, x2, ck, cap ? idxc : (const G*)nullptr, sc.tiny,
                                     sc.big);
    } else {
      G dxcv[3];
      if (cap) {
#pragma unroll
        for (int d = 0; d < 3; d++) dxcv[d] = ldg(sg.dxc + 3 * L + d);
      }
      dl = step_size(sc.stepsize, x2, ck, cap ? dxcv : (const G*)nullptr, sc.tiny, sc.big);
    }
    rk4_step<G, kComp, kNS, kShift>(sg.a, sg.hs, geo, dl);
    if constexpr (kMixed) ctr.fp64_steps++;
    dl_prev = fabs_t(dl);
    steps++;
    return true;
  }

  // The plasma stage of the sample at point (x0, k0, F0) of radius r, reached by a step of length hl (the reference's
  // process_sample, core/render/pixel.hpp:52-123).  The point comes in the geodesic's precision G; the fluid,
  // coefficients and transfer operator run in R.
  PHX_HD void process_sample(const SnapView<R, PT>& s, const SnapView<G, PT>& sg, const RenderConsts<R>& rc,
                             const G x0[4], const G k0[4], const G F0[4], G r, G hl, int right, RayCounters& ctr) {
    // null-condition renormalisation of the sample's wave vector, in the geodesic's precision (reference:
    // geodesic.hpp:297-306, applied when |k.k| > 1e-6 and r > 2)
    G kg[4] = {k0[0], k0[1], k0[2], k0[3]};
    const KerrPt<G> pg = kerr_point_r(sg.a, sg.hs, r, x0[2]);  // the sample's own (unwrapped) point
    {
      const Cov<G> g0 = cov_metric(pg, sg.a);
      if (fabs_t(dot(g0, kg, kg)) > G(1e-6) && r > G(2)) normalize_null(g0, kg);
    }
    // sampler (sampler.hpp:387-427): wrap, domain, cached leaf or a fresh lookup of the re-wrapped point, cell and
    // weights -- all in G; the weighted sum of the primitives in R
    G xg[4] = {x0[0], x0[1], x0[2], x0[3]};
    int ig = right;
    wrap_coords(xg);
    if (r < G(1)) return;  // exp(xg[1]): wrapping keeps x1
    if (outside_domain(sg, xg)) return;
    if (ig == -1 || !inside_cached(sg, ig, xg)) {
      wrap_coords(xg);
      bool scanned = false;
      ig = find_leaf(sg, xg, &scanned);
      ctr.scans += scanned;
    }
    if (ig == -1) return;
    R q[kNPrim];
    if constexpr (kMixed) {
      int c[3];
      G dd[3];
      cell_weights<G, PT, true>(sg, ig, xg, c, dd);
      const R del[3] = {R(dd[0]), R(dd[1]), R(dd[2])};
      gather_prims<R, PT>(s.prim, s.cells, s.nx, ig, c, del, q);
    } else {
      interp_prims<R, PT, !kComp>(s, ig, xg, q);
    }
    // the rest in R, at the wrapped point (x1 unchanged by the wrap, so its radius is r)
    const R x2w = R(xg[2]);
    const R rx = R(r);
    R k[4] = {R(kg[0]), R(kg[1]), R(kg[2]), R(kg[3])};
    const KerrPt<R> p = kerr_point_r(s.a, s.hs, rx, x2w);
    const Cov<R> g = cov_metric(p, s.a);
    const Contra<R> u = contra_metric(p, s.a);
    Fluid<R> fl;
    if (!derive_fluid(rc.pv, s.gam, rx, g, u, q, &fl)) return;
    if (!(r < rc.template steps_in<G>().rt_outer)) return;
    // k, U and B lowered once: every invariant below is then a 4-term inner product
    R kd[4], Ud[4], Bd[4];
    symv(g, k, kd);
    symv(g, fl.U, Ud);
    symv(g, fl.B, Bd);
    const R kU = dot4(kd, fl.U), kB = dot4(kd, fl.B), UB = dot4(Ud, fl.B), BB = dot4(Bd, fl.B);
    // pitch angle of k to B in the plasma frame (tetrad.hpp:138-154): only its sine and cosine enter the
    // coefficients, so they are formed from mu = cos(pitch) directly; acos(mu) is 0 or pi exactly when mu = +-1
    const R Bn = fastm::sqrt(fabs_t(BB));
    R sth = R(1), cth = R(0);
    if (Bn != R(0)) {
      R mu = fastm::div(kB, fabs_t(kU) * Bn);
      if (fabs_t(mu) > R(1)) mu /= fabs_t(mu);
      if (mu == R(1) || mu == R(-1)) return;
      sth = fastm::sqrt((R(1) - mu) * (R(1) + mu));
      cth = mu;
    }
    // polarization axes of the plasma frame with B as reference direction; EVPA rotation from the transported F1
    R perp[4], para[4];
    observer_axes_lowered(sqrt_neg_g(p), k, fl.U, fl.B, kd, Ud, Bd, -kU, kB, UB, BB, perp, para);
    R C, S;
    if constexpr (kWP) {
      // the transported F1's components on (perp, para), from kappa at the point the state describes
      if constexpr (sizeof(G) == sizeof(R)) {
        wp_components(s.a, pg, k, perp, para, kappa, &C, &S);
      } else {
        // the FP64 geometry of this point, rounded (no second metric point: wp_components reads r, sin, cos, theta')
        KerrPt<R> p0;
        p0.r = R(pg.r);
        p0.s = R(pg.s);
        p0.c = R(pg.c);
        p0.s2 = R(pg.s2);
        p0.tp = R(pg.tp);
        p0.tpp = R(pg.tpp);
        p0.sig = R(pg.sig);
        p0.isig = R(pg.isig);
        p0.q = R(pg.q);
        wp_components(s.a, p0, k, perp, para, kappa, &C, &S);
      }
    } else {
      const R F[4] = {R(F0[0]), R(F0[1]), R(F0[2]), R(F0[3])};
      R pFd[4];
      symv(g, F, pFd);
      C = dot4(pFd, perp);
      S = dot4(pFd, para);
    }
    const R inn = fastm::rcp(C * C + S * S);
    const R c2 = (C * C - S * S) * inn, s2 = R(2) * C * S * inn;
    const R ratio = -kU;  // nu_plasma / nu_camera
    const SynchroSample<R> ss = synchro_sample(fl.theta_e, fl.n_e, fl.Bmag, sth, cth);
    const R hlr = R(hl);
#pragma unroll
    for (int f = 0; f < NF; f++) {
      if (f >= rc.nfreqs) break;
      const R nu = rc.freq[f] * ratio;
      const Coeffs<R> cf = synchro_coeffs(ss, nu, rc.jscale[f]);
      R K[4][4], jv[4], E[4][4], Sg[4];
      build_K(cf, c2, s2, K, jv);
      const R h = hlr * rc.hconst[f];
      bool fp64 = false;
      if constexpr (kMixed) {
        const R kmax = fmax_t(fmax_t(fabs_t(cf.aI), fabs_t(cf.rV)), fabs_t(cf.rQ));
        fp64 = h * kmax > rc.tau_fp64;
      }
      if (fp64) {
        SegmentIn<R> in;
        in.h = h;
        for (int a = 0; a < 4; a++) {
          in.j[a] = jv[a];
          for (int b = 0; b < 4; b++) in.K[a][b] = K[a][b];
        }
        const SegmentOut<R> o = segment_operator_fp64(in);
        for (int a = 0; a < 4; a++) {
          Sg[a] = o.S[a];
          for (int b = 0; b < 4; b++) E[a][b] = o.E[a][b];
        }
        ctr.fp64_ops++;
      } else {
        segment_operator<R>(K, jv, h, E, Sg);
      }
      if (!all_finite(E, Sg)) {
        bad++;
        continue;
      }
      acc_add<R, kMixed>(acc, f, E, Sg, cf.aI * h, fabs_t(cf.rV * h));
    }
    nplasma++;
  }

  // FreqOut records (I, Q, U, V, tau, tauF as doubles) of this pixel; zeros when no plasma segment was crossed.
  PHX_HD void write(double* out, int nfreqs) {
#pragma unroll
    for (int f = 0; f < NF; f++) {
      if (f >= nfreqs) break;
      double* o = out + ((size_t)pix * nfreqs + f) * 6;
      const bool any = nplasma > 0;
      using W = AccWords<kMixed>;
      o[0] = any ? (double)acc.at(f, W::kS) : 0.0;
      o[1] = any ? (double)acc.at(f, W::kS + 1) : 0.0;
      o[2] = any ? (double)acc.at(f, W::kS + 2) : 0.0;
      o[3] = any ? (double)acc.at(f, W::kS + 3) : 0.0;
      o[4] = any ? (double)acc.at(f, W::kTau) : 0.0;
      o[5] = any ? (double)acc.at(f, W::kTauF) : 0.0;
    }
  }
};

}  // namespace phx
