// Polarized transfer: the single-pass transfer-operator method (Landi Degl'Innocenti & Landi Degl'Innocenti 1985,
// Dexter 2016 sec. 2.5.2) with the implicit-trapezoid (Crank-Nicolson) segment operator the reference uses
// (core/transfer/operators.hpp:74-176):
//   dS/ds = j - K S,  P = I + (h/2) K,  A_seg = P^-1 (I - (h/2) K),  S_seg = h P^-1 j,
//   S_tot += A_acc S_seg,  A_acc = A_acc A_seg  (camera side first: the ray runs backwards).
//
// The same operator is computed in deviation form, which is exact algebra but keeps FP32 accurate in optically thin
// plasma, where A_seg = I - O(h K) and A_acc stays near I:
//   E = A_seg - I = -h P^-1 K,   S_seg = h P^-1 j     (one Gauss-Jordan solve of P X = [K | j], partial pivoting)
// and the accumulated transmission is held as D = A_acc - I until it departs from I (|D_ii| > 1/2), after which it
// is held as A_acc itself:  D <- D + E + D E,   A <- A + A E.
#pragma once

#include "defs.cuh"
#include "synchro.cuh"

namespace phx {

// The 4x4 absorption / Faraday matrix in the camera polarization basis; c2, s2 = cos 2 chi, sin 2 chi rotate the
// plasma-frame coefficients (whose U components vanish by construction of the plasma tetrad).
template <class R>
PHX_HD void build_K(const Coeffs<R>& c, R c2, R s2, R K[4][4], R j[4]) {
  const R aQ = c2 * c.aQ, aU = -s2 * c.aQ;
  const R rQ = c2 * c.rQ, rU = -s2 * c.rQ;
  const R aI = c.aI, aV = c.aV, rV = c.rV;
  K[0][0] = aI; K[0][1] = aQ;  K[0][2] = aU;  K[0][3] = aV;
  K[1][0] = aQ; K[1][1] = aI;  K[1][2] = rV;  K[1][3] = -rU;
  K[2][0] = aU; K[2][1] = -rV; K[2][2] = aI;  K[2][3] = rQ;
  K[3][0] = aV; K[3][1] = rU;  K[3][2] = -rQ; K[3][3] = aI;
  j[0] = c.jI;
  j[1] = c2 * c.jQ;
  j[2] = -s2 * c.jQ;
  j[3] = c.jV;
}

// E = -h P^-1 K and S = h P^-1 j by Gauss-Jordan elimination with partial pivoting on [P | K | j].
template <class R>
PHX_HD void segment_operator(const R K[4][4], const R j[4], R h, R E[4][4], R S[4]) {
  R M[4][9];
  const R hh = R(0.5) * h;
#pragma unroll
  for (int i = 0; i < 4; i++) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      M[i][k] = (i == k ? R(1) : R(0)) + hh * K[i][k];
      M[i][4 + k] = K[i][k];
    }
    M[i][8] = j[i];
  }
#pragma unroll
  for (int c = 0; c < 4; c++) {
#pragma unroll
    for (int r = c + 1; r < 4; r++) {
      const bool sw = fabs_t(M[r][c]) > fabs_t(M[c][c]);
#pragma unroll
      for (int q = c; q < 9; q++) {
        const R t = M[c][q];
        M[c][q] = sw ? M[r][q] : t;
        M[r][q] = sw ? t : M[r][q];
      }
    }
    const R inv = fastm::rcp(M[c][c]);  // FP32: hardware reciprocal (2 ulp); FP64: exact
#pragma unroll
    for (int q = c; q < 9; q++) M[c][q] *= inv;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      if (r == c) continue;
      const R f = M[r][c];
#pragma unroll
      for (int q = c; q < 9; q++) M[r][q] -= f * M[c][q];
    }
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
#pragma unroll
    for (int k = 0; k < 4; k++) E[i][k] = -h * M[i][4 + k];
    S[i] = h * M[i][8];
  }
}

// The segment operator evaluated in FP64 for a step of large optical or Faraday depth (the mixed mode; a few percent of
// its samples).  Out of line, arguments and results by value, so that the FP64 copy of the 4x4 solve stays out of the
// march loop beside the FP32 one.
template <class R>
struct SegmentIn {
  R K[4][4], j[4], h;
};
template <class R>
struct SegmentOut {
  R E[4][4], S[4];
};

template <class R>
PHX_HD_OUTLINE SegmentOut<R> segment_operator_fp64(SegmentIn<R> in) {
  double K[4][4], j[4], E[4][4], S[4];
  for (int a = 0; a < 4; a++) {
    j[a] = in.j[a];
    for (int b = 0; b < 4; b++) K[a][b] = in.K[a][b];
  }
  segment_operator<double>(K, j, (double)in.h, E, S);
  SegmentOut<R> o;
  for (int a = 0; a < 4; a++) {
    o.S[a] = R(S[a]);
    for (int b = 0; b < 4; b++) o.E[a][b] = R(E[a][b]);
  }
  return o;
}

template <class R>
PHX_HD bool all_finite(const R E[4][4], const R S[4]) {
  R s = R(0);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    s += S[i] * R(0);
#pragma unroll
    for (int k = 0; k < 4; k++) s += E[i][k] * R(0);
  }
  return s == R(0);  // any inf or NaN makes the sum NaN
}

// Per-ray, per-frequency accumulator record, as words of precision R:
//   X[4][4]  D = A - I while in deviation form, else A;   S[4] Stokes sums;   Sc[4] their Kahan compensation (kKahan);
//   tau, tauF;   dev (1: X holds D, 0: X holds A).
template <bool kKahan>
struct AccWords {
  static constexpr int kX = 0, kS = 16, kSc = 20, kTau = kKahan ? 24 : 20, kTauF = kTau + 1, kDev = kTau + 2,
                       kN = kTau + 3;
};

// Records in the thread's registers (FP64 and the 32-slot kernels).
template <class R, bool kKahan, int NF>
struct AccRegs {
  static constexpr size_t kSmemPerThread = 0;
  R w[NF][AccWords<kKahan>::kN];
  PHX_HD R& at(int f, int e) { return w[f][e]; }
};

#if defined(__CUDACC__)
extern __shared__ __align__(16) unsigned char phx_dyn_smem[];
#endif

// Records in the block's dynamic shared memory: word e of slot f of a thread at [(f * kN + e) * blockDim.x + tid],
// so the 32 lanes of a warp touch 32 consecutive words (no bank conflicts).  Keeping the 4x4 operator out of the
// registers shortens the live state the geodesic step carries by a record per slot (23 words in FP32).
template <class R, bool kKahan, int NF>
struct AccShared {
  static constexpr size_t kSmemPerThread = sizeof(R) * NF * AccWords<kKahan>::kN;
  PHX_HD R& at(int f, int e) {
#if defined(__CUDA_ARCH__)
    return reinterpret_cast<R*>(phx_dyn_smem)[(f * AccWords<kKahan>::kN + e) * blockDim.x + threadIdx.x];
#else
    static R unused;  // the host pass of nvcc compiles this but never runs it (g++ builds keep records in registers)
    return unused;
#endif
  }
};

template <class R, bool kKahan, class St>
PHX_HD void acc_reset(St& st, int f) {
  using W = AccWords<kKahan>;
#pragma unroll
  for (int e = 0; e < W::kN; e++) st.at(f, e) = R(0);
  st.at(f, W::kDev) = R(1);
}

// Appends one segment (E = A_seg - I, Sg = S_seg) and its optical depths to slot f:
//   S += A Sg with the accumulated operator before this segment (Kahan-compensated when kKahan);
//   X <- X + X E (+ E in deviation form), switching to the plain form once |D_ii| > 1/2.
template <class R, bool kKahan, class St>
PHX_HD void acc_add(St& st, int f, const R E[4][4], const R Sg[4], R dtau, R dtauF) {
  using W = AccWords<kKahan>;
  R X[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) X[i][k] = st.at(f, W::kX + 4 * i + k);
  bool dev = st.at(f, W::kDev) != R(0);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    R t = dev ? Sg[i] : R(0);
#pragma unroll
    for (int k = 0; k < 4; k++) t += X[i][k] * Sg[k];
    const R S = st.at(f, W::kS + i);
    if constexpr (kKahan) {
      const R c = st.at(f, W::kSc + i);
      const R y = t - c;
      const R s = S + y;
      st.at(f, W::kSc + i) = (s - S) - y;
      st.at(f, W::kS + i) = s;
    } else {
      st.at(f, W::kS + i) = S + t;
    }
  }
  R Y[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      R t = dev ? E[i][k] : R(0);
#pragma unroll
      for (int m = 0; m < 4; m++) t += X[i][m] * E[m][k];
      Y[i][k] = t;
    }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) X[i][k] += Y[i][k];
  if (dev) {
    R m = R(0);
#pragma unroll
    for (int i = 0; i < 4; i++) m = fmax_t(m, fabs_t(X[i][i]));
    if (m > R(0.5)) {
#pragma unroll
      for (int i = 0; i < 4; i++) X[i][i] += R(1);
      dev = false;
      st.at(f, W::kDev) = R(0);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) st.at(f, W::kX + 4 * i + k) = X[i][k];
  st.at(f, W::kTau) += dtau;
  st.at(f, W::kTauF) += dtauF;
}

}  // namespace phx
