// Image, spectrum and flux outputs of a render, in the reference's formats (src/host/io/output.hpp:43-167,
// src/main.cpp:52-86).  res holds W * H * F records at (i * H + j) * F + f.
#pragma once

#include <string>
#include <vector>

#include "../../../include/phoenix_b200.h"

namespace phx {

// Total Stokes flux [Jy] of frequency index f; pixels with a non-finite I+Q+U+V are skipped.
void compute_spec(const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int f, double S[4]);
// Mean tau and tauF over the finite pixels.
void compute_tau(const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int f, double T[2]);
// Text image: one row per pixel (i outer, j inner): x, y [arcsec], I, Q, U, V [Jy / pixel], tau, tauF.
bool write_image_text(const std::string& path, const PhxRenderParams& p, const std::vector<PhxFreqOut>& res, int f);
// One row per frequency: nu, I, Q, U, V [Jy], mean tau, mean tauF.
bool write_spectrum(const std::string& path, const PhxRenderParams& p, const std::vector<PhxFreqOut>& res);
// RAPTOR-format HDF5 image: per frequency I%e, tau%e, Q%e, U%e, V%e, tauF%e, plus alpha and beta, each float64
// [(W/bs)(H/bs)][bs*bs] with block b = bi * (H/bs) + bj and in-block pixel pi * bs + pj; I..V in Jy/sr.
bool write_image_hdf5(const std::string& path, const PhxRenderParams& p, int block_size,
                      const std::vector<PhxFreqOut>& res, std::string* err);

}  // namespace phx
