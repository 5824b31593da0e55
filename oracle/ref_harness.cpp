// Driver for the reference renderer's own CPU path (test infrastructure: the oracle, not the product).
//
// It is compiled against the reference's unmodified headers where they lie (see oracle/build_ref.py) and does what
// PHOENIX's main() does for the CPU build (src/main.cpp:88-205) minus HDF5 output:
//   host::config::load_config (host/io/config.hpp:229) -> host::bhac_io::load_bhac_grid (host/io/bhac_io.hpp:143)
//   -> host::bhac_io::load (bhac_io.hpp:331, host decode) -> an OpenMP dynamic loop over pixels like
//   host::jobs::process (host/render/jobs.hpp:50-92) calling core::pixel::render_pixel (core/render/pixel.hpp:134).
// The total flux follows host::output::compute_spec (host/io/output.hpp:43-53).
//
// usage: ref_render CONFIG [section.key=value ...] [--pixels FILE] [--out FILE] [--stats FILE] [--threads N]
//                   [--inclinations A,B,...] [--repeat R]
//   --pixels        int32 pixel indices i*img_height+j to render (default: every pixel, row-major)
//   --out           FreqOut records (6 doubles) per requested pixel and frequency, in request order
//   --stats         int64 (steps, nplasma, bad) per requested pixel
//   --inclinations  render the pixel list once per inclination (camera.inclination only enters the camera set-up,
//                   so the snapshot is read and decoded once); outputs hold the last inclination
//   --repeat        passes over the whole list (timing); one JSON line per pass
// Prints one JSON line per pass: pixels, steps, nplasma, bad, seconds (pixel loops only), threads, precision and
// (single full-image passes) the flux.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "host/io/config.hpp"
#include "host/io/bhac_io.hpp"
#include "core/render/headers.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s CONFIG [key=value ...] [--pixels F] [--out F] [--stats F] [--threads N]\n", argv[0]);
    return 2;
  }
  const std::string cfg = argv[1];
  std::vector<std::string> overrides;
  std::string pix_path, out_path, stats_path;
  int threads = 0, repeat = 1;
  std::vector<double> incls;
  for (int i = 2; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--inclinations" && i + 1 < argc) {
      std::string t = argv[++i];
      size_t p0 = 0;
      while (p0 <= t.size()) {
        const size_t p1 = t.find(',', p0);
        const std::string tok = t.substr(p0, p1 == std::string::npos ? std::string::npos : p1 - p0);
        if (!tok.empty()) incls.push_back(std::atof(tok.c_str()));
        if (p1 == std::string::npos) break;
        p0 = p1 + 1;
      }
    } else if (a == "--repeat" && i + 1 < argc) repeat = std::max(1, std::atoi(argv[++i]));
    else if (a == "--pixels" && i + 1 < argc) pix_path = argv[++i];
    else if (a == "--out" && i + 1 < argc) out_path = argv[++i];
    else if (a == "--stats" && i + 1 < argc) stats_path = argv[++i];
    else if (a == "--threads" && i + 1 < argc) threads = std::atoi(argv[++i]);
    else overrides.push_back(a);
  }
  if (threads > 0) omp_set_num_threads(threads);

  core::bhac::Model model = {};
  host::config::Params params;
  try {
    host::config::load_config(cfg, overrides, params, &model.uparams);
    host::bhac_io::load_bhac_grid(&model.gparams, params.grid_file);
    host::bhac_io::load(&model, params.dump_file, false);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_render: %s\n", e.what());
    return 1;
  }
  const core::bhac::UserParams& up = model.uparams;
  const int W = up.img_width, H = up.img_height, F = up.nfreqs;

  std::vector<int> pix;
  if (!pix_path.empty()) {
    FILE* f = std::fopen(pix_path.c_str(), "rb");
    if (!f) {
      std::fprintf(stderr, "ref_render: cannot open %s\n", pix_path.c_str());
      return 1;
    }
    int v;
    while (std::fread(&v, sizeof v, 1, f) == 1) pix.push_back(v);
    std::fclose(f);
  } else {
    for (int n = 0; n < W * H; n++) pix.push_back(n);
  }
  const int np = (int)pix.size();
  std::vector<core::pixel::FreqOut> res((size_t)np * F);
  std::vector<long long> st((size_t)np * 3);

  if (incls.empty()) incls.push_back(up.inclination);
  long steps = 0, segs = 0, bad = 0;
  double secs = 0.0;
  for (int pass = 0; pass < repeat; pass++) {
    steps = segs = bad = 0;
    secs = 0.0;
    for (double incl : incls) {
      model.uparams.inclination = incl;
      const auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : steps, segs, bad)
      for (int n = 0; n < np; n++) {
        const int idx = pix[n];
        const int i = idx / H, j = idx % H;
        double a0, b0;
        core::camera::pixel_impact(i, j, W, H, up.fov_x, up.fov_y, &a0, &b0);
        const double alpha = a0 * model.cos_pa + b0 * model.sin_pa;
        const double beta = -a0 * model.sin_pa + b0 * model.cos_pa;
        const core::pixel::RunStats rs = core::pixel::render_pixel(&model, alpha, beta, &res[(size_t)n * F]);
        st[3 * (size_t)n + 0] = rs.steps;
        st[3 * (size_t)n + 1] = rs.nplasma;
        st[3 * (size_t)n + 2] = rs.bad;
        steps += rs.steps;
        segs += rs.nplasma;
        bad += rs.bad;
      }
      secs += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    if (pass + 1 < repeat) {
      std::printf("{\"pixels\": %d, \"steps\": %ld, \"nplasma\": %ld, \"bad\": %ld, \"seconds\": %.6f, "
                  "\"threads\": %d, \"precision\": \"%s\"}\n",
                  np * (int)incls.size(), steps, segs, bad, secs, omp_get_max_threads(), accuracy_name());
    }
  }

  if (!out_path.empty()) {
    FILE* f = std::fopen(out_path.c_str(), "wb");
    if (!f || std::fwrite(res.data(), sizeof(core::pixel::FreqOut), res.size(), f) != res.size()) return 1;
    std::fclose(f);
  }
  if (!stats_path.empty()) {
    FILE* f = std::fopen(stats_path.c_str(), "wb");
    if (!f || std::fwrite(st.data(), sizeof(long long), st.size(), f) != st.size()) return 1;
    std::fclose(f);
  }

  std::printf("{\"pixels\": %d, \"steps\": %ld, \"nplasma\": %ld, \"bad\": %ld, \"seconds\": %.6f, \"threads\": %d, "
              "\"precision\": \"%s\"",
              np * (int)incls.size(), steps, segs, bad, secs, omp_get_max_threads(), accuracy_name());
  if (pix_path.empty() && incls.size() == 1) {
    const double dOmega = core::camera::pixel_solid_angle(&model);
    std::printf(", \"flux\": [");
    for (int f = 0; f < F; f++) {
      double S[4] = {0, 0, 0, 0};
      for (int n = 0; n < np; n++) {
        const core::pixel::FreqOut& r = res[(size_t)n * F + f];
        if (!std::isfinite(r.IQUV[0] + r.IQUV[1] + r.IQUV[2] + r.IQUV[3])) continue;
        for (int q = 0; q < 4; q++) S[q] += r.IQUV[q] * dOmega;
      }
      std::printf("%s[%.17g, %.17g, %.17g, %.17g, %.17g]", f ? ", " : "", up.frequencies[f], S[0] * 1e23,
                  S[1] * 1e23, S[2] * 1e23, S[3] * 1e23);
    }
    std::printf("]");
  }
  std::printf("}\n");
  host::bhac_io::free_model(&model);
  return 0;
}
