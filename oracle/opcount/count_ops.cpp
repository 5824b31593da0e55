// Per-pixel operation counts of the reference's FP32 raymarch -- TEST INFRASTRUCTURE ONLY.
//
// Compiled with oracle/opcount/ ahead of the reference's src/ on the include path (see count_flops.py), so that the
// reference's unmodified headers run with the op-counting `scalar` of opcount.hpp.  Like oracle/ref_harness.cpp it
// reads the config and the BHAC snapshot with the reference's own host code, then renders the requested pixels one
// at a time with core::pixel::render_pixel (core/render/pixel.hpp:134-224) and writes, per pixel, its steps, plasma
// segments and bad segments followed by the tally of every operation class (opcount.hpp) over that pixel.
//
// usage: count_ops CONFIG [section.key=value ...] --pixels FILE --out FILE
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "core/numerics/precision.hpp"
#include "host/io/config.hpp"
#include "host/io/bhac_io.hpp"
#include "core/render/headers.hpp"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s CONFIG [key=value ...] --pixels F --out F\n", argv[0]);
    return 2;
  }
  const std::string cfg = argv[1];
  std::vector<std::string> overrides;
  std::string pix_path, out_path;
  for (int i = 2; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--pixels" && i + 1 < argc) pix_path = argv[++i];
    else if (a == "--out" && i + 1 < argc) out_path = argv[++i];
    else overrides.push_back(a);
  }
  core::bhac::Model model = {};
  host::config::Params params;
  try {
    host::config::load_config(cfg, overrides, params, &model.uparams);
    host::bhac_io::load_bhac_grid(&model.gparams, params.grid_file);
    host::bhac_io::load(&model, params.dump_file, false);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "count_ops: %s\n", e.what());
    return 1;
  }
  const core::bhac::UserParams& up = model.uparams;
  const int W = up.img_width, H = up.img_height, F = up.nfreqs;
  std::vector<int> pix;
  FILE* f = std::fopen(pix_path.c_str(), "rb");
  if (!f) return 1;
  int v;
  while (std::fread(&v, sizeof v, 1, f) == 1) pix.push_back(v);
  std::fclose(f);
  std::vector<core::pixel::FreqOut> res((size_t)F);
  std::vector<unsigned long long> rows;
  for (const int idx : pix) {
    const int i = idx / H, j = idx % H;
    double a0, b0;
    core::camera::pixel_impact(i, j, W, H, up.fov_x, up.fov_y, &a0, &b0);
    const double alpha = a0 * model.cos_pa + b0 * model.sin_pa;
    const double beta = -a0 * model.sin_pa + b0 * model.cos_pa;
    phx_opcount::tally() = phx_opcount::Tally{};
    const core::pixel::RunStats rs = core::pixel::render_pixel(&model, alpha, beta, res.data());
    rows.push_back((unsigned long long)rs.steps);
    rows.push_back((unsigned long long)rs.nplasma);
    rows.push_back((unsigned long long)rs.bad);
    for (int k = 0; k < phx_opcount::kNumOps; k++) rows.push_back(phx_opcount::tally().n[k]);
  }
  FILE* o = std::fopen(out_path.c_str(), "wb");
  if (!o || std::fwrite(rows.data(), sizeof(unsigned long long), rows.size(), o) != rows.size()) return 1;
  std::fclose(o);
  std::printf("{\"pixels\": %zu, \"columns\": %d}\n", pix.size(), 3 + phx_opcount::kNumOps);
  host::bhac_io::free_model(&model);
  return 0;
}
