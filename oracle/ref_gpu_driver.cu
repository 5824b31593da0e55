// Driver for the reference renderer's own CUDA path (test infrastructure: a baseline, not the product).
//
// Compiled with the reference's unmodified src/device/kernel.cu where it lies (see oracle/build_ref.py).  It does what
// PHOENIX's main() does for a GPU build (src/main.cpp:120-205) minus HDF5 output:
//   host::config::load_config (host/io/config.hpp:229) -> host::bhac_io::load_bhac_grid (bhac_io.hpp:143)
//   -> host::bhac_io::load (bhac_io.hpp:331, host decode) -> device::render (device/kernel.cu:284-360) over the
//   Morton-ordered job list.
// The Morton order is restated here (host/render/jobs.hpp:18-45 is not compiled: its header pulls in HDF5): jobs
// i * H + j sorted by the bit interleave of i (even bits) and j (odd bits).
//
// usage: ref_gpu CONFIG [section.key=value ...] [--inclinations A,B,...] [--repeat R] [--out FILE]
// Prints one JSON line per pass with the reference's own timings (device::Info: upload_s, kernel_s, the sum of its
// CUDA-event-timed chunk launches) and counters; --out writes the last image's FreqOut records.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "device/kernel.cuh"
#include "host/io/bhac_io.hpp"
#include "host/io/config.hpp"

static std::vector<int> morton_jobs(int W, int H) {
  std::vector<std::pair<unsigned long long, int>> keyed((size_t)W * H);
  for (int i = 0; i < W; i++)
    for (int j = 0; j < H; j++) {
      unsigned long long z = 0;
      for (int b = 0; b < 16; b++)
        z |= ((unsigned long long)((i >> b) & 1) << (2 * b)) | ((unsigned long long)((j >> b) & 1) << (2 * b + 1));
      keyed[(size_t)i * H + j] = {z, i * H + j};
    }
  std::sort(keyed.begin(), keyed.end());
  std::vector<int> jobs(keyed.size());
  for (size_t n = 0; n < keyed.size(); n++) jobs[n] = keyed[n].second;
  return jobs;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s CONFIG [key=value ...] [--inclinations A,B] [--repeat R] [--out F]\n", argv[0]);
    return 2;
  }
  const std::string cfg = argv[1];
  std::vector<std::string> overrides;
  std::vector<double> incls;
  std::string out_path;
  int repeat = 1;
  for (int i = 2; i < argc; i++) {
    const std::string a = argv[i];
    if (a == "--inclinations" && i + 1 < argc) {
      std::string t = argv[++i];
      size_t p0 = 0;
      for (;;) {
        const size_t p1 = t.find(',', p0);
        const std::string tok = t.substr(p0, p1 == std::string::npos ? std::string::npos : p1 - p0);
        if (!tok.empty()) incls.push_back(std::atof(tok.c_str()));
        if (p1 == std::string::npos) break;
        p0 = p1 + 1;
      }
    } else if (a == "--repeat" && i + 1 < argc) {
      repeat = std::max(1, std::atoi(argv[++i]));
    } else if (a == "--out" && i + 1 < argc) {
      out_path = argv[++i];
    } else {
      overrides.push_back(a);
    }
  }
  core::bhac::Model model = {};
  host::config::Params params;
  try {
    host::config::load_config(cfg, overrides, params, &model.uparams);
    host::bhac_io::load_bhac_grid(&model.gparams, params.grid_file);
    host::bhac_io::load(&model, params.dump_file, false);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_gpu: %s\n", e.what());
    return 1;
  }
  const int W = model.uparams.img_width, H = model.uparams.img_height, F = model.uparams.nfreqs;
  const std::vector<int> jobs = morton_jobs(W, H);
  std::vector<device::FreqOut> res((size_t)W * H * F);
  if (incls.empty()) incls.push_back(model.uparams.inclination);
  try {
    for (int pass = 0; pass < repeat; pass++) {
      double kernel_s = 0.0, upload_s = 0.0;
      long steps = 0, nplasma = 0, bad = 0;
      device::Info info;
      for (double incl : incls) {
        model.uparams.inclination = incl;
        std::memset(res.data(), 0, res.size() * sizeof(device::FreqOut));
        device::render(&model, params.dump_file.c_str(), jobs.data(), (int)jobs.size(), res.data(), &info, nullptr,
                       nullptr);
        kernel_s += info.kernel_s;
        upload_s += info.upload_s;
        steps += info.steps;
        nplasma += info.nplasma;
        bad += info.bad;
      }
      std::printf("{\"pass\": %d, \"images\": %d, \"pixels\": %ld, \"steps\": %ld, \"nplasma\": %ld, \"bad\": %ld, "
                  "\"kernel_s\": %.6f, \"upload_s\": %.6f, \"regs\": %d, \"local_bytes\": %d, \"blocks\": %d, "
                  "\"block\": %d, \"device\": \"%s\"}\n",
                  pass, (int)incls.size(), (long)W * H * (long)incls.size(), steps, nplasma, bad, kernel_s, upload_s,
                  info.regs, info.local_bytes, info.blocks, info.block, info.device);
      std::fflush(stdout);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_gpu: %s\n", e.what());
    return 1;
  }
  if (!out_path.empty()) {
    FILE* f = std::fopen(out_path.c_str(), "wb");
    if (!f || std::fwrite(res.data(), sizeof(device::FreqOut), res.size(), f) != res.size()) return 1;
    std::fclose(f);
  }
  return 0;
}
