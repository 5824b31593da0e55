// PHOENIX command-line renderer on the B200 path: the reference's CLI (src/main.cpp:88-242) over this library.
//
//   PHOENIX [config.toml] [section.key=value ...]        (default config: input/config.toml; -h / --help)
//
// Same config keys, overrides, console messages, output files (img_data.h5, image[_f].dat, spectrum.dat) and
// per-frequency flux line.  Settings of this build that the reference fixes at compile time are read from the
// environment so that config files stay valid for both: PHX_PRECISION = fp32 (default) | fp64 | mixed,
// PHX_PERIOD (march passes between lane refills), PHX_BLOCKS_PER_SM (register-cap variant).
// PHX_PRINT_CONFIG=1 prints the parsed configuration as JSON and exits.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/phoenix_b200.h"
#include "config.hpp"
#include "output.hpp"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void say(const char* tag, const char* fmt, va_list ap) {
  std::fprintf(stderr, "%s", tag);
  std::vfprintf(stderr, fmt, ap);
}
void infomsg(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  say("[ \033[1;36mINFO\033[0m ] ", fmt, ap);
  va_end(ap);
}
void okmsg(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  say("\r[ \033[1;32m OK \033[0m ] ", fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "\n");
}
void failmsg(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  say("\r[ \033[1;31mFAIL\033[0m ] ", fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "\n");
}
void warnmsg(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  say("[ \033[1;33mWARN\033[0m ] ", fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "\n");
}
void timemsg(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  say("[ \033[1;33mTIME\033[0m ] ", fmt, ap);
  va_end(ap);
}
void hline() {
  for (int i = 0; i < 75; i++) std::fprintf(stderr, "─");
  std::fprintf(stderr, "\n");
}

int env_int(const char* name, int fallback) {
  const char* e = std::getenv(name);
  return (e && std::atoi(e) > 0) ? std::atoi(e) : fallback;
}

void print_config(const phx::RunConfig& c) {
  const PhxRenderParams& p = c.render;
  std::printf("{\"show_header\": %s, \"outdir\": \"%s\", \"image\": \"%s\", \"block_size\": %d, \"dump_file\": \"%s\", "
              "\"grid_file\": \"%s\", \"gpu_decode\": %s, \"nspin\": %d, \"bpol\": %d, \"sfc\": %d, \"nlevels\": %d, "
              "\"inclination\": %.17g, \"img_width\": %d, \"img_height\": %d, \"fov_x\": %.17g, \"fov_y\": %.17g, "
              "\"r_cam\": %.17g, \"t_init\": %.17g, \"pa\": %.17g, \"phi\": %.17g, \"mass\": %.17g, \"distance\": "
              "%.17g, \"stepsize\": %.17g, \"max_steps\": %d, \"horizon_margin\": %.17g, \"max_order\": %d, "
              "\"m_unit\": %.17g, \"r_low\": %.17g, \"r_high\": %.17g, \"beta_c\": %.17g, \"sigma_cut\": %.17g, "
              "\"thetae_min\": %.17g, \"thetae_max\": %.17g, \"rt_outer\": %.17g, \"frequencies\": [",
              c.show_header ? "true" : "false", c.outdir.c_str(), c.image.c_str(), c.block_size, c.dump_file.c_str(),
              c.grid_file.c_str(), c.gpu_decode ? "true" : "false", c.read.nspin, c.read.bpol, c.read.sfc,
              c.read.nlevels, p.inclination, p.img_width, p.img_height, p.fov_x, p.fov_y, p.r_cam, p.t_init, p.pa, p.phi,
              p.mass, p.distance, p.stepsize, p.max_steps, p.horizon_margin, p.max_order, p.m_unit, p.r_low, p.r_high,
              p.beta_c, p.sigma_cut, p.thetae_min, p.thetae_max, p.rt_outer);
  for (int f = 0; f < p.nfreqs; f++) std::printf("%s%.17g", f ? ", " : "", p.frequencies[f]);
  std::printf("]}\n");
}

}  // namespace

int main(int argc, char** argv) {
  const double t_start = now_s();
  std::string cfgpath = "input/config.toml";
  int first = 1;
  if (argc > 1 && std::strchr(argv[1], '=') == nullptr) {
    if (!std::strcmp(argv[1], "-h") || !std::strcmp(argv[1], "--help")) {
      infomsg("usage: %s [input/config.toml] [section.key=value ...]\n", argv[0]);
      return 0;
    }
    cfgpath = argv[1];
    first = 2;
  }
  const std::vector<std::string> overrides(argv + first, argv + argc);

  phx::RunConfig cfg;
  try {
    cfg = phx::load_config(cfgpath, overrides);
  } catch (const std::exception& e) {
    failmsg("%s", e.what());
    return EXIT_FAILURE;
  }
  if (std::getenv("PHX_PRINT_CONFIG")) {
    print_config(cfg);
    return 0;
  }
  PhxRenderParams& p = cfg.render;
  const char* prec = std::getenv("PHX_PRECISION");
  p.precision = !prec ? PHX_PREC_FP32
                      : !std::strcmp(prec, "fp64") ? PHX_PREC_FP64
                                                   : !std::strcmp(prec, "mixed") ? PHX_PREC_MIXED : PHX_PREC_FP32;
  p.period = env_int("PHX_PERIOD", 0);
  p.blocks_per_sm = env_int("PHX_BLOCKS_PER_SM", 0);

  if (cfg.show_header) {
    std::fprintf(stderr, "\n  PHOENIX — GRRT raymarcher (B200 path, %s)\n", phx_version());
    hline();
  }
  infomsg("Input Filepaths\n");
  okmsg("Load config file      \"%s\"", cfgpath.c_str());
  const double t_model = now_s();
  PhxSnapshot* snap = nullptr;
  const int32_t flags = (p.precision == PHX_PREC_FP64 ? PHX_SNAP_F64_PRIMS : 0) | (cfg.gpu_decode ? PHX_SNAP_GPU_DECODE : 0);
  if (phx_snapshot_load(cfg.dump_file.c_str(), cfg.grid_file.c_str(), &cfg.read, flags, &snap) != PHX_OK) {
    failmsg("%s", phx_last_error());
    return EXIT_FAILURE;
  }
  okmsg("Load GRMHD data       \"%s\"", cfg.dump_file.c_str());
  timemsg(" ⇥ Loaded in %.2f s (%.3f GB resident on the device)\n", now_s() - t_model,
          phx_snapshot_bytes(snap) * 1e-9);
  hline();
  infomsg("Precision: %s\n", p.precision == PHX_PREC_FP64 ? "FP64" : p.precision == PHX_PREC_MIXED ? "MIXED" : "FP32");
  infomsg("Black Hole & Plasma:\n     ⇥ Mass    = %.4e M_sun\n     ⇥ Dist    = %.4e kpc\n     ⇥ M_unit  = "
          "%.2e grams\n     ⇥ r_low   = %g\n     ⇥ r_high  = %g\n     ⇥ beta_c  = %g\n",
          p.mass, p.distance, p.m_unit, p.r_low, p.r_high, p.beta_c);
  infomsg("Camera:\n     ⇥ Inclination = %g deg\n     ⇥ Azimuth     = %g deg\n     ⇥ Pos. Angle  = %g deg\n"
          "     ⇥ Resolution  = %d x %d px\n     ⇥ FOV         = %g x %g Rg\n     ⇥ r_cam       = %g Rg\n"
          "     ⇥ Frequencies = %d\n",
          p.inclination, p.phi, p.pa, p.img_width, p.img_height, p.fov_x, p.fov_y, p.r_cam, p.nfreqs);
  hline();

  const size_t npix = (size_t)p.img_width * p.img_height;
  std::vector<PhxFreqOut> res(npix * p.nfreqs);
  std::memset(res.data(), 0, res.size() * sizeof(PhxFreqOut));
  PhxRenderInfo gi;
  const double t_ray = now_s();
  if (phx_render(snap, &p, nullptr, 0, res.data(), &gi) != PHX_OK) {
    failmsg("%s", phx_last_error());
    phx_snapshot_destroy(snap);
    return EXIT_FAILURE;
  }
  timemsg("Raymarch: %.2f s\n", now_s() - t_ray);
  infomsg(" ⇥ Model upload %.2f s, kernel %.2f s\n", gi.upload_s, gi.kernel_s);
  hline();
  long badpix = 0;
  for (size_t q = 0; q < npix; q++) {
    int nonfinite = 0;
    for (int f = 0; f < p.nfreqs; f++)
      for (int c = 0; c < 4; c++) nonfinite |= !std::isfinite(res[q * p.nfreqs + f].IQUV[c]);
    badpix += nonfinite;
  }
  infomsg("%.0f geodesic samples/pixel, %.0f plasma segments/pixel (mean)\n", (double)gi.steps / npix,
          (double)gi.nplasma / npix);
  infomsg("Non-finite segment operators: %ld, pixels with non-finite IQUV: %ld\n", (long)gi.bad, badpix);
  infomsg("Device: %s, %d SMs\n", gi.device, gi.sms);
  infomsg("Launch: %d blocks x %d threads, %d registers/thread, %d B local memory/thread\n", gi.blocks, gi.block,
          gi.regs, gi.local_bytes);

  mkdir(cfg.outdir.c_str(), 0755);
  okmsg("Create output directory \"%s\"", cfg.outdir.c_str());
  hline();
  const double t_out = now_s();
  bool want_text = cfg.image == "text" || cfg.image == "both";
  const bool want_h5 = cfg.image == "hdf5" || cfg.image == "both";
  if (want_h5) {
    const std::string hp = cfg.outdir + "/img_data.h5";
    std::string err;
    if (phx::write_image_hdf5(hp, p, cfg.block_size, res, &err)) {
      okmsg("Wrote %s", hp.c_str());
    } else {
      if (!err.empty()) std::fprintf(stderr, "%s\n", err.c_str());
      warnmsg("Failed to write \"%s\" writing text instead...", hp.c_str());
      want_text = true;
    }
  }
  if (want_text) {
    for (int f = 0; f < p.nfreqs; f++) {
      const std::string ip = cfg.outdir + "/image" + (p.nfreqs == 1 ? "" : "_" + std::to_string(f)) + ".dat";
      phx::write_image_text(ip, p, res, f);
      okmsg("Wrote %s", ip.c_str());
    }
  }
  const std::string sp = cfg.outdir + "/spectrum.dat";
  phx::write_spectrum(sp, p, res);
  okmsg("Wrote %s", sp.c_str());
  hline();
  for (int f = 0; f < p.nfreqs; f++) {
    double S[4];
    phx::compute_spec(p, res, f, S);
    infomsg("Flux at %.4e Hz (Jy): \033[1;38;5;160mI\033[0m %+.9e \033[1;38;5;77mQ\033[0m %+.9e \033[1;38;5;27mU\033[0m "
            "%+.9e \033[1;38;5;11mV\033[0m %+.9e\n",
            p.frequencies[f], S[0], S[1], S[2], S[3]);
  }
  timemsg("Output: %.2f s\n", now_s() - t_out);
  phx_snapshot_destroy(snap);
  timemsg("Execution: %.2f s\n", now_s() - t_start);
  return EXIT_SUCCESS;
}
