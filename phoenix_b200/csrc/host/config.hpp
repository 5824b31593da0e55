// config.toml + command-line overrides for the PHOENIX command line.  The accepted keys, their meaning, the override
// syntax and the error messages are the reference renderer's (src/host/io/config.hpp:35-381), so that its config
// files and scripts keep working:
//   * a TOML subset: [section] headers, key = value, '#' comments outside double quotes, "quoted" strings; a key
//     given twice is an error;
//   * `section.key=value` overrides; an override of any camera.frequenc* key first drops every frequency form the
//     file gave;
//   * exactly one frequency form: frequency, frequency_list [a, b, ...], frequency_linspace / frequency_logspace
//     [start, stop, n]; duplicate frequencies (by their "%e" spelling, which names the HDF5 datasets) are an error;
//   * typed required and optional keys; every missing required key is listed; any key not in the table is an error.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "../../../include/phoenix_b200.h"

namespace phx {

struct RunConfig {
  bool show_header = false;
  std::string outdir;
  std::string image = "hdf5";  // hdf5, text, both or none
  int block_size = 10;         // HDF5 pixels per block side
  std::string dump_file, grid_file;
  bool gpu_decode = false;
  PhxReadOptions read{3, 1, 1, -1};
  PhxRenderParams render{};
  std::vector<double> frequencies;
};

// Flat "section.key" -> raw value map of a config text.  Throws std::runtime_error("Line N: ...") on malformed input.
std::map<std::string, std::string> parse_toml(const std::string& text);

// The frequencies of the one frequency form present in `kv`; its key is appended to `consumed`.
// Throws std::runtime_error with the reference's messages.
std::vector<double> read_frequencies(const std::map<std::string, std::string>& kv,
                                     std::vector<std::string>& consumed);

// Loads `path`, applies the overrides, validates.  Throws std::runtime_error with the reference's messages.
RunConfig load_config(const std::string& path, const std::vector<std::string>& overrides);

}  // namespace phx
