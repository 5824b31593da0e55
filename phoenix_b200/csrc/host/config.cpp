// config.toml reader (see config.hpp).
#include "config.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <stdexcept>

namespace phx {

namespace {

std::string trim(const std::string& t, const char* ws = " \t\r") {
  const size_t p = t.find_first_not_of(ws), q = t.find_last_not_of(ws);
  return p == std::string::npos ? std::string() : t.substr(p, q - p + 1);
}

bool starts_with(const std::string& s, const char* prefix) { return s.compare(0, std::strlen(prefix), prefix) == 0; }

}  // namespace

void parse_toml(const std::string& text, std::map<std::string, std::string>& kv) {
  std::istringstream in(text);
  std::string line, section;
  int ln = 0;
  while (std::getline(in, line)) {
    ln++;
    bool quoted = false;  // a '#' outside double quotes starts a comment
    for (size_t i = 0; i < line.size(); i++) {
      if (line[i] == '"') quoted = !quoted;
      if (line[i] == '#' && !quoted) {
        line.resize(i);
        break;
      }
    }
    line = trim(line);
    if (line.empty()) continue;
    if (line[0] == '[') {
      if (line.back() != ']') throw std::runtime_error("Line " + std::to_string(ln) + ": bad section header");
      section = trim(line.substr(1, line.size() - 2));
      continue;
    }
    const size_t eq = line.find('=');
    if (eq == std::string::npos) throw std::runtime_error("Line " + std::to_string(ln) + ": expected key = value");
    const std::string key = trim(line.substr(0, eq));
    std::string val = trim(line.substr(eq + 1));
    if (val.size() >= 2 && val.front() == '"' && val.back() == '"') val = val.substr(1, val.size() - 2);
    const std::string full = section.empty() ? key : section + "." + key;
    if (kv.count(full)) throw std::runtime_error("Line " + std::to_string(ln) + ": duplicate key " + full);
    kv[full] = val;
  }
}

void read_frequencies(const std::map<std::string, std::string>& kv, std::vector<std::string>& used,
                      std::vector<double>& out) {
  static const char* forms[4] = {"camera.frequency", "camera.frequency_list", "camera.frequency_linspace",
                                 "camera.frequency_logspace"};
  int given = 0, form = 0;
  for (int i = 0; i < 4; i++)
    if (kv.count(forms[i])) {
      given++;
      form = i;
    }
  if (given != 1) throw std::runtime_error("Too many (or no) frequency forms given!");
  const std::string key = forms[form];
  const std::string& text = kv.at(key);
  used.push_back(key);

  auto number = [&](const std::string& t) {
    char* end = nullptr;
    const double v = std::strtod(t.c_str(), &end);
    if (end == t.c_str() || *end != '\0') throw std::runtime_error(key + ": not a number: " + t);
    return v;
  };
  auto numbers = [&]() {
    const size_t a = text.find('['), b = text.rfind(']');
    if (a == std::string::npos || b == std::string::npos || b < a)
      throw std::runtime_error(key + " must be a list on ONE line: [a, b, ...]");
    std::vector<double> v;
    std::stringstream ss(text.substr(a + 1, b - a - 1));
    std::string tok;
    while (std::getline(ss, tok, ',')) {
      const std::string t = trim(tok, " \t");
      if (t.empty()) continue;  // trailing comma
      v.push_back(number(t));
    }
    return v;
  };

  out.clear();
  if (form == 0) {
    out.push_back(number(text));
  } else {
    const std::vector<double> v = numbers();
    if (form == 1) {
      if (v.empty()) throw std::runtime_error(key + " is empty!");
      out = v;
    } else {
      if (v.size() != 3)
        throw std::runtime_error(key + " has " + std::to_string(v.size()) + "arguments! (Expected 3)");
      const double lo = v[0], hi = v[1];
      if (!(v[2] >= 2.0 && v[2] <= 1e6) || v[2] != std::floor(v[2]))
        throw std::runtime_error(key + ": n must be an integer >= 2! (use frequency = nu for a single frequency)");
      if (!(lo > 0.0) || !(hi > lo)) throw std::runtime_error(key + ": need 0 < start < stop!");
      const int n = (int)v[2];
      for (int i = 0; i < n; i++) {
        const double x = double(i) / (n - 1);
        out.push_back(i == n - 1 ? hi : (form == 3 ? lo * std::pow(hi / lo, x) : lo + (hi - lo) * x));
      }
    }
  }
  std::set<std::string> seen;
  for (double v : out) {
    if (!(v > 0.0) || !std::isfinite(v)) throw std::runtime_error("frequencies must be positive and finite");
    char b[64];
    std::snprintf(b, sizeof b, "%e", v);
    if (!seen.insert(b).second)
      throw std::runtime_error(std::string("duplicate frequency ") + b + " (they are used to name the HDF5 datasets)");
  }
}

RunConfig load_config(const std::string& path, const std::vector<std::string>& overrides) {
  std::ifstream file(path);
  if (!file) throw std::runtime_error("Cannot open file " + path + ". Perhaps it's a malformed TOML key-value pair?");
  std::stringstream buf;
  buf << file.rdbuf();
  std::map<std::string, std::string> kv;
  parse_toml(buf.str(), kv);

  bool freq_override = false;
  for (const std::string& a : overrides) {
    const size_t eq = a.find('=');
    if (eq == std::string::npos) throw std::runtime_error("Override must be section.key=value: " + a);
    if (starts_with(a, "camera.frequenc") && !freq_override) {  // an override replaces every frequency form
      freq_override = true;
      for (auto it = kv.begin(); it != kv.end();) it = starts_with(it->first, "camera.frequenc") ? kv.erase(it) : std::next(it);
    }
    kv[a.substr(0, eq)] = a.substr(eq + 1);
  }

  RunConfig c;
  phx_default_params(&c.render);
  PhxRenderParams& p = c.render;
  std::vector<std::string> used;
  std::string missing;
  auto str = [&](const char* k, std::string& dst, bool required) {
    auto it = kv.find(k);
    if (it != kv.end()) {
      dst = it->second;
      used.push_back(k);
    } else if (required) {
      missing += std::string(" ") + k;
    }
  };
  auto dbl = [&](const char* k, double& dst, bool required) {
    std::string t;
    str(k, t, required);
    if (!t.empty()) dst = std::atof(t.c_str());
  };
  auto integer = [&](const char* k, int32_t& dst, bool required) {
    double v = dst;
    dbl(k, v, required);
    dst = (int32_t)v;
  };
  auto boolean = [&](const char* k, bool& dst, bool required) {
    std::string t;
    str(k, t, required);
    if (!t.empty()) dst = (t == "true" || t == "1");
  };

  boolean("visual.show_header", c.show_header, true);
  dbl("black_hole.mass", p.mass, true);
  dbl("black_hole.distance", p.distance, true);
  dbl("integration.stepsize", p.stepsize, true);
  integer("integration.max_steps", p.max_steps, true);
  dbl("integration.horizon_margin", p.horizon_margin, true);
  integer("integration.max_order", p.max_order, true);
  dbl("camera.inclination", p.inclination, true);
  integer("camera.img_width", p.img_width, true);
  integer("camera.img_height", p.img_height, true);
  dbl("camera.fov_x", p.fov_x, true);
  dbl("camera.fov_y", p.fov_y, true);
  dbl("camera.r_cam", p.r_cam, true);
  dbl("camera.t_init", p.t_init, true);
  p.pa = 0.0;
  p.phi = 0.0;
  dbl("camera.pa", p.pa, false);
  dbl("camera.phi", p.phi, false);
  try {
    read_frequencies(kv, used, c.frequencies);
    if (c.frequencies.size() > (size_t)PHX_MAX_FREQS)
      throw std::runtime_error("at most " + std::to_string(PHX_MAX_FREQS) + " frequencies (PHX_MAX_FREQS), got " +
                               std::to_string(c.frequencies.size()));
    p.nfreqs = (int32_t)c.frequencies.size();
    for (size_t f = 0; f < c.frequencies.size(); f++) p.frequencies[f] = c.frequencies[f];
  } catch (const std::exception& e) {
    throw std::runtime_error(path + ": " + e.what());
  }
  str("output.dir", c.outdir, true);
  str("output.image", c.image, false);
  integer("output.block_size", c.block_size, false);
  if (c.image != "hdf5" && c.image != "text" && c.image != "both" && c.image != "none")
    throw std::runtime_error(path + ": output.image must be hdf5, text, both or none");
  if (c.block_size < 1) throw std::runtime_error(path + ": output.block_size must be >= 1");
  str("grmhd.dump_file", c.dump_file, true);
  str("grmhd.grid_file", c.grid_file, true);
  boolean("grmhd.gpu_decode", c.gpu_decode, true);
  integer("grmhd.nspin", c.read.nspin, true);
  bool sfc = c.read.sfc != 0;
  boolean("grmhd.sfc", sfc, true);
  c.read.sfc = sfc ? 1 : 0;
  integer("grmhd.nlevels", c.read.nlevels, true);
  integer("grmhd.bpol", c.read.bpol, true);
  dbl("plasma.m_unit", p.m_unit, true);
  dbl("plasma.r_low", p.r_low, true);
  dbl("plasma.r_high", p.r_high, true);
  dbl("plasma.sigma_cut", p.sigma_cut, true);
  dbl("plasma.thetae_min", p.thetae_min, true);
  dbl("plasma.thetae_max", p.thetae_max, true);
  dbl("plasma.rt_outer", p.rt_outer, true);
  p.beta_c = 1.0;
  dbl("plasma.beta_c", p.beta_c, false);
  if (!(p.beta_c > 0.0)) throw std::runtime_error(path + ": plasma.beta_c must be > 0");
  if (!missing.empty()) throw std::runtime_error(path + ": missing required key(s):" + missing);
  for (const auto& e : kv)
    if (std::find(used.begin(), used.end(), e.first) == used.end())
      throw std::runtime_error(path + ": unknown key " + e.first);
  return c;
}

}  // namespace phx
