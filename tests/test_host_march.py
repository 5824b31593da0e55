"""The raymarch's own code (core/ray.cuh and everything it includes), compiled for the host by g++, against the
reference's golden per-pixel statistics (CPU).

The kernels' Ray state machine is host-and-device code: compiled with g++ (IEEE arithmetic, no multiply-add
contraction, glibc's libm) it runs each pixel's march on the CPU exactly as a GPU lane does, minus the device's
fast-math intrinsics.  The FP64 path and the mixed path (FP64 geodesic, FP32 plasma stage) must then take the
reference's steps and plasma segments pixel for pixel on every golden case: that pins the algorithm -- step-size rule,
liveness, turning points, leaf lookup, sample placement -- independently of the GPU's arithmetic.
"""
from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT, golden_arrays
from tests.golden.cases import CASES, SNAPSHOTS, case_params

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host/render_setup.hpp"
#include "host/snapshot.hpp"

using namespace phx;

template <class R, class PT>
SnapView<R, PT> view(const HostSnapshot& h, const R* lb, const R* dxc, const PT* prim, const std::vector<int32_t>& fmap) {
  SnapView<R, PT> v{};
  v.lb = lb;
  v.dxc = dxc;
  v.prim = prim;
  v.fmap = fmap.data();
  for (int d = 0; d < 3; d++) {
    v.fd[d] = h.ng[d] << (h.nlevels - 1);
    v.nx[d] = h.nx[d];
    v.x_lo[1 + d] = R(h.x_lo[d]);
    v.x_hi[1 + d] = R(h.x_hi[d]);
    v.w0[d] = R((h.x_hi[d] - h.x_lo[d]) / h.ng[d]);
    v.iw0up[d] = R(double(1 << (h.nlevels - 1)) * h.ng[d] / (h.x_hi[d] - h.x_lo[d]));
    v.xlo_d[1 + d] = h.x_lo[d];
    v.xhi_d[1 + d] = h.x_hi[d];
    v.w0_d[d] = (h.x_hi[d] - h.x_lo[d]) / h.ng[d];
  }
  v.nleafs = h.nleafs;
  v.nlevels = h.nlevels;
  v.cells = h.cells;
  v.a = R(h.a);
  v.hs = R(h.hslope);
  v.gam = R(h.gam);
  v.lbd = h.lb.data();
  v.dxcd = h.dxc.data();
  v.a_d = h.a;
  v.hs_d = h.hslope;
  return v;
}

template <Mode M, class PT>
void march(const SnapView<typename Policy<M>::R, PT>& s, const SnapView<double, PT>& sd, const PhxRenderParams& p,
           const HostSnapshot& h, std::vector<int>& out) {
  const auto rc = make_consts<typename Policy<M>::R>(p, h.a, h.hslope);
  const int n = p.img_width * p.img_height;
  out.assign(2 * (size_t)n, 0);
#pragma omp parallel for schedule(dynamic, 16)
  for (int pix = 0; pix < n; pix++) {
    Ray<M, PT, 1> ray;
    RayCounters ctr{};
    ray.init(s, sd, rc, pix);
    while (ray.advance(s, sd, rc, ctr)) {
    }
    out[2 * (size_t)pix] = ray.steps;
    out[2 * (size_t)pix + 1] = ray.nplasma;
  }
}

// usage: march dump grid nlevels sfc W H incl freq m_unit fov_x fov_y phi pa out
int main(int argc, char** argv) {
  if (argc != 15) return 2;
  SnapshotOptions o;
  o.nlevels = std::atoi(argv[3]);
  o.sfc = std::atoi(argv[4]) != 0;
  o.keep_f64 = true;
  const HostSnapshot h = load_bhac(argv[1], argv[2], o);
  const std::vector<int32_t> fmap = flatten_level_maps(h.level_map, h.ng, h.nlevels);
  const std::vector<float> lbf(h.lb.begin(), h.lb.end()), dxf(h.dxc.begin(), h.dxc.end());
  PhxRenderParams p;
  phx_default_params(&p);
  p.img_width = std::atoi(argv[5]);
  p.img_height = std::atoi(argv[6]);
  p.inclination = std::atof(argv[7]);
  p.frequencies[0] = std::atof(argv[8]);
  p.m_unit = std::atof(argv[9]);
  p.fov_x = std::atof(argv[10]);
  p.fov_y = std::atof(argv[11]);
  p.phi = std::atof(argv[12]);
  p.pa = std::atof(argv[13]);
  const auto s64 = view<double, double>(h, h.lb.data(), h.dxc.data(), h.prim_f64.data(), fmap);
  const auto s32 = view<float, float>(h, lbf.data(), dxf.data(), h.prim_f32.data(), fmap);
  const auto s32d = s32.fp64_view();
  std::vector<int> a, b;
  p.precision = PHX_PREC_FP64;
  march<Mode::kFP64, double>(s64, s64, p, h, a);
  p.precision = PHX_PREC_MIXED;
  march<Mode::kMixed, float>(s32, s32d, p, h, b);
  FILE* f = std::fopen(argv[14], "wb");
  std::fwrite(a.data(), sizeof(int), a.size(), f);
  std::fwrite(b.data(), sizeof(int), b.size(), f);
  std::fclose(f);
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(built, tmp_path_factory):
    d = tmp_path_factory.mktemp("host_march")
    src, exe = d / "march.cpp", d / "march"
    src.write_text(DRIVER)
    csrc = os.path.join(ROOT, "phoenix_b200", "csrc")
    lib = os.path.dirname(built["lib"])
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-fopenmp", "-I" + csrc, "-I" + os.path.join(ROOT, "include"),
                           str(src), os.path.join(csrc, "host", "snapshot.cpp"), "-o", str(exe), "-L" + lib,
                           "-lphoenix_b200", "-Wl,-rpath," + lib])
    return str(exe)


@pytest.mark.parametrize("name", sorted(CASES))
def test_host_march_takes_the_reference_steps(driver, snapshots, name, tmp_path):
    """FP64 and mixed marches, pixel by pixel: the reference's steps and plasma segments exactly."""
    case = CASES[name]
    dump, grid, spec = snapshots[case["snapshot"]]
    kw = case_params(name)
    W, H = kw["img_width"], kw["img_height"]
    out = tmp_path / "stats.bin"
    subprocess.check_call([driver, dump, grid, str(spec["nlevels"]), "1" if spec["sfc"] else "0", str(W), str(H),
                           repr(kw["inclination"]), repr(kw["frequencies"][0]), repr(kw["m_unit"]), repr(kw["fov_x"]),
                           repr(kw["fov_y"]), repr(kw["phi"]), repr(kw["pa"]), str(out)])
    st = np.fromfile(str(out), dtype=np.int32).reshape(2, W, H, 2)
    ref = golden_arrays(name)["stats_fp64"][..., :2]
    for mode, got in (("fp64", st[0]), ("mixed", st[1])):
        diff = np.argwhere((got != ref).any(axis=-1))
        assert len(diff) == 0, (mode, len(diff), diff[:8].tolist())
