"""Build the PHOENIX-B200 native code in-tree (phoenix_b200/_build/).

  libphoenix_b200.so   the C ABI of include/phoenix_b200.h: sm_100a raymarch kernels + C++17 host code
  PHOENIX              the command-line renderer (same CLI, config keys and outputs as the reference's PHOENIX)
  phx_gen_snapshot     seeded synthetic BHAC snapshot generator

Everything is compiled for sm_100a only (nvcc -gencode arch=compute_100a,code=sm_100a); the host parts with g++
-std=c++17 -fopenmp.  Objects are rebuilt when a source or any header under csrc/ or include/ is newer.
usage: python -m phoenix_b200.build [-j N] [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp", "-Xptxas", "-v",
              "--expt-relaxed-constexpr"] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wextra"]

LIB = os.path.join(BUILD, "libphoenix_b200.so")
CLI = os.path.join(BUILD, "PHOENIX")
GEN = os.path.join(BUILD, "phx_gen_snapshot")

DEVICE_SRC = ["device/march_fp64_f64.cu", "device/march_fp64_f32.cu", "device/march_fp32_nf1.cu", "device/march_fp32_nf4.cu",
              "device/march_mixed_nf1.cu", "device/march_mixed_nf4.cu", "device/march_dispatch.cu", "device/capi.cu",
              "device/queue_fp32_nf1.cu", "device/queue_fp32_nf4.cu", "device/queue_mixed.cu", "device/queue_fp64.cu",
              "device/queue_dispatch.cu", "device/batch.cu", "device/server.cu",
              "device/decode.cu", "device/spectrum.cu", "device/peak.cu"]
HOST_SRC = ["host/snapshot.cpp", "host/output.cpp", "host/hdf5_writer.cpp"]
# The FP64 kernels follow the reference's FP64 CPU arithmetic, which rounds every product and sum separately: no
# multiply-add contraction there (explicit fma() calls stay fused).
NVCC_FILE_FLAGS = {src: ["-fmad=false"] for src in ("device/march_fp64_f64.cu", "device/march_fp64_f32.cu",
                                                     "device/queue_fp64.cu")}
CLI_SRC = ["host/main.cpp", "host/config.cpp"]


def _headers():
    hs = glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    hs += glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True)
    hs += glob.glob(os.path.join(CSRC, "**", "*.inc"), recursive=True)
    hs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose, log=None):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if log:
        with open(log, "w") as f:
            f.write(r.stdout)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ... " + cmd[-1])
    return r.stdout


def build(jobs: int = 0, force: bool = False, verbose: bool = False) -> dict:
    if not shutil.which("nvcc"):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build phoenix_b200")
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    objs, tasks = [], []
    for src in DEVICE_SRC + HOST_SRC:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src.replace("/", "_") + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            if src.endswith(".cu"):
                cmd = ["nvcc"] + NVCC_FLAGS + NVCC_FILE_FLAGS.get(src, []) + ["-I" + INCLUDE, "-c", path, "-o", obj]
            else:
                cmd = ["g++"] + CXX_FLAGS + ["-I" + INCLUDE, "-c", path, "-o", obj]
            tasks.append((cmd, obj + ".log"))
    n = jobs if jobs > 0 else max(1, min(len(tasks), os.cpu_count() or 4))
    with ThreadPoolExecutor(max_workers=n) as ex:
        for f in [ex.submit(_run, c, verbose, log) for c, log in tasks]:
            f.result()
    if force or tasks or _stale(LIB, objs):
        _run(["nvcc", "-shared"] + ARCH + ["-Xcompiler", "-fopenmp", "-o", LIB] + objs + ["-lgomp"], verbose)
    out = {"lib": LIB}
    # command-line renderer
    cli_src = [os.path.join(CSRC, s) for s in CLI_SRC]
    if all(os.path.exists(s) for s in cli_src):
        if force or _stale(CLI, cli_src + headers + [LIB]):
            _run(["g++"] + CXX_FLAGS + ["-I" + INCLUDE] + cli_src + ["-o", CLI, "-L" + BUILD, "-lphoenix_b200",
                                                                    "-Wl,-rpath,$ORIGIN"], verbose)
        out["cli"] = CLI
    gen_src = os.path.join(CSRC, "tools", "gen_snapshot.cpp")
    if force or _stale(GEN, [gen_src] + headers):
        _run(["g++"] + CXX_FLAGS + [gen_src, "-o", GEN], verbose)
    out["gen"] = GEN
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, a.verbose))
