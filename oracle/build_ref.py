"""Build the reference renderer's own code paths into oracle/_ref/ (test infrastructure: the checker, not the product).

The reference (nohgz/phoenix) needs HDF5 for its CMake build and main.cpp, which this machine lacks, so its build
system is not used.  Instead its hot-path headers are compiled where they lie with a driver of ours:

  ref_render_fp64 / ref_render_fp32   oracle/ref_harness.cpp + the reference's src/core/, host/io/config.hpp and
                                      host/io/bhac_io.hpp, g++ -O3 -fopenmp, ACCURACY=FP64 / FP32
                                      (the reference's CPU/OpenMP path, src/host/render/jobs.hpp:50-92)
  ref_gpu_fp32                        oracle/ref_gpu_driver.cu + the reference's src/device/kernel.cu, nvcc for sm_100a,
                                      ACCURACY=FP32 (the reference's CUDA path, src/device/kernel.cu:284-360)

Outputs go to oracle/_ref/ only (git-ignored; they travel with the working tree).  Nothing is built when the reference
tree is absent.  The tree is taken from --src, else from the PHX_REFERENCE_SRC environment variable, else from a
checkout named `reference` beside this repository.
Usage: python oracle/build_ref.py [--src /path/to/reference] [--no-gpu]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")


def default_src() -> str:
    """PHX_REFERENCE_SRC, else a `reference` checkout next to the repository."""
    env = os.environ.get("PHX_REFERENCE_SRC")
    return env if env else os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference"))


def _newer(target: str, deps) -> bool:
    return os.path.exists(target) and all(os.path.getmtime(target) >= os.path.getmtime(d) for d in deps)


def build(src: str = "", gpu: bool = True, verbose: bool = False) -> dict:
    built = {}
    src = src or default_src()
    inc = os.path.join(src, "src")
    if not os.path.isdir(inc):
        return built
    os.makedirs(OUT, exist_ok=True)
    harness = os.path.join(HERE, "ref_harness.cpp")
    for prec in ("FP64", "FP32"):
        exe = os.path.join(OUT, "ref_render_" + prec.lower())
        if not _newer(exe, [harness]):
            cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", f"-DACCURACY={prec}", "-DPHX_GPU_ENABLED=0",
                   "-DPHX_MAX_FREQS=32", "-DPHX_CAMERA_PHI=1", "-I" + inc, harness, "-o", exe]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        built["cpu_" + prec.lower()] = exe
    drv = os.path.join(HERE, "ref_gpu_driver.cu")
    if gpu and shutil.which("nvcc") and os.path.exists(drv):
        exe = os.path.join(OUT, "ref_gpu_fp32")
        kernel = os.path.join(inc, "device", "kernel.cu")
        if not _newer(exe, [drv]):
            cmd = ["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
                   "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets", "-DACCURACY=FP32", "-DPHX_GPU_ENABLED=1",
                   "-DPHX_MAX_FREQS=1", "-DPHX_CAMERA_PHI=1", "-DGPU_BLOCK=128", "-DGPU_MINBLOCKS=3",
                   "-Xcompiler", "-fopenmp", "-I" + inc, drv, kernel, "-o", exe, "-lgomp"]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        built["gpu_fp32"] = exe
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default="")
    ap.add_argument("--no-gpu", action="store_true")
    a = ap.parse_args()
    res = build(a.src, gpu=not a.no_gpu, verbose=True)
    print(res if res else "reference tree not found: nothing built", file=sys.stderr)
