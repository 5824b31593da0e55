"""Algorithmic FP32 flops per unit of raymarch work, counted in the reference's own code -- TEST INFRASTRUCTURE ONLY.

Builds oracle/_ref/count_ops (oracle/opcount/count_ops.cpp against the reference's unmodified headers, with the
op-counting `scalar` of oracle/opcount/), renders strided pixel samples of a workload at one and at three frequencies,
and fits per-pixel flop totals to

    flops(pixel) = F_step * steps + F_sample * emitting samples + F_freq * emitting samples * frequencies

by least squares (no per-ray term: the per-ray set-up is FP64 and uncounted).  Flops: additions, subtractions and multiplications count 1; a division or square root, and each
transcendental, counts the FP32 instructions of an accurate GPU evaluation (WEIGHTS).  Comparisons, min/max/abs are
tallied but are not flops.  The FP64 camera set-up of each ray is not `scalar` arithmetic and is not counted.

usage: python oracle/opcount/count_flops.py [--src REFERENCE_TREE] [--workload plain|cfg1] [--stride N]
Prints one JSON object (the fitted constants, their residual, and the operation mix per ray-step).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
sys.path.insert(0, ROOT)
sys.path.insert(0, ORACLE)

OPS = ["add", "mul", "div", "sqrt", "cmp", "minmaxabs", "exp", "log", "sin", "cos", "pow", "cbrt", "acos", "expm1",
       "tanh", "sinh", "cosh", "acosh", "fmod", "floor"]
# FP32 flop equivalents per operation
WEIGHTS = dict(add=1, mul=1, div=4, sqrt=4, cmp=0, minmaxabs=0, exp=8, log=8, sin=10, cos=10, pow=20, cbrt=12,
               acos=12, expm1=10, tanh=10, sinh=10, cosh=10, acosh=16, fmod=4, floor=1)


def build(src: str) -> str:
    exe = os.path.join(ORACLE, "_ref", "count_ops")
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-DPHX_GPU_ENABLED=0", "-DPHX_MAX_FREQS=32", "-DPHX_CAMERA_PHI=1",
           "-I" + HERE, "-I" + os.path.join(src, "src"), os.path.join(HERE, "count_ops.cpp"), "-o", exe]
    subprocess.check_call(cmd)
    return exe


def counts(exe, cfg, pixels, tmp, overrides=()):
    pfile, ofile = os.path.join(tmp, "pix.bin"), os.path.join(tmp, "ops.bin")
    np.asarray(pixels, dtype=np.int32).tofile(pfile)
    subprocess.check_call([exe, cfg, *overrides, "--pixels", pfile, "--out", ofile], stdout=subprocess.DEVNULL)
    return np.fromfile(ofile, dtype=np.uint64).reshape(len(pixels), 3 + len(OPS)).astype(np.float64)


def main():
    import build_ref
    from tests.golden.cases import write_config
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default="")
    ap.add_argument("--workload", default="plain", choices=["plain", "cfg1"])
    ap.add_argument("--stride", type=int, default=0)
    a = ap.parse_args()
    exe = build(a.src or build_ref.default_src())
    import bench
    if a.workload == "plain":
        w = dict(bench.WORKLOAD)
        dump, grid = bench.snapshot_files(w)
        stride = a.stride or 997
    else:
        w = dict(bench.WORKLOAD, img=64, nlevels=3)
        dump, grid = bench.generated_snapshot(bench.BATCH["gen"])
        stride = a.stride or 7
    npix = w["img"] * w["img"]
    pix = np.arange(0, npix, stride, dtype=np.int64)
    pix = ((pix + (pix // w["img"]) * 7) % npix).astype(np.int32)
    rows, nf = [], []
    with tempfile.TemporaryDirectory() as tmp:
        for incl in w["inclinations"]:
            case = dict(snapshot="cfg1", inclination=incl, img_width=w["img"], img_height=w["img"],
                        frequencies=[w["frequency"]], m_unit=w["m_unit"])
            cfg = os.path.join(tmp, "c.toml")
            write_config(cfg, case, dump, grid, tmp)
            with open(cfg) as f:
                text = f.read().replace("nlevels = 3", f"nlevels = {w['nlevels']}")
            with open(cfg, "w") as f:
                f.write(text)
            for freqs in ([w["frequency"]], [86e9, 230e9, 345e9]):
                over = ["camera.frequency_list=[" + ", ".join(repr(x) for x in freqs) + "]"]
                c = counts(exe, cfg, pix, tmp, over)
                rows.append(c)
                nf.append(np.full(len(pix), len(freqs), dtype=np.float64))
    c = np.concatenate(rows)
    nfreq = np.concatenate(nf)
    steps, nplasma = c[:, 0], c[:, 1]
    ops = c[:, 3:]
    w_vec = np.array([WEIGHTS[o] for o in OPS], dtype=np.float64)
    flops = ops @ w_vec
    live = steps > 0
    X = np.stack([steps, nplasma, nplasma * nfreq], axis=1)[live]
    coef, *_ = np.linalg.lstsq(X, flops[live], rcond=None)
    pred = X @ coef
    resid = float(np.abs(pred - flops[live]).sum() / flops[live].sum())
    tot_steps = steps.sum()
    mix = {o: float(ops[:, k].sum() / tot_steps) for k, o in enumerate(OPS)}
    out = {"workload": a.workload, "pixels_per_run": int(len(pix)), "runs": len(rows),
           "F_step": float(coef[0]), "F_sample": float(coef[1]), "F_freq": float(coef[2]),
           "fit_residual_l1": resid, "weights": WEIGHTS, "ops_per_step": mix,
           "flops_total": float(flops.sum()), "steps_total": float(tot_steps), "samples_total": float(nplasma.sum())}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
