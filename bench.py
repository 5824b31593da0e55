"""Benchmark of the PHOENIX-B200 raymarch path: ray-steps/s on the plain-GPU-path workload.

Workload (one bench step = one pass of the hot path over one batch): a synthetic BHAC-format snapshot with a
192x96x96 base grid in 8^3 blocks, base + 2 refinement levels (15.6M cells, 8 FP32 primitives per cell, 0.5 GB on the
device), seed 0; three 512x512 images at inclinations 10, 60 and 163 deg, 230 GHz, m_unit 1.2e18, FoV 40 r_g, the
reference's default integration settings.  Inputs are resident in HBM when the timed region starts; the snapshot
(0.5 GB) is larger than L2 and L2 is also flushed (256 MB write) before every timed step.

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp32|fp64|mixed]
Multi-GPU: one process per GPU under torch.distributed.run; every rank renders the same three images (weak scaling,
no data-path collective); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GEN = os.path.join(ROOT, "phoenix_b200", "_build", "phx_gen_snapshot")
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "ref_render_fp32")
REF_CPU64 = os.path.join(ROOT, "oracle", "_ref", "ref_render_fp64")
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_fp32")

WORKLOAD = dict(base=(192, 96, 96), nlevels=3, refine=(3.5, 25.0, 0.55), seed=0, img=512,
                inclinations=(10.0, 60.0, 163.0), frequency=230e9, m_unit=1.2e18)
# Algorithmic FP32 flops per unit of work: per ray-step (RK4 with four metric/Christoffel evaluations, step size),
# per emitting sample (metric, fluid, tetrad, pitch angle), per (sample, frequency) (coefficients, segment operator,
# accumulation).  Counted in the reference's own FP32 code with an op-counting scalar and fitted over pixel samples of
# this workload (oracle/opcount/count_flops.py --workload plain: 3445.2 / 869.7 / 1223.6, fit residual 0.4%; add,
# sub, mul 1 flop; div, sqrt 4; exp, log 8; sin, cos 10; other transcendentals 10-20), frozen here.
FLOPS = dict(step=3445.0, sample=870.0, freq=1224.0)
# Algorithmic bytes the march requests from the memory system: per emitting sample the 8 corners x 8 FP32 primitives
# of the trilinear gather (256 B); per step the flattened leaf-map entry (4 B) and the leaf's lb/dxc (24 B); per ray
# its job index (4 B) and one 48 B FreqOut record per frequency.
BYTES = dict(sample=256.0, step=28.0, ray=4.0, ray_freq=48.0)
# DRAM bytes (read + write) per ray-step of k_march, from an ncu capture of one launch of this workload (the 60 deg
# image, default job order and refill policy): dram__bytes_read.sum + dram__bytes_write.sum = 773.3 MB over the
# launch's 726.6M ray-steps.  Scaled to the average launch by its ray-steps.
DRAM_BYTES_PER_STEP = 1.064
# FMA-pipe share of active cycles of k_march on this workload (ncu sm__pipe_fma_cycles_active.avg.pct_of_peak_
# sustained_active, one launch of the 60 deg image, default job order and refill policy).
FMA_PIPE_ACTIVE = 0.465
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")


def measured_peaks():
    """HBM copy bandwidth measured on this pool's B200s, else the earlier measurement (6.65 TB/s)."""
    try:
        with open(PEAKS_FILE) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def job_list(P, p, order):
    """The plain path's job list of an image: the library's default pixel order for it ("auto": 4x8 tiles, centre
    first) or a named tile order."""
    shape = P.default_pixel_order(p) if order == "auto" else order
    return P.schedule_tiles(p.img_width, p.img_height, shape)


def order_desc(P, params, order):
    if order != "auto":
        return order
    names = {v: k for k, v in P.TILE_SHAPES.items()}
    return "auto: " + ", ".join(names[P.default_pixel_order(p)] for p in params)


def generated_snapshot(gen_args, root=None):
    """Generate (once per machine) a synthetic BHAC snapshot with phx_gen_snapshot; returns (dump, grid)."""
    key = hashlib.sha1(json.dumps(list(gen_args)).encode()).hexdigest()[:12]
    d = os.path.join(root or tempfile.gettempdir(), "phx_bench_" + key)
    dump, grid = os.path.join(d, "dump.dat"), os.path.join(d, "grid.in")
    done = os.path.join(d, "done")
    if not os.path.exists(done):
        os.makedirs(d, exist_ok=True)
        subprocess.check_call([GEN, "--out", d] + list(gen_args), stdout=subprocess.DEVNULL)
        open(done, "w").close()
    return dump, grid


def snapshot_files(w=WORKLOAD, root=None):
    """The plain-path workload's snapshot; returns (dump, grid)."""
    return generated_snapshot(["--seed", str(w["seed"]), "--base", *map(str, w["base"]), "--nlevels",
                               str(w["nlevels"]), "--nws", "0", "--refine", *map(str, w["refine"])], root)


def render_kwargs(w=WORKLOAD):
    return dict(img=w["img"], frequencies=[w["frequency"]], m_unit=w["m_unit"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _cpu_passes(dump, grid, w, stride, ncores, repeat, tmp):
    """Time `repeat` passes of the CPU path over a strided pixel sample of the workload's three images (snapshot read
    once).  Returns (kind, pixels per pass, [(steps, seconds) per pass])."""
    pix = np.arange(0, w["img"] * w["img"], stride, dtype=np.int64)
    pix = ((pix + (pix // w["img"]) * 7) % (w["img"] * w["img"])).astype(np.int32)
    if os.path.exists(REF_CPU):
        from tests.golden.cases import write_config
        case = dict(snapshot="cfg1", inclination=w["inclinations"][0], img_width=w["img"], img_height=w["img"],
                    frequencies=[w["frequency"]], m_unit=w["m_unit"])
        cfg = os.path.join(tmp, "c.toml")
        write_config(cfg, case, dump, grid, tmp)
        with open(cfg) as f:
            text = f.read().replace("nlevels = 3", f"nlevels = {w['nlevels']}")
        with open(cfg, "w") as f:
            f.write(text)
        pfile = os.path.join(tmp, "pix.bin")
        pix.tofile(pfile)
        out = subprocess.check_output([REF_CPU, cfg, "--pixels", pfile, "--threads", str(ncores), "--inclinations",
                                       ",".join(str(i) for i in w["inclinations"]), "--repeat", str(repeat)])
        passes = [json.loads(l) for l in out.decode().splitlines() if l.strip()]
        return "reference", pix.size * len(w["inclinations"]), [(p["steps"], p["seconds"], p["nplasma"])
                                                                  for p in passes]
    from oracle.oracle import Oracle
    os_ = [Oracle(dump, grid, inclination=i, img_width=w["img"], img_height=w["img"], frequencies=(w["frequency"],),
                  m_unit=w["m_unit"], nlevels=w["nlevels"]) for i in w["inclinations"]]
    passes = []
    for _ in range(repeat):
        st_sum, sec, np_sum = 0, 0.0, 0
        for o in os_:
            _, st, secs = o.render(pix, threads=ncores)
            st_sum += int(st[:, 0].sum())
            np_sum += int(st[:, 1].sum())
            sec += secs
        passes.append((st_sum, sec, np_sum))
    for o in os_:
        o.close()
    return "port", pix.size * len(w["inclinations"]), passes


def _ref_config(tmp, dump, grid, w, inclination):
    from tests.golden.cases import write_config
    case = dict(snapshot="cfg1", inclination=inclination, img_width=w["img"], img_height=w["img"],
                frequencies=[w["frequency"]], m_unit=w["m_unit"])
    cfg = os.path.join(tmp, "c.toml")
    write_config(cfg, case, dump, grid, tmp)
    with open(cfg) as f:
        text = f.read().replace("nlevels = 3", f"nlevels = {w['nlevels']}")
    with open(cfg, "w") as f:
        f.write(text)
    return cfg


def oracle_errors(dump, grid, w, images, stride, threads=0):
    """Errors of the rendered images against the FP64 oracle on a strided pixel sample (the reference's own FP64 CPU
    build, oracle/_ref, or the FP64 C oracle port where that build is absent): per image the sample's total-flux
    error (I relative to I; Q, U, V relative to I) and per-pixel L1 / Linf of I.  images: [W*H, 1, 6] arrays in the
    order of w["inclinations"]."""
    ncores = threads or os.cpu_count()
    pix = np.arange(0, w["img"] * w["img"], stride, dtype=np.int64)
    pix = ((pix + (pix // w["img"]) * 7) % (w["img"] * w["img"])).astype(np.int32)
    out = []
    t0 = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        pfile = os.path.join(tmp, "pix.bin")
        pix.tofile(pfile)
        for incl, res in zip(w["inclinations"], images):
            if os.path.exists(REF_CPU64):
                kind = "reference FP64 CPU build (oracle/_ref)"
                ofile = os.path.join(tmp, "out.bin")
                subprocess.check_output([REF_CPU64, _ref_config(tmp, dump, grid, w, incl), "--pixels", pfile,
                                         "--out", ofile, "--threads", str(ncores)])
                ref = np.fromfile(ofile, dtype=np.float64).reshape(pix.size, 6)
            else:
                from oracle.oracle import Oracle
                kind = "FP64 C oracle port"
                o = Oracle(dump, grid, inclination=incl, img_width=w["img"], img_height=w["img"],
                           frequencies=(w["frequency"],), m_unit=w["m_unit"], nlevels=w["nlevels"])
                ref = o.render(pix, threads=ncores)[0].reshape(pix.size, 6)
                o.close()
            got = np.asarray(res).reshape(-1, 6)[pix]
            I, Ir = got[:, 0], ref[:, 0]
            sI = Ir.sum()
            out.append({"inclination": incl, "flux_I": float(abs(I.sum() - sI) / abs(sI)),
                        "flux_QUV": float(max(abs(got[:, q].sum() - ref[:, q].sum()) for q in (1, 2, 3)) / abs(sI)),
                        "l1_I": float(np.abs(I - Ir).sum() / np.abs(Ir).sum()),
                        "linf_I": float(np.abs(I - Ir).max() / np.abs(Ir).max())})
    return {"sample": f"every {stride}th pixel of each {w['img']}^2 image ({pix.size} pixels), {kind}",
            "images": out, "seconds": time.time() - t0}


def cpu_stride(dump, grid, w, ncores, tmp, seconds_target=10.0):
    """Pixel stride that makes one pass over the three images take about `seconds_target`."""
    _, _, passes = _cpu_passes(dump, grid, w, 1024, ncores, 1, tmp)
    return int(np.clip(1024 * passes[0][1] / seconds_target, 1, 1024))


def cpu_baseline(dump, grid, w, threads=0, repeat=1, stride=None):
    """The reference's own CPU path (its FP32 build, OpenMP over all host threads) -- or the FP64 C oracle port when
    the reference could not be compiled -- on a strided pixel sample of the workload's three images, sized by a short
    calibration run to about 10 s of pixel-loop wall time per pass.
    Returns (ray-steps/s per pass list, cores, kind, description, [(steps, seconds, emitting samples) per pass])."""
    ncores = threads or os.cpu_count()
    with tempfile.TemporaryDirectory() as tmp:
        stride = stride or cpu_stride(dump, grid, w, ncores, tmp)
        kind, npix, passes = _cpu_passes(dump, grid, w, stride, ncores, repeat, tmp)
    desc = (f"{npix} rays per pass (every {stride}th pixel of each {w['img']}^2 image, 3 inclinations), "
            f"{'reference FP32 CPU build (oracle/_ref)' if kind == 'reference' else 'FP64 C oracle port'}, "
            f"{ncores} OpenMP threads, pixel-loop wall time")
    return [p[0] / p[1] for p in passes], ncores, kind, desc, passes


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    dump, grid = snapshot_files()
    K = max(1, args.steps)
    rates, cores, kind, desc, passes = cpu_baseline(dump, grid, WORKLOAD, repeat=args.warmup + K)
    timed = passes[args.warmup:]
    steps = sum(p[0] for p in timed)
    secs = sum(p[1] for p in timed)
    emitting = sum(p[2] for p in timed) / max(steps, 1)
    value = steps / secs
    line = {"metric": "ray-steps/s", "value": value, "unit": "ray-steps/s", "n_gpus": args.gpus, "steps": K,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": "plain GPU path: 192x96x96 base grid, 8^3 blocks, 3 AMR levels (15.6M cells), "
                                   "3 x 512^2 images at 10/60/163 deg, 230 GHz, m_unit 1.2e18",
                       "sample": desc},
            "cpu_baseline": {"value": value, "unit": "ray-steps/s", "cores": cores, "kind": kind, "sample": desc,
                             "emitting_samples_per_step": emitting},
            "e2e": {"value": value, "unit": "ray-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# Batching workload: 128 images over the 64x32x32-base snapshot (3 levels, seed 0), drawn from seed 7.
BATCH = dict(gen=["--seed", "0", "--base", "64", "32", "32", "--nlevels", "3"], nlevels=3, nimages=128, seed=7,
             resolutions=(64, 128, 256, 512), incl=(5.0, 175.0), freq=(86e9, 690e9), m_unit=(1e17, 1e19))


def batch_images(b=BATCH):
    """The seeded image list: resolution uniform over the set, inclination uniform, frequency and m_unit
    log-uniform."""
    rng = np.random.default_rng(b["seed"])
    n = b["nimages"]
    res = rng.choice(b["resolutions"], n)
    inc = rng.uniform(*b["incl"], n)
    fr = np.exp(rng.uniform(np.log(b["freq"][0]), np.log(b["freq"][1]), n))
    mu = np.exp(rng.uniform(np.log(b["m_unit"][0]), np.log(b["m_unit"][1]), n))
    return [dict(img=int(res[k]), inclination=float(inc[k]), frequencies=[float(fr[k])], m_unit=float(mu[k]))
            for k in range(n)]


def run_batch(args):
    if args.batch_images:
        return run_batch_small(args)
    return run_batch_sweep(args)


def run_batch_small(args):
    """A small FP32 batch (the first N images of the sweep, all at 256^2): one graph launch per step, for profiling
    the queue kernel on a case that ncu can capture quickly.  The launch shape is the library's default (not
    autotuned) unless --blocks-per-sm / --period say otherwise."""
    import torch

    import phoenix_b200 as P
    dev = torch.device("cuda", 0)
    dump, grid = generated_snapshot(BATCH["gen"])
    snap = P.Snapshot.load(dump, grid, nlevels=BATCH["nlevels"])
    imgs = [dict(im, img=256) for im in batch_images()[:args.batch_images]]
    stream = torch.cuda.Stream(device=dev)
    b = P.Batch([(snap, P.make_params(precision="fp32", **im)) for im in imgs], blocks_per_sm=args.blocks_per_sm,
                period=args.period)
    ts = []
    for r in range(max(1, args.warmup) + max(1, args.steps)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            b.launch(stream.cuda_stream)
            e1.record(stream)
        stream.synchronize()
        ts.append(e0.elapsed_time(e1))
    steps = sum(b.result(k)[1]["steps"] for k in range(len(imgs)))
    ms = min(ts[max(1, args.warmup):])
    print(json.dumps({"workload": "batch-small", "images": len(imgs), "ms": ms, "ray_steps": steps,
                      "ray_steps_per_s": steps / (ms * 1e-3),
                      "tuning": {k: v for k, v in b.tuning().items()
                                 if k in ("blocks_per_sm", "period", "refill_lanes", "regs", "grid", "block")}}),
          flush=True)
    b.close()
    snap.close()


def run_batch_sweep(args):
    """Config 4: the 128-image sweep rendered one by one with the plain single-image path (FP32) and as one batch
    (FP32, mixed and FP64; autotuned launch shape).  Device-resident inputs, CUDA-event timing, L2 flushed between
    timed repetitions.  Prints one JSON line."""
    import torch

    import phoenix_b200 as P
    dev = torch.device("cuda", 0)
    dump, grid = generated_snapshot(BATCH["gen"])
    snap = P.Snapshot.load(dump, grid, nlevels=BATCH["nlevels"], f64_prims=True)
    imgs = batch_images()
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    K, W = max(1, args.steps), max(1, args.warmup)

    def timed(fn):
        ts = []
        for r in range(W + K):
            with torch.cuda.stream(stream):
                flush.fill_(r & 0xFF)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
            stream.synchronize()
            if r >= W:
                ts.append(e0.elapsed_time(e1))
        return ts

    # plain path, one launch per image
    params = [P.make_params(precision="fp32", **im) for im in imgs]
    jobs = [torch.from_numpy(job_list(P, p, args.order)).to(dev) for p in params]
    outs = [torch.zeros((p.img_width * p.img_height, 1, 6), dtype=torch.float64, device=dev) for p in params]
    ctr = torch.zeros((len(params), P.NUM_COUNTERS), dtype=torch.int64, device=dev)

    def plain():
        ctr.zero_()
        for k, p in enumerate(params):
            j = jobs[k]
            snap.render_async(p, j.data_ptr(), j.numel(), outs[k].data_ptr(), ctr[k].data_ptr(), 0, stream.cuda_stream)

    t_plain = timed(plain)
    steps = int(ctr[:, P.CTR["steps"]].sum())
    rays = sum(p.img_width * p.img_height for p in params)
    line = {"workload": "batch", "metric": "ray-steps/s", "unit": "ray-steps/s", "n_gpus": 1, "steps": K,
            "warmup": W, "data": "synthetic",
            "config": {"snapshot": "64x32x32 base grid, 8^3 blocks, 3 AMR levels, seed 0", "images": len(imgs),
                       "image_seed": BATCH["seed"], "resolutions": list(BATCH["resolutions"]), "rays": rays,
                       "l2": "flushed (256 MB write) before every timed repetition",
                       "plain_pixel_order": args.order},
            "ray_steps": steps}
    ms = min(t_plain)
    line["plain_fp32"] = {"ms": ms, "ray_steps_per_s": steps / (ms * 1e-3), "images_per_s": len(imgs) / (ms * 1e-3),
                          "launches": len(imgs)}
    ref_images = []
    for prec in ("fp64", "fp32", "mixed"):
        items = [(snap, P.make_params(precision=prec, **im)) for im in imgs]
        t0 = time.time()
        b = P.Batch(items, autotune=not args.no_autotune)
        create_s = time.time() - t0
        ts = timed(lambda: b.launch(stream.cuda_stream))
        tune = b.tuning()
        ms = min(ts)
        bsteps = 0
        errs = []
        for k in range(len(items)):
            res, info = b.result(k)
            bsteps += info["steps"]
            if prec == "fp64":
                ref_images.append(res)
            else:
                errs.append(image_errors(res, ref_images[k], items[k][1]))
        line["batch_" + prec] = {"ms": ms, "ray_steps_per_s": bsteps / (ms * 1e-3),
                                 "images_per_s": len(imgs) / (ms * 1e-3), "launches": 2,
                                 "create_s": create_s, "tuning": {k: tune[k] for k in
                                                                  ("blocks_per_sm", "period", "tile_rays", "grid",
                                                                   "regs", "ntiles", "device_bytes")},
                                 "candidates": tune["candidates"], "ray_steps": bsteps}
        if errs:
            fI = np.array([e["flux_I"] for e in errs])
            line["batch_" + prec]["errors_vs_fp64"] = {
                "flux_I_max": float(fI.max()), "flux_I_median": float(np.median(fI)),
                "images_flux_I_over_1e-4": int((fI > 1e-4).sum()),
                "flux_QUV_max": float(max(e["flux_QUV"] for e in errs)),
                "l1_I_max": float(max(e["l1_I"] for e in errs)), "linf_I_max": float(max(e["linf_I"] for e in errs))}
        b.close()
    pl = line["plain_fp32"]["ray_steps_per_s"]
    line["speedup_vs_plain_fp32"] = {p: line["batch_" + p]["ray_steps_per_s"] / pl for p in ("fp32", "mixed", "fp64")}
    snap.close()
    print(json.dumps(line), flush=True)


# Serving workload: 4 resident snapshots (seeds 0-3, base grids 96x48x48 .. 256x128x128, 2-4 AMR levels, FP32
# fields) and seeded Poisson request streams.
SERVE = dict(
    snapshots=[["--seed", "0", "--base", "96", "48", "48", "--nlevels", "2", "--nws", "0"],
               ["--seed", "1", "--base", "128", "64", "64", "--nlevels", "3", "--nws", "0"],
               ["--seed", "2", "--base", "192", "96", "96", "--nlevels", "3", "--nws", "0", "--refine", "3.5", "25",
                "0.55"],
               ["--seed", "3", "--base", "256", "128", "128", "--nlevels", "4", "--nws", "0", "--refine", "3.5", "15",
                "0.4"]],
    nlevels=[2, 3, 3, 4], seed=11, resolutions=(64, 128, 256, 512, 1024), freq=(86e9, 345e9), nfreq=(1, 4),
    incl=(5.0, 175.0), m_unit=(1e17, 1e19), rates=(1, 2, 10, 50, 100, 200), requests=48, budget=150 << 30)


def serve_requests(n, seed, cfg=SERVE):
    """Seeded request list: snapshot, resolution, 1-4 frequencies, inclination, m_unit."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nf = int(rng.integers(cfg["nfreq"][0], cfg["nfreq"][1] + 1))
        fr = np.sort(np.exp(rng.uniform(np.log(cfg["freq"][0]), np.log(cfg["freq"][1]), nf)))
        out.append(dict(snapshot=int(rng.integers(0, len(cfg["snapshots"]))),
                        img=int(rng.choice(cfg["resolutions"])), frequencies=[float(f) for f in fr],
                        inclination=float(rng.uniform(*cfg["incl"])),
                        m_unit=float(np.exp(rng.uniform(np.log(cfg["m_unit"][0]), np.log(cfg["m_unit"][1]))))))
    return out


def run_serve(args):
    """Config 5: Poisson request streams at several rates through the continuous-batching server; p50/p99 latency
    (submission to result in host memory), throughput, and latency over the same request's isolated latency (the
    request alone on the server).  Prints one JSON line."""
    import threading

    import phoenix_b200 as P
    snaps = []
    t0 = time.time()
    for g, nl in zip(SERVE["snapshots"], SERVE["nlevels"]):
        dump, grid = generated_snapshot(g)
        snaps.append(P.Snapshot.load(dump, grid, nlevels=nl))
    setup_s = time.time() - t0
    reqs = serve_requests(args.requests or SERVE["requests"], SERVE["seed"])
    params = [P.make_params(precision="fp32", img=r["img"], frequencies=r["frequencies"],
                            inclination=r["inclination"], m_unit=r["m_unit"]) for r in reqs]
    line = {"workload": "serve", "metric": "latency p50/p99 and rays/s", "n_gpus": 1, "data": "synthetic",
            "config": {"snapshots": [" ".join(g) for g in SERVE["snapshots"]],
                       "snapshot_bytes": [s.nbytes() for s in snaps], "requests": len(reqs),
                       "request_seed": SERVE["seed"], "resolutions": list(SERVE["resolutions"]),
                       "precision": "fp32", "budget_bytes": SERVE["budget"]},
            "setup_s": setup_s}
    # the same requests rendered one after another by the plain single-image path (device buffers, CUDA events)
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    pj = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    outs = [torch.zeros((p.img_width * p.img_height, p.nfreqs, 6), dtype=torch.float64, device=dev) for p in params]
    ctr = torch.zeros((len(params), P.NUM_COUNTERS), dtype=torch.int64, device=dev)
    for p in params:
        key = (p.img_width, P.default_pixel_order(p) if args.order == "auto" else args.order)
        if key not in pj:
            pj[key] = torch.from_numpy(job_list(P, p, args.order)).to(dev)
    for rep in range(2):  # the first pass warms up
        ctr.zero_()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k, (r, p) in enumerate(zip(reqs, params)):
                j = pj[(p.img_width, P.default_pixel_order(p) if args.order == "auto" else args.order)]
                snaps[r["snapshot"]].render_async(p, j.data_ptr(), j.numel(), outs[k].data_ptr(), ctr[k].data_ptr(), 0,
                                                  stream.cuda_stream)
            e1.record(stream)
        stream.synchronize()
    plain_s = e0.elapsed_time(e1) * 1e-3
    plain_steps = int(ctr[:, P.CTR["steps"]].sum())
    nrays = sum(p.img_width * p.img_height for p in params)
    line["plain_one_by_one"] = {"seconds": plain_s, "rays_per_s": nrays / plain_s, "ray_steps_per_s": plain_steps / plain_s}
    del outs
    with P.Server(snaps, "fp32", memory_budget=SERVE["budget"]) as srv:
        # isolated latency of every request (alone on the server), after one warm-up request
        w = srv.submit(0, params[0])
        srv.wait(w)
        srv.result(w)
        iso = []
        for r, p in zip(reqs, params):
            rid = srv.submit(r["snapshot"], p)
            srv.wait(rid)
            iso.append(srv.result(rid)[1]["done_s"])
        iso = np.array(iso)
        rays = np.array([p.img_width * p.img_height for p in params], dtype=np.float64)
        line["isolated"] = {"total_s": float(iso.sum()), "p50_s": float(np.median(iso)),
                            "p99_s": float(np.percentile(iso, 99)), "rays_per_s": float(rays.sum() / iso.sum())}
        runs = []
        for rate in (args.rates or SERVE["rates"]):
            rng = np.random.default_rng(SERVE["seed"] + int(rate))
            arrivals = np.cumsum(rng.exponential(1.0 / rate, len(reqs)))
            ids = [None] * len(reqs)
            start = time.perf_counter()

            def submitter():
                for k, (r, p) in enumerate(zip(reqs, params)):
                    delay = arrivals[k] - (time.perf_counter() - start)
                    if delay > 0:
                        time.sleep(delay)
                    ids[k] = srv.submit(r["snapshot"], p)

            th = threading.Thread(target=submitter)
            th.start()
            th.join()
            lat, steps, sub = [], 0, []
            for rid in ids:
                srv.wait(rid)
                _, t = srv.result(rid)
                lat.append(t["done_s"])
                sub.append(t["submitted_s"])
                steps += t["steps"]
            span = time.perf_counter() - start
            lat = np.array(lat)
            ratio = lat / iso
            # requests whose time on the server overlapped another's, against those that had it to themselves
            t0s, t1s = np.array(sub), np.array(sub) + lat
            shared = np.array([((t0s < t1s[k]) & (t1s > t0s[k])).sum() > 1 for k in range(len(lat))])
            alone_r, shared_r = ratio[~shared], ratio[shared]
            runs.append({"rate_per_s": rate, "offered_rays_per_s": float(rays.sum() / arrivals[-1]),
                         "makespan_s": span, "rays_per_s": float(rays.sum() / span),
                         "ray_steps_per_s": steps / span, "requests_per_s": len(reqs) / span,
                         "p50_s": float(np.median(lat)), "p99_s": float(np.percentile(lat, 99)),
                         "ratio_to_isolated_p50": float(np.median(ratio)),
                         "ratio_to_isolated_p99": float(np.percentile(ratio, 99)),
                         "requests_overlapping_another": int(shared.sum()),
                         "ratio_p99_not_overlapping": float(np.percentile(alone_r, 99)) if alone_r.size else None,
                         "ratio_p99_overlapping": float(np.percentile(shared_r, 99)) if shared_r.size else None})
        line["runs"] = runs
        line["server"] = srv.stats()
    for s in snaps:
        s.close()
    print(json.dumps(line), flush=True)


def max_time_sum_work(t_local, work_local, device, world):
    """Whole-job figures of N independent replicas: the slowest rank's time and the work of all ranks (every rank
    takes part in the same two collectives)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(t_local)], dtype=torch.float64, device=device)
    n = torch.tensor([float(work_local)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return float(t.item()), float(n.item())


def run_reference_gpu(args):
    """The reference's own CUDA kernel (src/device/kernel.cu built for sm_100a from its sources, FP32, one frequency
    slot, 128 threads x 3 blocks/SM as its CMake defaults) on the plain-path workload, timed by its own CUDA events
    (device::Info.kernel_s: the kernel launches only, not its per-call model upload)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(REF_GPU):
        print(json.dumps({"impl": "reference_gpu", "unavailable": "oracle/_ref/ref_gpu_fp32 was not built "
                                                                   "(the reference tree is needed to build it)"}))
        return
    from tests.golden.cases import write_config
    w = dict(WORKLOAD)
    w["img"] = args.img
    dump, grid = snapshot_files(w)
    K, W = max(1, args.steps), max(0, args.warmup)
    with tempfile.TemporaryDirectory() as tmp:
        case = dict(snapshot="cfg1", inclination=w["inclinations"][0], img_width=w["img"], img_height=w["img"],
                    frequencies=[w["frequency"]], m_unit=w["m_unit"])
        cfg = os.path.join(tmp, "c.toml")
        write_config(cfg, case, dump, grid, tmp)
        with open(cfg) as f:
            text = f.read().replace("nlevels = 3", f"nlevels = {w['nlevels']}")
        with open(cfg, "w") as f:
            f.write(text)
        out = subprocess.check_output([REF_GPU, cfg, "--inclinations", ",".join(str(i) for i in w["inclinations"]),
                                       "--repeat", str(W + K)])
    passes = [json.loads(l) for l in out.decode().splitlines() if l.strip().startswith("{")][W:]
    steps = sum(p["steps"] for p in passes)
    secs = sum(p["kernel_s"] for p in passes)
    value = steps / secs
    line = {"metric": "ray-steps/s", "value": value, "unit": "ray-steps/s", "n_gpus": 1, "steps": K, "warmup": W,
            "ms_per_step": 1e3 * secs / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference_gpu",
            "config": {"workload": "plain GPU path: 192x96x96 base grid, 8^3 blocks, 3 AMR levels (15.6M cells), "
                                   f"3 x {w['img']}^2 images at 10/60/163 deg, 230 GHz, m_unit 1.2e18",
                       "kernel": "reference src/device/kernel.cu k_render, FP32, PHX_MAX_FREQS=1, 128 x 3 blocks/SM",
                       "timing": "the reference's own CUDA events around its launches (device::Info.kernel_s)"},
            "regs": passes[-1]["regs"], "local_bytes": passes[-1]["local_bytes"],
            "upload_s_per_step": sum(p["upload_s"] for p in passes) / K,
            "ray_steps_per_step": steps / K}
    print(json.dumps(line), flush=True)


def image_errors(res, ref, params):
    """Per-frequency total-flux error relative to Stokes I, and per-pixel L1 / Linf of I relative to the image's I."""
    import phoenix_b200 as P
    f, g = P.flux(res, params), P.flux(ref, params)
    ferr = np.abs(f - g) / np.abs(g[:, :1])
    I, Iref = res[..., 0], ref[..., 0]
    ok = np.isfinite(I) & np.isfinite(Iref)
    d = np.abs(np.where(ok, I - Iref, 0.0))
    return {"flux_I": float(ferr[:, 0].max()), "flux_QUV": float(ferr[:, 1:].max()),
            "l1_I": float(d.sum() / np.abs(np.where(ok, Iref, 0.0)).sum()),
            "linf_I": float(d.max() / np.abs(np.where(ok, Iref, 0.0)).max())}


# Mixed-precision workload: the plain-path generator at seed 1, 1024^2 and 2048^2 images, three frequencies, m_unit 1e19
# (optically and Faraday thick regions).
MIXED = dict(seed=1, images=(1024, 2048), frequencies=(86e9, 230e9, 345e9), m_unit=1e19, inclination=60.0)


def run_mixed(args):
    """Config 3: FP32, mixed and FP64 renders of the same images; per-image flux and per-pixel errors of FP32 and mixed
    against the FP64 path (itself pinned to the FP64 oracle on the parity cases), and device times.  Prints one line."""
    import torch

    import phoenix_b200 as P
    w = dict(WORKLOAD)
    w["seed"] = MIXED["seed"]
    dump, grid = snapshot_files(w)
    snap = P.Snapshot.load(dump, grid, nlevels=w["nlevels"], f64_prims=True)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {"workload": "mixed", "config": {"snapshot": "192x96x96 base grid, 8^3 blocks, 3 AMR levels, seed 1",
                                           "frequencies": list(MIXED["frequencies"]), "m_unit": MIXED["m_unit"],
                                           "inclination": MIXED["inclination"]}, "images": []}
    for side in MIXED["images"]:
        npix = side * side
        nf = len(MIXED["frequencies"])
        row = {"image": side}
        results = {}
        for prec in ("fp64", "fp32", "mixed"):
            p = P.make_params(precision=prec, img=side, frequencies=list(MIXED["frequencies"]),
                              m_unit=MIXED["m_unit"], inclination=MIXED["inclination"])
            jobs = torch.from_numpy(job_list(P, p, args.order)).to(dev)
            res = torch.zeros((npix, nf, 6), dtype=torch.float64, device=dev)
            ctr = torch.zeros(P.NUM_COUNTERS, dtype=torch.int64, device=dev)
            best = None
            for r in range(2):
                with torch.cuda.stream(stream):
                    flush.fill_(r)
                    ctr.zero_()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    snap.render_async(p, jobs.data_ptr(), npix, res.data_ptr(), ctr.data_ptr(), 0, stream.cuda_stream)
                    e1.record(stream)
                stream.synchronize()
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            steps = int(ctr[P.CTR["steps"]])
            row[prec] = {"ms": best, "ray_steps_per_s": steps / (best * 1e-3),
                         "fp64_steps": int(ctr[P.CTR["fp64_steps"]]), "fp64_ops": int(ctr[P.CTR["fp64_ops"]])}
            # FreqOut index (i * H + j) * F + f: the device buffer is in pixel order already
            results[prec] = (res.cpu().numpy().reshape(side, side, nf, 6), p)
        ref = results["fp64"][0]
        for prec in ("fp32", "mixed"):
            row[prec]["errors_vs_fp64"] = image_errors(results[prec][0], ref, results[prec][1])
        row["speed_mixed_vs_fp32"] = row["mixed"]["ray_steps_per_s"] / row["fp32"]["ray_steps_per_s"]
        row["speed_mixed_vs_fp64"] = row["mixed"]["ray_steps_per_s"] / row["fp64"]["ray_steps_per_s"]
        out["images"].append(row)
    snap.close()
    print(json.dumps(out), flush=True)


def run_ingest(args):
    """Snapshot admission: the plain-path workload's dump read and made resident with the host decode (16 OpenMP
    threads on the GPU box) and with the GPU decode (cells decoded on the device while the dump streams in).  The dump
    is read once first so that both runs read it from the page cache.  Prints one JSON line."""
    import phoenix_b200 as P
    dump, grid = snapshot_files(WORKLOAD)
    with open(dump, "rb") as f:
        while f.read(64 << 20):
            pass
    out = {"workload": "ingest", "config": {"dump_bytes": os.path.getsize(dump),
                                            "snapshot": "192x96x96 base grid, 8^3 blocks, 3 AMR levels (15.6M cells)"}}
    for gpu in (False, True, False, True):
        t0 = time.perf_counter()
        s = P.Snapshot.load(dump, grid, nlevels=WORKLOAD["nlevels"], gpu_decode=gpu)
        wall = time.perf_counter() - t0
        i = s.info()
        s.close()
        out["gpu_decode" if gpu else "host_decode"] = {"wall_s": wall, "read_s": i["read_s"],
                                                       "decode_s": i["decode_s"], "upload_s": i["upload_s"],
                                                       "cells_per_s": i["nleafs"] * i["cells"] / wall}
    out["host_threads"] = os.cpu_count()
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference_gpu"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "mixed"])
    ap.add_argument("--img", type=int, default=WORKLOAD["img"], help="image side (profiling runs use smaller)")
    ap.add_argument("--period", type=int, default=0)
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="register-cap variant (0: the mode's default)")
    ap.add_argument("--order", default="auto", choices=["auto", "morton", "16x2", "32x1", "4x8", "2x16", "center4x8"],
                    help="pixel order of the plain path's job lists: the library's per-image default "
                         "(phx_default_pixel_order) or a named tile order (phx_schedule_tiles)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="plain", choices=["plain", "batch", "serve", "ingest", "mixed"],
                    help="plain: the headline single-image path (default); batch: the 128-image sweep; "
                         "serve: Poisson request streams through the server")
    ap.add_argument("--requests", type=int, default=0, help="serve: requests per stream")
    ap.add_argument("--rates", type=float, nargs="*", default=None, help="serve: arrival rates [1/s]")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--batch-images", type=int, default=0, help="batch: a small 256^2 batch of this many images")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.impl == "reference_gpu":
        return run_reference_gpu(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "ingest":
        return run_ingest(args)
    if args.workload == "mixed":
        return run_mixed(args)

    import torch
    import torch.distributed as dist

    import phoenix_b200 as P

    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    w = dict(WORKLOAD)
    w["img"] = args.img

    if rank == 0:
        dump, grid = snapshot_files(w)
    if world > 1:
        dist.barrier()
    dump, grid = snapshot_files(w)
    t0 = time.time()
    snap = P.Snapshot.load(dump, grid, nlevels=w["nlevels"])
    log(f"[rank {rank}] snapshot resident: {snap.nbytes() / 1e9:.3f} GB in {time.time() - t0:.1f} s")

    stream = torch.cuda.Stream(device=dev)
    params = [P.make_params(inclination=i, precision=args.precision, period=args.period,
                            blocks_per_sm=args.blocks_per_sm, **render_kwargs(w)) for i in w["inclinations"]]
    npix = w["img"] * w["img"]
    jobs = [torch.from_numpy(job_list(P, p, args.order)).to(dev) for p in params]
    res = [torch.zeros((npix, 1, 6), dtype=torch.float64, device=dev) for _ in params]
    ctr = torch.zeros((len(params), P.NUM_COUNTERS), dtype=torch.int64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def one_step():
        ctr.zero_()
        for k, p in enumerate(params):
            snap.render_async(p, jobs[k].data_ptr(), npix, res[k].data_ptr(), ctr[k].data_ptr(), 0, stream.cuda_stream)

    # the FP32 roofline's denominator, measured on this GPU before the timed region
    fp32_peak = P.measure_fp32_peak() if rank == 0 else 0.0
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one_step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in params]
           for _ in range(args.steps)]
    steps_total = 0
    nplasma_total = 0
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(s & 0xFF)  # L2 flush, outside the timed region
                ev[s][0].record(stream)
                ctr.zero_()
                for k, p in enumerate(params):
                    kev[s][k][0].record(stream)
                    snap.render_async(p, jobs[k].data_ptr(), npix, res[k].data_ptr(), ctr[k].data_ptr(), 0,
                                      stream.cuda_stream)
                    kev[s][k][1].record(stream)
                ev[s][1].record(stream)
            stream.synchronize()
            c = ctr.cpu().numpy()
            steps_per_launch = [int(v) for v in c[:, P.CTR["steps"]]]
            steps_total += int(c[:, P.CTR["steps"]].sum())
            nplasma_total += int(c[:, P.CTR["nplasma"]].sum())
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    kms = [a.elapsed_time(b) for row in kev for a, b in row]
    ms_max, steps_all = max_time_sum_work(ms, steps_total, dev, world)
    value = steps_all / (ms_max * 1e-3)

    # end to end through the public API: pinned host job list in, host FreqOut image out, every step
    e2e = None
    if not args.no_e2e:
        jobs_h = [torch.from_numpy(job_list(P, p, args.order)).pin_memory() for p in params]
        outs = [torch.zeros((w["img"], w["img"], 1, 6), dtype=torch.float64).pin_memory() for _ in params]
        for k, p in enumerate(params):
            snap.render(p, jobs=jobs_h[k].numpy(), out=outs[k].numpy())
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e_steps = 0
        t1 = time.perf_counter()
        for _ in range(args.steps):
            for k, p in enumerate(params):
                _, info = snap.render(p, jobs=jobs_h[k].numpy(), out=outs[k].numpy())
                e_steps += info["steps"]
        e_s = time.perf_counter() - t1
        te_max, ne_all = max_time_sum_work(e_s, e_steps, dev, world)
        e2e = {"value": ne_all / te_max, "unit": "ray-steps/s",
               "h2d_bytes_per_step": len(params) * npix * 4,
               "d2h_bytes_per_step": len(params) * (npix * 48 + P.NUM_COUNTERS * 8)}

    if rank == 0:
        nimg = len(params) * args.steps
        nfreq = 1
        nlaunch = len(kms)
        kavg_s = sum(kms) / nlaunch * 1e-3
        flops = FLOPS["step"] * steps_total + (FLOPS["sample"] + nfreq * FLOPS["freq"]) * nplasma_total
        fp32_achieved = flops / nlaunch / kavg_s / 1e12
        rays = nimg * npix
        nbytes = (BYTES["sample"] * nplasma_total + BYTES["step"] * steps_total +
                  (BYTES["ray"] + nfreq * BYTES["ray_freq"]) * rays)
        hbm_achieved = nbytes / nlaunch / kavg_s / 1e9
        hbm_peak, peak_kind = measured_peaks()
        traffic = None if DRAM_BYTES_PER_STEP is None else DRAM_BYTES_PER_STEP * steps_total / nlaunch
        line = {
            "metric": "ray-steps/s", "value": value, "unit": "ray-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else args.precision,
            "data": "synthetic",
            "config": {"workload": "plain GPU path: 192x96x96 base grid, 8^3 blocks, 3 AMR levels (15.6M cells, FP32 "
                                   f"primitives), 3 x {w['img']}^2 images at 10/60/163 deg, 230 GHz, m_unit 1.2e18",
                       "precision": args.precision, "images_per_step": len(params), "rays_per_step": len(params) * npix,
                       "l2": "flushed (256 MB write) before every timed step; snapshot 0.5 GB > L2",
                       "parallelism": f"{world} GPU(s), independent replicas",
                       "pixel_order": order_desc(P, params, args.order),
                       "refill": ("whole warp (a warp takes new jobs when all its rays have ended)"
                                  + (f", or its finished lanes every {args.period} passes" if args.period > 0 else ""))},
            "images_per_s": nimg / (ms_max * 1e-3) * world,
            "rays_per_s": nimg * npix / (ms_max * 1e-3) * world,
            "ray_steps_per_step": steps_total / args.steps,
            "ray_steps_per_launch": steps_per_launch,
            "emitting_samples_per_step": nplasma_total / max(steps_total, 1),
            "gpu_launches": nlaunch,
            "roofline": {"bound": "fp32", "achieved": fp32_achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": fp32_achieved / fp32_peak, "traffic": traffic, "kernel": "k_march",
                         "launch_ms": kavg_s * 1e3, "flops_per_launch": flops / nlaunch,
                         "flops_per_unit": FLOPS,
                         "fma_pipe_active": FMA_PIPE_ACTIVE if args.precision == "fp32" else None,
                         "note": "the march is bound by FP32 instruction issue: algorithmic FP32 flops per launch "
                                 "(per ray-step, per emitting sample, per sample-frequency, counted in the reference's "
                                 "own FP32 code) over the CUDA-event launch time; peak = FP32 FMA issue rate measured on this GPU in this run "
                                 "(phx_measure_fp32_peak); traffic = DRAM bytes per launch; fma_pipe_active = the "
                                 "FMA-pipe share of cycles from ncu on this workload (FP32 path only; the mixed and "
                                 "FP64 paths run their geodesic in FP64, so the same FP32-flop count over their "
                                 "time is a lower share)"},
            "roofline_hbm": {"bound": "hbm", "achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s",
                             "frac": hbm_achieved / hbm_peak, "traffic": traffic,
                             "algorithmic_bytes_per_launch": nbytes / nlaunch,
                             "note": f"secondary roofline ({peak_kind} HBM copy peak): the bytes the march requests "
                                     "(256 B gather per emitting sample, 28 B leaf lookup per step, 52 B per ray) per "
                                     "launch over the CUDA-event launch time; most hit L1/L2, traffic is the DRAM "
                                     "share"},
            "clocks": clocks,
            "e2e": e2e,
        }
        if world == 1 and not args.no_cpu:
            rates, cores, kind, desc, cpass = cpu_baseline(dump, grid, w)
            line["cpu_baseline"] = {"value": rates[0], "unit": "ray-steps/s", "cores": cores, "kind": kind,
                                    "sample": desc, "emitting_samples_per_step": cpass[0][2] / max(cpass[0][0], 1)}
            line["oracle_errors"] = oracle_errors(dump, grid, w, [r.cpu().numpy() for r in res], stride=10)
        print(json.dumps(line), flush=True)
    snap.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
