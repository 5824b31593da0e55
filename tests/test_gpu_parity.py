"""Parity of the sm_100a raymarch kernels with the FP64 oracle and the reference's golden outputs (needs a GPU).

Tolerances (total flux relative to Stokes I of the same frequency; L1 relative over the image):
  FP64   flux 1e-9, per-pixel L1 1e-8, per-pixel step and plasma-segment counts identical to the reference's
  FP32   flux I <= 1e-4 and Q/U/V <= 1e-3 of I (the path's stated bar), L1 <= 1e-3
  mixed  same bar as FP32
"""
from __future__ import annotations

import numpy as np
import pytest

import phoenix_b200 as P
from tests.conftest import golden_arrays
from tests.golden.cases import CASES, case_params

pytestmark = pytest.mark.gpu

TOL = {"fp64": dict(flux=1e-9, l1=1e-8), "fp32": dict(flux=1e-4, pol=1e-3, l1=1e-3),
       "mixed": dict(flux=1e-4, pol=1e-3, l1=1e-3)}


def render_case(snaps, name, precision, **over):
    kw = case_params(name)
    kw.update(over)
    p = P.make_params(precision=precision, **kw)
    res, info = snaps[CASES[name]["snapshot"]].render(p)
    return res, info, p


def flux_errors(res, ref, p):
    f = P.flux(res, p)
    g = P.flux(ref, p)
    err = np.abs(f - g) / np.abs(g[:, :1])
    return err  # [nfreqs, 4] relative to I


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "fp32", "mixed"])
def test_matches_oracle(gpu_snapshots, oracle_results, name, precision):
    ref, st_ref, _ = oracle_results(name)
    res, info, p = render_case(gpu_snapshots, name, precision)
    assert info["bad"] == 0 or precision != "fp64"
    err = flux_errors(res, ref, p)
    l1 = np.abs(res[..., :4] - ref[..., :4]).sum() / np.abs(ref[..., :4]).sum()
    t = TOL[precision]
    if precision == "fp64":
        assert err.max() <= t["flux"], err
    else:
        assert err[:, 0].max() <= t["flux"], err
        assert err[:, 1:].max() <= t["pol"], err
    assert l1 <= t["l1"], l1
    assert np.isfinite(res).all()
    # the march visits the same samples: exactly with an FP64 geodesic (FP64, mixed), closely in FP32
    if precision == "fp32":
        assert abs(info["steps"] - int(st_ref[..., 0].sum())) <= 0.002 * st_ref[..., 0].sum()
    else:
        assert info["steps"] == int(st_ref[..., 0].sum()) and info["nplasma"] == int(st_ref[..., 1].sum())


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fp64_steps_per_pixel(gpu_snapshots, oracle_results, snapshots, name, precision):
    """FP64 and mixed marches (both with an FP64 geodesic) take the reference's steps and plasma segments pixel by pixel:
    identical to the reference's own FP64 build (golden stats) and to the oracle on every pixel (pixel statistics via
    the async entry point).  The FP64 kernels are compiled without multiply-add contraction, like the reference's CPU
    build."""
    import torch
    ref, st_ref, _ = oracle_results(name)
    kw = case_params(name)
    p = P.make_params(precision=precision, **kw)
    W, H, F = p.img_width, p.img_height, p.nfreqs
    dev = torch.device("cuda")
    jobs = torch.from_numpy(P.schedule_morton(W, H)).to(dev)
    res = torch.zeros((W, H, F, 6), dtype=torch.float64, device=dev)
    ps = torch.zeros((W, H, 3), dtype=torch.int32, device=dev)
    ctr = torch.zeros(P.NUM_COUNTERS, dtype=torch.int64, device=dev)
    snap = gpu_snapshots[CASES[name]["snapshot"]]
    stream = torch.cuda.current_stream()
    snap.render_async(p, jobs.data_ptr(), jobs.numel(), res.data_ptr(), ctr.data_ptr(), ps.data_ptr(),
                      stream.cuda_stream)
    torch.cuda.synchronize()
    st = ps.cpu().numpy()
    golden = golden_arrays(name)["stats_fp64"]
    for ref in (st_ref, golden):
        diff = np.argwhere((st[..., :2] != ref[..., :2]).any(axis=-1))
        assert len(diff) == 0, (precision, len(diff), diff[:8].tolist())
    assert int(ctr[P.CTR["rays"]]) == W * H
    assert int(ctr[P.CTR["steps"]]) == int(st[..., 0].sum())


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_reference_golden(gpu_snapshots, golden_meta, name):
    """Against the reference's own FP64 output (committed fixture)."""
    g = golden_arrays(name)["res_fp64"]
    res, info, p = render_case(gpu_snapshots, name, "fp64")
    assert flux_errors(res, g, p).max() <= 1e-9
    assert info["steps"] == golden_meta["cases"][name]["reference"]["fp64"]["steps"]


def test_job_subset_leaves_other_pixels(gpu_snapshots):
    p = P.make_params(precision="fp32", **case_params("edge"))
    W, H, F = p.img_width, p.img_height, p.nfreqs
    full, _ = gpu_snapshots["small"].render(p)
    sentinel = np.full((W, H, F, 6), -7.0)
    jobs = np.array([0, 5, W * H - 1, 17], dtype=np.int32)
    part, info = gpu_snapshots["small"].render(p, jobs=jobs, out=sentinel.copy())
    flat_full, flat_part = full.reshape(W * H, F, 6), part.reshape(W * H, F, 6)
    mask = np.zeros(W * H, bool)
    mask[jobs] = True
    assert np.array_equal(flat_part[mask], flat_full[mask])
    assert np.all(flat_part[~mask] == -7.0)
    empty, info0 = gpu_snapshots["small"].render(p, jobs=np.zeros(0, np.int32), out=sentinel.copy())
    assert np.all(empty == -7.0) and info0["steps"] == 0


def test_frequencies_are_independent(gpu_snapshots):
    """A three-frequency render equals three single-frequency renders (per-frequency state only)."""
    kw = case_params("thick")
    multi, _ = gpu_snapshots["cfg1"].render(P.make_params(precision="fp64", **kw))
    for f, nu in enumerate(kw["frequencies"]):
        one = dict(kw)
        one["frequencies"] = [nu]
        single, _ = gpu_snapshots["cfg1"].render(P.make_params(precision="fp64", **one))
        scale = np.abs(single).max()
        assert np.abs(multi[:, :, f] - single[:, :, 0]).max() <= 1e-12 * scale


@pytest.mark.parametrize("bps", [0, 1, 4])
def test_results_independent_of_scheduling(gpu_snapshots, bps):
    """A ray's arithmetic does not depend on which lane, warp or refill round runs it: for one compiled variant the
    image is bit-identical whatever the refill period or threshold.  Variants compiled for other register caps round
    differently (separate compilations), so across them the images agree to FP32 rounding."""
    kw = case_params("cfg1")
    base, _ = gpu_snapshots["cfg1"].render(P.make_params(precision="fp32", blocks_per_sm=bps, period=1, **kw))
    for period, refill in ((4, 0), (16, 0), (64, 1), (256, 8), (1 << 20, 24), (1 << 20, 32)):
        other, _ = gpu_snapshots["cfg1"].render(P.make_params(precision="fp32", blocks_per_sm=bps, period=period,
                                                              refill_lanes=refill, **kw))
        assert np.array_equal(base, other), (bps, period, refill)
    default, _ = gpu_snapshots["cfg1"].render(P.make_params(precision="fp32", **kw))
    l1 = np.abs(default[..., :4] - base[..., :4]).sum() / np.abs(base[..., :4]).sum()
    assert l1 <= 1e-5, l1
    with pytest.raises(P.PhxError, match="refill_lanes"):
        gpu_snapshots["cfg1"].render(P.make_params(precision="fp32", refill_lanes=33, **kw))


@pytest.mark.parametrize("bps", [3, 4])
def test_whole_sm_blocks(gpu_snapshots, bps):
    """Register-cap variants 3 and 4 run as one 384 / 512-thread block per SM once the job list gives every SM such a
    block (a 320^2 image: 102,400 rays >= 148 SMs x 512).  That shape is bit-identical across refill periods, agrees
    with the 128-thread shape of the same cap (a small job subset; separate compilations round differently) within
    1e-4 L1, and matches the FP64 render to the FP32 flux bar."""
    kw = case_params("cfg1")
    kw.update(img=320, fov_x=2 * kw["fov_x"], fov_y=2 * kw["fov_y"])
    snap = gpu_snapshots["cfg1"]
    base, info = snap.render(P.make_params(precision="fp32", blocks_per_sm=bps, period=64, **kw))
    assert info["block"] == 128 * bps and info["blocks"] == info["sms"], info
    other, _ = snap.render(P.make_params(precision="fp32", blocks_per_sm=bps, period=4, **kw))
    assert np.array_equal(base, other)
    # 2,048 jobs: too few for whole-SM blocks, so the same pixels run on the 128-thread shape
    jobs = P.schedule_morton(320, 320)[::50].copy()
    small, sinfo = snap.render(P.make_params(precision="fp32", blocks_per_sm=bps, **kw), jobs=jobs)
    assert sinfo["block"] == 128, sinfo
    sel = np.sort(jobs)
    a, b = small.reshape(-1, 6)[sel], base.reshape(-1, 6)[sel]
    assert np.abs(a[:, :4] - b[:, :4]).sum() <= 1e-4 * np.abs(b[:, :4]).sum()
    p64 = P.make_params(precision="fp64", **kw)
    ref, _ = snap.render(p64)
    f, g = P.flux(base, p64), P.flux(ref, p64)
    assert np.abs(f[:, 0] - g[:, 0]).max() <= 1e-4 * np.abs(g[:, 0]).max()
    assert np.abs(f[:, 1:] - g[:, 1:]).max() <= 1e-3 * np.abs(g[:, 0]).max()


def test_invalid_arguments_are_reported(gpu_snapshots):
    p = P.make_params(img=0)
    with pytest.raises(P.PhxError) as e:
        gpu_snapshots["small"].render(p, out=np.zeros((0, 0, 1, 6)))
    assert e.value.code == -1
    p = P.make_params(img=8)
    with pytest.raises(P.PhxError):
        gpu_snapshots["small"].render(p, jobs=np.array([64], np.int32))
