"""Batches: many images in one graph-captured launch of the queue kernel (needs a GPU).

Every item of a batch must meet the same bars against the FP64 oracle as a single-image render of the same
parameters (tests/test_gpu_parity.py), a ray's result must not depend on which other images share its launch, and
replaying the captured launch must reproduce its results bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

import phoenix_b200 as P
from tests.golden.cases import CASES, case_params
from tests.test_gpu_parity import TOL, flux_errors

pytestmark = pytest.mark.gpu


def _item(snaps, name, precision, **over):
    kw = case_params(name)
    kw.update(over)
    return (snaps[CASES[name]["snapshot"]], P.make_params(precision=precision, **kw))


@pytest.mark.parametrize("precision", ["fp32", "fp64", "mixed"])
def test_batch_items_match_oracle(gpu_snapshots, oracle_results, precision):
    names = ["thick", "cfg1", "edge"]  # two snapshots, three resolutions, one and three frequencies
    items = [_item(gpu_snapshots, n, precision) for n in names]
    with P.Batch(items) as b:
        b.run()
        for k, name in enumerate(names):
            ref, st_ref, _ = oracle_results(name)
            res, info = b.result(k)
            p = items[k][1]
            err = flux_errors(res, ref, p)
            l1 = np.abs(res[..., :4] - ref[..., :4]).sum() / np.abs(ref[..., :4]).sum()
            t = TOL[precision]
            if precision == "fp64":
                assert err.max() <= t["flux"], (name, err)
            else:
                assert err[:, 0].max() <= t["flux"], (name, err)
                assert err[:, 1:].max() <= t["pol"], (name, err)
            assert l1 <= t["l1"], (name, l1)
            assert np.isfinite(res).all()
            assert abs(info["steps"] - int(st_ref[..., 0].sum())) <= 0.002 * st_ref[..., 0].sum(), name


def test_result_independent_of_the_refill_policy(gpu_snapshots):
    """Claiming slots for finished lanes every few passes, once a part of the warp has finished, or only when the whole
    warp has: the same images bit for bit (only which lanes run which rays, and when, changes)."""
    items = [_item(gpu_snapshots, n, "fp32") for n in ("thick", "cfg1", "edge")]
    out = []
    for period, refill in ((16, 1), (1 << 20, 24), (1 << 20, 32), (0, 0)):
        with P.Batch(items, blocks_per_sm=4, period=period, refill_lanes=refill) as b:
            b.run()
            out.append([b.result(k)[0] for k in range(len(items))])
            if (period, refill) == (0, 0):
                t = b.tuning()
                assert (t["period"], t["refill_lanes"]) == (1 << 20, 32)
    for other in out[1:]:
        for a, c in zip(out[0], other):
            assert np.array_equal(a, c)
    with pytest.raises(P.PhxError, match="refill_lanes"):
        P.Batch(items, refill_lanes=33)


def test_result_independent_of_the_mix(gpu_snapshots):
    """An image rendered alone and in a batch with other images (other snapshots, cameras, sizes) is bit-identical:
    a ray's arithmetic does not depend on its lane, warp or the rays around it."""
    opts = dict(blocks_per_sm=3, period=32)
    alone_item = _item(gpu_snapshots, "cfg1", "fp32")
    with P.Batch([alone_item], **opts) as b:
        b.run()
        alone, _ = b.result(0)
    mix = [_item(gpu_snapshots, "edge", "fp32"), _item(gpu_snapshots, "cfg1", "fp32", inclination=75.0, img_width=48,
                                                         img_height=40),
           alone_item, _item(gpu_snapshots, "edge", "fp32", m_unit=1e19)]
    with P.Batch(mix, tile_rays=64, **opts) as b:
        b.run()
        mixed, info = b.result(2)
        again_first, _ = b.result(0)
        b.run()
        again, _ = b.result(2)
        second_first, _ = b.result(0)
    assert np.array_equal(alone, mixed)
    assert np.array_equal(mixed, again) and np.array_equal(again_first, second_first)
    assert info["steps"] > 0


def test_batch_against_single_render_and_job_subsets(gpu_snapshots):
    """Job subsets: pixels outside an item's job list stay zero; pixels in it equal the full batch's."""
    full_item = _item(gpu_snapshots, "edge", "fp64")
    p = full_item[1]
    jobs = np.array([0, 7, p.img_width * p.img_height - 1, 33], dtype=np.int32)
    with P.Batch([full_item, (full_item[0], p, jobs)]) as b:
        b.run()
        full, _ = b.result(0)
        part, info = b.result(1)
    flat_f, flat_p = full.reshape(-1, p.nfreqs, 6), part.reshape(-1, p.nfreqs, 6)
    mask = np.zeros(flat_f.shape[0], bool)
    mask[jobs] = True
    assert np.array_equal(flat_p[mask], flat_f[mask])
    assert np.all(flat_p[~mask] == 0.0)
    single, _ = gpu_snapshots["small"].render(p)
    assert np.abs(full - single).max() <= 1e-9 * np.abs(single).max()


def test_autotuner_and_stream_launch(gpu_snapshots):
    import torch
    items = [_item(gpu_snapshots, "cfg1", "fp32", inclination=float(i)) for i in (10, 50, 120, 170)]
    with P.Batch(items, autotune=True, sample_stride=4) as b:
        t = b.tuning()
        # 3 register caps x 3 refill periods, then the 5 other tile shapes at the best of those
        assert t["ncand"] == 14 and len(t["candidates"]) == 14
        assert sorted(c["tile_shape"] for c in t["candidates"][9:]) == [1, 2, 3, 4, 5]
        best = min(t["candidates"], key=lambda c: c["ms"])
        assert (t["blocks_per_sm"], t["period"], t["tile_shape"]) == (best["blocks_per_sm"], best["period"],
                                                                      best["tile_shape"])
        assert t["nrays"] == 4 * 64 * 64 and t["ntiles"] == 4 * 64 * 64 // 32
        s = torch.cuda.Stream()
        b.launch(s.cuda_stream)
        s.synchronize()
        res0, _ = b.result(0)
        ref, _ = gpu_snapshots["cfg1"].render(items[0][1])
        err = flux_errors(res0, ref, items[0][1])
        assert err.max() <= 1e-4


@pytest.mark.parametrize("precision", ["fp32", "mixed", "fp64"])
def test_ray_setup_kernel_matches_lane_setup(gpu_snapshots, precision):
    """The batch's ray-setup kernel (every job's camera ray at full SIMD width, before the queue kernel) starts the rays
    exactly as a lane that sets up its own ray does: bit-identical images, for every tile shape."""
    items = [_item(gpu_snapshots, n, precision) for n in ("thick", "edge", "cfg1")]
    for shape in (0, 2):
        out = []
        for lane in (False, True):
            with P.Batch(items, blocks_per_sm=0, period=32, tile_shape=shape, lane_setup=lane) as b:
                b.run()
                out.append([b.result(k)[0] for k in range(len(items))])
        for a, c in zip(*out):
            assert np.array_equal(a, c), (precision, shape)


def test_batch_rejects_bad_input(gpu_snapshots):
    a = _item(gpu_snapshots, "cfg1", "fp32")
    b = _item(gpu_snapshots, "cfg1", "fp64")
    with pytest.raises(P.PhxError, match="same precision"):
        P.Batch([a, b])
    many = _item(gpu_snapshots, "cfg1", "mixed", frequencies=[100e9 + 1e9 * k for k in range(6)])
    with pytest.raises(P.PhxError, match="FP32 only"):
        P.Batch([many])
    with pytest.raises(P.PhxError, match="job index"):
        P.Batch([(a[0], a[1], np.array([64 * 64], np.int32))])
