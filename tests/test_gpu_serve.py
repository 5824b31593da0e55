"""The served render loop (needs a GPU): requests merged into one running queue kernel.

Each request must meet the single-image bars against the FP64 oracle, a request's result must be the same alone and
in a mix of concurrent requests (bit for bit: one compiled kernel, and a ray's arithmetic does not depend on its
lane or neighbours), admission must respect the result arena, and the kernel must restart after the server idles.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

import phoenix_b200 as P
from tests.golden.cases import CASES, case_params
from tests.test_gpu_parity import TOL, flux_errors

pytestmark = pytest.mark.gpu

WAIT = 300.0


def _params(name, precision, **over):
    kw = case_params(name)
    kw.update(over)
    return P.make_params(precision=precision, **kw)


@pytest.fixture(scope="module")
def snaps(gpu_snapshots):
    return [gpu_snapshots["cfg1"], gpu_snapshots["small"]]


def _sid(name):
    return 0 if CASES[name]["snapshot"] == "cfg1" else 1


def test_alone_and_in_a_mix(snaps, oracle_results):
    with P.Server(snaps, "fp32") as srv:
        rid = srv.submit(0, _params("cfg1", "fp32"))
        srv.wait(rid, WAIT)
        alone, t_alone = srv.result(rid)
        mix = [("thick", {}), ("cfg1", dict(inclination=120.0)), ("edge", {}), ("cfg1", {}),
               ("edge", dict(m_unit=1e19)), ("cfg1", dict(img_width=48, img_height=40))]
        ids = [srv.submit(_sid(n), _params(n, "fp32", **o)) for n, o in mix]
        out = {}
        for rid, (n, o) in zip(ids, mix):
            srv.wait(rid, WAIT)
            out[(n, tuple(sorted(o.items())))] = srv.result(rid)
        st = srv.stats()
    assert np.array_equal(out[("cfg1", ())][0], alone)
    assert t_alone["rays"] == 64 * 64 and t_alone["steps"] > 0 and t_alone["done_s"] >= t_alone["admitted_s"]
    for name in ("thick", "edge"):
        ref, st_ref, _ = oracle_results(name)
        res, t = out[(name, ())]
        p = _params(name, "fp32")
        err = flux_errors(res, ref, p)
        assert err[:, 0].max() <= TOL["fp32"]["flux"] and err[:, 1:].max() <= TOL["fp32"]["pol"], (name, err)
        assert abs(t["steps"] - int(st_ref[..., 0].sum())) <= 0.002 * st_ref[..., 0].sum()
    assert st["completed"] == 7 and st["inflight"] == 0 and st["pending"] == 0


def test_fp64_server_matches_single_render(snaps):
    p = _params("edge", "fp64")
    with P.Server(snaps, "fp64", max_freqs=1) as srv:
        rid = srv.submit(1, p)
        srv.wait(rid, WAIT)
        res, _ = srv.result(rid)
    single, _ = snaps[1].render(p)
    assert np.abs(res - single).max() <= 1e-9 * np.abs(single).max()


def test_admission_by_arena_and_oversized_request(snaps):
    # room for about four 64x64 one-frequency results (196,608 B each) beside the 64x64 job table
    with P.Server(snaps, "fp32", max_freqs=1, arena_bytes=1 << 20) as srv:
        ids = [srv.submit(0, _params("cfg1", "fp32", inclination=10.0 + 20 * k)) for k in range(8)]
        for rid in ids:
            srv.wait(rid, WAIT)
        results = [srv.result(rid)[0] for rid in ids]
        big = srv.submit(0, _params("cfg1", "fp32", img_width=256, img_height=256))
        with pytest.raises(P.PhxError, match="does not fit"):
            srv.wait(big, WAIT)
        st = srv.stats()
    assert st["completed"] == 8
    assert all(np.isfinite(r).all() and np.abs(r[..., 0]).sum() > 0 for r in results)
    single, _ = snaps[0].render(_params("cfg1", "fp32", inclination=10.0))
    err = flux_errors(results[0], single, _params("cfg1", "fp32"))
    assert err.max() <= 1e-5


def test_kernel_restarts_after_idle(snaps):
    with P.Server(snaps, "fp32", max_freqs=1, linger_ms=5.0) as srv:
        first = srv.submit(1, _params("edge", "fp32"))
        srv.wait(first, WAIT)
        a, _ = srv.result(first)
        time.sleep(0.3)
        second = srv.submit(1, _params("edge", "fp32"))
        srv.wait(second, WAIT)
        b, _ = srv.result(second)
        st = srv.stats()
    assert st["generations"] >= 2
    assert np.array_equal(a, b)


def test_small_request_overtakes_a_large_one(snaps):
    """A small request enters the queue whole, ahead of the rest of a large one that is published a chunk at a time:
    submitted right after the large one, it finishes first, and both results stay the ones each gets alone."""
    big_p = _params("cfg1", "fp32", img_width=256, img_height=256)
    small_p = _params("edge", "fp32")
    with P.Server(snaps, "fp32", max_freqs=1, backlog_rays=4096, publish_chunk=16, small_rays=1024) as srv:
        big = srv.submit(0, big_p)
        small = srv.submit(1, small_p)
        srv.wait(small, WAIT)
        srv.wait(big, WAIT)
        rs, ts = srv.result(small)
        rb, tb = srv.result(big)
        alone = srv.submit(1, small_p)
        srv.wait(alone, WAIT)
        ra, _ = srv.result(alone)
    assert ts["submitted_s"] + ts["done_s"] < tb["submitted_s"] + tb["done_s"]
    assert np.array_equal(rs, ra)
    single, _ = snaps[0].render(big_p)
    assert flux_errors(rb, single, big_p).max() <= 1e-5


def test_idle_limit_exit_then_clean_relaunch(snaps):
    """The queue kernel's idle wait is bounded: with a small idle_limit and a long linger, the kernel gives up on its
    own after the first request (status word set, no request lost), and the next submission relaunches it in a new
    generation with the same result."""
    p = _params("edge", "fp32")
    with P.Server(snaps, "fp32", max_freqs=1, idle_limit=200, idle_ns=1000, linger_ms=600000.0) as srv:
        first = srv.submit(1, p)
        srv.wait(first, WAIT)
        a, _ = srv.result(first)
        t0 = time.time()
        while srv.stats()["idle_exits"] < 1 and time.time() - t0 < 30.0:
            time.sleep(0.01)
        st = srv.stats()
        assert st["idle_exits"] >= 1 and st["inflight"] == 0
        second = srv.submit(1, p)
        srv.wait(second, WAIT)
        b, _ = srv.result(second)
        st = srv.stats()
    assert st["generations"] >= 2 and st["completed"] == 2
    assert np.array_equal(a, b)


def test_requests_survive_kernel_idle_exits(snaps):
    """An idle_limit of a few polls makes the kernel leave whenever the queue runs dry for a moment, also while other
    requests are still in flight (a warp that gives up may hold a claim past the tail).  Requests caught by such an
    exit go back to the queue and are rendered again; every result equals the request rendered alone."""
    ps = [_params("edge", "fp32", inclination=150.0 + 5 * k) for k in range(6)]
    with P.Server(snaps, "fp32", max_freqs=1, idle_limit=2, idle_ns=100, linger_ms=600000.0) as srv:
        ids = []
        for p in ps:
            ids.append(srv.submit(1, p))
            time.sleep(0.002)
        got = []
        for rid in ids:
            srv.wait(rid, WAIT)
            got.append(srv.result(rid)[0])
        st = srv.stats()
    assert st["completed"] == len(ps) and st["idle_exits"] >= 1
    for p, r in zip(ps, got):
        single, _ = snaps[1].render(p)
        assert flux_errors(r, single, p).max() <= 1e-5
