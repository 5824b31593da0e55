"""The allocation-free render entry point (phx_render_noalloc) against the existing asynchronous one.

Callers that cannot call cudaMalloc -- an application whose device memory is all owned by its own pool, or a serving
loop where an allocation would synchronize the device -- use phx_render_noalloc, which keeps its job list and scratch
in a fixed library-owned device array.  This file is collected last on purpose; it creates its own snapshot, so it
passes both alone in a fresh process and after the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import phoenix_b200 as P
from phoenix_b200 import native
from tests.golden.cases import CASES, case_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def snap(snapshots):
    dump, grid, spec = snapshots[CASES["cfg1"]["snapshot"]]
    s = P.Snapshot.load(dump, grid, nlevels=spec["nlevels"], sfc=spec["sfc"])
    yield s
    s.close()


def test_noalloc_matches_async_entry_point(snap):
    import torch
    kw = case_params("cfg1")
    p = P.make_params(precision="fp32", **kw)
    W, H, F = p.img_width, p.img_height, p.nfreqs
    jobs = P.schedule_morton(W, H)
    dev = torch.device("cuda")
    stream = torch.cuda.current_stream()

    # the existing entry point: caller-provided job list and counter block on the device
    res_ref = torch.zeros((W, H, F, 6), dtype=torch.float64, device=dev)
    d_jobs = torch.from_numpy(jobs).to(dev)
    ctr = torch.zeros(P.NUM_COUNTERS, dtype=torch.int64, device=dev)
    snap.render_async(p, d_jobs.data_ptr(), jobs.size, res_ref.data_ptr(), ctr.data_ptr(), 0, stream.cuda_stream)
    torch.cuda.synchronize()
    ref = res_ref.cpu().numpy()
    scale = np.abs(ref[..., :4]).sum()

    L = native.lib()
    for call in range(2):  # two calls in a row share the scratch array
        res = torch.full((W, H, F, 6), float("nan"), dtype=torch.float64, device=dev)
        rc = L.phx_render_noalloc(snap.handle, C.byref(p), jobs.ctypes.data, jobs.size, res.data_ptr(),
                                  stream.cuda_stream)
        assert rc == native.PHX_OK, L.phx_last_error()
        torch.cuda.synchronize()
        got = res.cpu().numpy()
        assert np.isfinite(got).all(), f"call {call}: pixels left unwritten"
        # same kernel and arithmetic: identical, and in any case within the FP32 parity bar (L1 <= 1e-3)
        assert np.abs(got[..., :4] - ref[..., :4]).sum() <= 1e-3 * scale
        assert np.array_equal(got, ref), f"call {call} differs from phx_render_async"


def test_noalloc_rejects_oversized_job_lists(snap):
    p = P.make_params(precision="fp32", img=1025)
    jobs = np.zeros(native.NOALLOC_MAX_JOBS + 1, dtype=np.int32)
    L = native.lib()
    rc = L.phx_render_noalloc(snap.handle, C.byref(p), jobs.ctypes.data, jobs.size, C.c_void_p(1), None)
    assert rc == native.PHX_E_INVALID
    assert b"exceeds the no-allocation limit" in L.phx_last_error()
