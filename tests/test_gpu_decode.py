"""GPU decode of a BHAC dump (needs a GPU): the cells decoded on the device, while the dump streams in, equal the host
reader's decode, and renders of both snapshots agree."""
from __future__ import annotations

import numpy as np
import pytest

import phoenix_b200 as P
from tests.golden.cases import case_params

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cfg1", "small"])
def test_gpu_decode_matches_host_decode(snapshots, name):
    dump, grid, spec = snapshots[name]
    kw = dict(nlevels=spec["nlevels"], sfc=spec["sfc"], f64_prims=True)
    with P.Snapshot.load(dump, grid, **kw) as host, P.Snapshot.load(dump, grid, gpu_decode=True, **kw) as dev:
        hi, di = host.info(), dev.info()
        assert di["gpu_decoded"] == 1 and hi["gpu_decoded"] == 0
        for k in ("nleafs", "cells", "nlevels", "nx", "ng", "a", "hslope", "gam", "bytes"):
            assert hi[k] == di[k], k
        hf, hd = host.download(f64=True)
        df, dd = dev.download(f64=True)
        # the same FP64 routine on both sides; only the contraction of multiply-adds may differ.  Differences are
        # measured against each variable's scale over the snapshot: the internal energy and velocities come out of
        # differences of nearly equal terms, where a last-bit change in an input is a larger relative change
        vscale = np.maximum(np.abs(hd).reshape(-1, 8).max(axis=0), 1e-300)  # (a field may be zero everywhere)
        err = (np.abs(dd - hd) / vscale).reshape(-1, 8).max(axis=0)
        assert np.all(err <= 1e-12), err
        ferr = (np.abs(df.astype(np.float64) - hf) / vscale).reshape(-1, 8).max(axis=0)
        assert np.all(ferr <= 2.0 ** -22), ferr
        assert (df != hf).mean() < 1e-2
        p = P.make_params(precision="fp64", **case_params("cfg1" if name == "cfg1" else "edge"))
        a, _ = host.render(p)
        b, _ = dev.render(p)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max()
