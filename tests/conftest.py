"""Shared fixtures: built native code, generated snapshots (checked against the golden hashes), the FP64 oracle."""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from tests.golden.cases import CASES, SNAPSHOTS, case_params  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    from phoenix_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def golden_meta():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def _sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 20), b""):
            h.update(blk)
    return h.hexdigest()


@pytest.fixture(scope="session")
def snapshots(built, tmp_path_factory, golden_meta):
    """name -> (dump path, grid path, snapshot spec) for every golden snapshot, regenerated byte-identically."""
    out = {}
    base = tmp_path_factory.mktemp("snapshots")
    for name, spec in SNAPSHOTS.items():
        d = base / name
        d.mkdir()
        subprocess.check_call([built["gen"], "--out", str(d)] + spec["gen_args"], stdout=subprocess.DEVNULL)
        dump, grid = str(d / "dump.dat"), str(d / "grid.in")
        assert _sha256(dump) == golden_meta["snapshots"][name]["sha256"], f"generator output changed for {name}"
        out[name] = (dump, grid, spec)
    return out


@pytest.fixture(scope="session")
def oracle_results(snapshots):
    """case -> (res[W,H,F,6], stats[W,H,3], oracle) rendered by the FP64 oracle."""
    from oracle.oracle import Oracle
    cache = {}

    def get(name):
        if name not in cache:
            case = CASES[name]
            dump, grid, spec = snapshots[case["snapshot"]]
            kw = case_params(name)
            kw = {("phi_cam" if k == "phi" else k): v for k, v in kw.items()}
            o = Oracle(dump, grid, nlevels=spec["nlevels"], sfc=1 if spec["sfc"] else 0, **kw)
            res, st, _ = o.render()
            W, H, F = o.width, o.height, o.nfreqs
            cache[name] = (res.reshape(W, H, F, 6), st.reshape(W, H, 3), o)
        return cache[name]

    return get


def golden_arrays(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.fixture(scope="module")
def gpu_snapshots(snapshots):
    """The parity snapshots resident on the GPU (FP32 and FP64 primitives)."""
    import phoenix_b200 as P
    out = {}
    for name, (dump, grid, spec) in snapshots.items():
        out[name] = P.Snapshot.load(dump, grid, nlevels=spec["nlevels"], sfc=spec["sfc"], f64_prims=True)
    yield out
    for s in out.values():
        s.close()
