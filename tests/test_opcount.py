"""The algorithmic flop constants of bench.py against a fresh count in the reference's own FP32 code (CPU).

oracle/opcount/count_flops.py counts the reference's per-pixel operations with an op-counting scalar; bench.py froze
the constants fitted on the plain workload.  Here the count runs on the config-1 snapshot (fast): the per-step figure
must agree with the frozen one, and the linear model must explain the per-pixel totals."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from oracle import build_ref
from tests.conftest import ROOT


@pytest.mark.skipif(not os.path.isdir(os.path.join(build_ref.default_src(), "src")),
                    reason="the reference tree is not on this machine")
def test_counted_flops_match_frozen_constants(built):
    import bench
    out = subprocess.check_output([sys.executable, os.path.join(ROOT, "oracle", "opcount", "count_flops.py"),
                                   "--workload", "cfg1", "--stride", "23"], text=True)
    d = json.loads(out.strip().splitlines()[-1])
    assert d["fit_residual_l1"] < 0.01, d
    assert abs(d["F_step"] - bench.FLOPS["step"]) <= 0.03 * bench.FLOPS["step"], d
    assert 0.5 * bench.FLOPS["freq"] <= d["F_freq"] <= 1.5 * bench.FLOPS["freq"], d
    assert d["ops_per_step"]["mul"] > d["ops_per_step"]["add"] > 0
