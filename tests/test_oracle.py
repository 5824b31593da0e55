"""The FP64 oracle against the reference's own outputs (golden fixtures) and against independent mathematics."""
from __future__ import annotations

import numpy as np
import pytest
from scipy.special import kve

from oracle import oracle as orc
from tests.conftest import golden_arrays
from tests.golden.cases import CASES


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_reference(name, oracle_results, golden_meta):
    """Same inputs -> same per-pixel steps and segments, tau bit for bit, Stokes within 1e-12 of the largest value
    (the only arithmetic difference is the Bessel-ratio evaluation)."""
    res, st, o = oracle_results(name)
    g = golden_arrays(name)
    assert np.array_equal(st, g["stats_fp64"])
    assert np.array_equal(res[..., 4], g["res_fp64"][..., 4])
    for q in (0, 1, 2, 3, 5):
        scale = np.abs(g["res_fp64"][..., q]).max() or 1.0
        assert np.abs(res[..., q] - g["res_fp64"][..., q]).max() <= 1e-12 * scale
    fl = o.flux(res.reshape(-1, res.shape[2], 6))
    ref = np.array(golden_meta["cases"][name]["reference"]["fp64"]["flux"])[:, 1:]
    assert np.allclose(fl, ref, rtol=1e-12, atol=1e-12 * np.abs(ref[:, :1]))


def test_bessel_ratios_against_scipy():
    for x in np.geomspace(0.2, 500.0, 400):
        r10, r02 = orc.bessel_ratios(float(x))
        k0, k1, k2 = kve(0, x), kve(1, x), kve(2, x)
        assert r10 == pytest.approx(k1 / k2, rel=1e-12)
        assert r02 == pytest.approx(k0 / k2, rel=1e-12 if x < 30 else 1e-9)


def test_metric_inverse():
    import ctypes as C
    rng = np.random.default_rng(1)
    L = orc.lib()
    for _ in range(50):
        X = np.array([0.0, rng.uniform(0.1, 7.0), rng.uniform(0.05, 3.09), rng.uniform(0, 6.28)])
        gd = np.zeros((4, 4))
        gu = np.zeros((4, 4))
        L.orc_metric_dd(0.9375, 0.25, X.ctypes.data, gd.ctypes.data)
        L.orc_metric_uu(0.9375, 0.25, X.ctypes.data, gu.ctypes.data)
        assert np.allclose(gd @ gu, np.eye(4), atol=1e-11)
    del C
