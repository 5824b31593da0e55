"""Per-frequency image totals reduced on the device (phx_spectrum_async, phx_batch_spectrum) against the host
reduction of the reference's output code (host/io/output.hpp:43-74, restated by phoenix_b200.flux and the
spectrum-file means), including pixels with non-finite values, which both skip (needs a GPU)."""
from __future__ import annotations

import numpy as np
import pytest

import phoenix_b200 as P
from tests.golden.cases import CASES, case_params

pytestmark = pytest.mark.gpu


def host_spectrum(res, p):
    """(I, Q, U, V [Jy], mean tau, mean tauF) per frequency, as the reference's compute_spec / compute_tau."""
    r = res.reshape(-1, p.nfreqs, 6)
    flux = P.flux(res, p)
    rows = []
    for f in range(p.nfreqs):
        ok = np.isfinite(r[:, f, :6].sum(axis=-1))
        tau = r[ok, f, 4].mean() if ok.any() else 0.0
        tauF = r[ok, f, 5].mean() if ok.any() else 0.0
        rows.append(list(flux[f]) + [tau, tauF])
    return np.array(rows)


@pytest.mark.parametrize("W,H,F", [(64, 64, 1), (37, 53, 3), (1, 1, 2), (300, 200, 4)])
def test_device_spectrum_matches_host(W, H, F):
    import torch
    rng = np.random.default_rng(W * H + F)
    res = rng.standard_normal((W, H, F, 6))
    res[..., :4] *= 1e-15
    res[..., 4:] = np.abs(res[..., 4:])
    if W * H > 4:
        flat = res.reshape(-1, F, 6)
        flat[1, 0, 2] = np.nan     # skipped by the flux and the means
        flat[3, F - 1, 0] = np.inf
        flat[2, 0, 4] = np.nan     # kept by the flux, skipped by the means
    p = P.make_params(img_width=W, img_height=H, frequencies=[100e9 * (f + 1) for f in range(F)])
    d_res = torch.from_numpy(res).cuda()
    d_spec = torch.zeros((F, 8), dtype=torch.float64, device="cuda")  # PhxSpectrum: 6 doubles + 2 int64
    P.device_spectrum(p, d_res.data_ptr(), d_spec.data_ptr())
    torch.cuda.synchronize()
    spec = d_spec.cpu().numpy()
    want = host_spectrum(res, p)
    np.testing.assert_allclose(spec[:, :6], want, rtol=1e-12, atol=0)
    counts = d_spec.cpu().view(torch.int64).numpy()[:, 6:]
    r = res.reshape(-1, F, 6)
    for f in range(F):
        assert counts[f, 0] == np.isfinite(r[:, f, :4].sum(-1)).sum()
        assert counts[f, 1] == np.isfinite(r[:, f, :6].sum(-1)).sum()


def test_batch_spectrum_matches_downloaded_image(gpu_snapshots):
    items = []
    for name in ("thick", "cfg1", "edge"):
        items.append((gpu_snapshots[CASES[name]["snapshot"]], P.make_params(precision="fp32", **case_params(name))))
    with P.Batch(items) as b:
        b.run()
        for k, (_, p) in enumerate(items):
            res, _ = b.result(k)
            np.testing.assert_allclose(b.spectrum(k), host_spectrum(res, p), rtol=1e-12, atol=0)
