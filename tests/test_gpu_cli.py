"""The PHOENIX command line end to end on the GPU: config -> render -> img_data.h5 / image.dat / spectrum.dat and the
per-frequency flux line, against the FP64 oracle."""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

from tests.golden.cases import CASES, write_config
from tests.h5mini import H5File

pytestmark = pytest.mark.gpu

FLUX = re.compile(r"Flux at (\S+) Hz \(Jy\): \S*I\S* (\S+) \S*Q\S* (\S+) \S*U\S* (\S+) \S*V\S* (\S+)")


@pytest.mark.parametrize("precision,gpu_decode", [("fp32", False), ("fp64", False), ("fp32", True)])
def test_cli_end_to_end(built, snapshots, oracle_results, tmp_path, precision, gpu_decode):
    name = "thick"
    case = CASES[name]
    dump, grid, _ = snapshots[case["snapshot"]]
    out = tmp_path / "out"
    cfg = tmp_path / "config.toml"
    write_config(str(cfg), case, dump, grid, str(out))
    env = dict(os.environ, PHX_PRECISION=precision)
    r = subprocess.run([built["cli"], str(cfg), "output.image=both", "output.block_size=8",
                        "grmhd.gpu_decode=" + ("true" if gpu_decode else "false")], capture_output=True,
                       text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = FLUX.findall(re.sub(r"\x1b\[[0-9;]*m", "", r.stderr))
    assert len(lines) == len(case["frequencies"])
    ref, _, o = oracle_results(name)
    W, H, F = ref.shape[:3]
    fref = o.flux(ref.reshape(-1, F, 6))
    for f, (nu, *iquv) in enumerate(lines):
        assert float(nu) == case["frequencies"][f]
        got = np.array([float(v) for v in iquv])
        tol = 1e-9 if precision == "fp64" else 1e-4
        assert np.abs(got - fref[f]).max() <= tol * abs(fref[f][0]) + 1e-9 * abs(fref[f][0])
    h5 = H5File(str(out / "img_data.h5"))
    nu0 = "%e" % case["frequencies"][0]
    img = h5.read("I" + nu0)
    bs = 8
    nbj = H // bs
    b = np.arange((W // bs) * nbj)[:, None]
    q = np.arange(bs * bs)[None, :]
    ii, jj = (b // nbj) * bs + q // bs, (b % nbj) * bs + q % bs
    # the file holds exactly what the library renders for the same parameters
    import phoenix_b200 as P
    from tests.golden.cases import case_params
    with P.Snapshot.load(dump, grid, nlevels=3, f64_prims=precision == "fp64", gpu_decode=gpu_decode) as snap:
        mine, _ = snap.render(P.make_params(precision=precision, **case_params(name)))
    np.testing.assert_array_equal(img, mine[ii, jj, 0, 0] * 1e23)
    assert (out / "image_0.dat").exists() and (out / "image_2.dat").exists() and (out / "spectrum.dat").exists()
