"""The PHOENIX command line (config.toml + overrides) and the output writers, without a GPU."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

import phoenix_b200 as P
from tests.golden.cases import CASES, write_config
from tests.h5mini import H5File


def _run(built, args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([built["cli"]] + args, capture_output=True, text=True, env=e)


@pytest.fixture()
def cfg(tmp_path):
    path = str(tmp_path / "config.toml")
    write_config(path, CASES["cfg1"], "/data/dump.dat", "/data/grid.in", str(tmp_path / "out"))
    return path


def parsed(built, args):
    r = _run(built, args, {"PHX_PRINT_CONFIG": "1"})
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_config_values_and_overrides(built, cfg):
    c = parsed(built, [cfg])
    assert c["inclination"] == 10.0 and c["img_width"] == 64 and c["frequencies"] == [230e9]
    assert c["nlevels"] == 3 and c["sfc"] == 1 and c["max_steps"] == 10000
    c = parsed(built, [cfg, "camera.inclination=60", "plasma.m_unit=1e19", "integration.max_steps=2.5e3"])
    assert c["inclination"] == 60.0 and c["m_unit"] == 1e19 and c["max_steps"] == 2500
    # any frequency override replaces every frequency form of the file
    c = parsed(built, [cfg, "camera.frequency_list=[86e9, 345e9,]"])
    assert c["frequencies"] == [86e9, 345e9]
    c = parsed(built, [cfg, "camera.frequency_linspace=[100e9, 400e9, 4]"])
    assert c["frequencies"] == [100e9, 200e9, 300e9, 400e9]
    c = parsed(built, [cfg, "camera.frequency_logspace=[100e9, 400e9, 3]"])
    assert c["frequencies"][0] == 100e9 and c["frequencies"][2] == 400e9
    assert c["frequencies"][1] == pytest.approx(200e9, rel=1e-15)


@pytest.mark.parametrize("over,msg", [
    (["bogus.key=1"], "unknown key bogus.key"),
    (["camera.frequency_list=[230e9, 2.3e11]"], "duplicate frequency 2.300000e+11"),
    (["camera.frequency_linspace=[1e9, 2e9]"], "has 2arguments! (Expected 3)"),
    (["camera.frequency_linspace=[1e9, 2e9, 2.5]"], "n must be an integer >= 2"),
    (["camera.frequency_logspace=[3e9, 2e9, 4]"], "need 0 < start < stop!"),
    (["camera.frequency=abc"], "camera.frequency: not a number: abc"),
    (["camera.frequency_list=230e9"], "must be a list on ONE line"),
    (["output.image=png"], "output.image must be hdf5, text, both or none"),
    (["output.block_size=0"], "output.block_size must be >= 1"),
    (["plasma.beta_c=0"], "plasma.beta_c must be > 0"),
    (["noequals"], "Override must be section.key=value: noequals"),
])
def test_config_errors(built, cfg, over, msg):
    r = _run(built, [cfg] + over)
    assert r.returncode == 1
    assert msg in r.stderr


REF_FP64 = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                        "ref_render_fp64")


@pytest.mark.skipif(not os.path.exists(REF_FP64), reason="the reference's CPU build (oracle/_ref) is not built here")
@pytest.mark.parametrize("over", [
    ["bogus.key=1"], ["camera.frequency_list=[230e9, 2.3e11]"], ["camera.frequency_linspace=[1e9, 2e9]"],
    ["camera.frequency_linspace=[1e9, 2e9, 2.5]"], ["camera.frequency_logspace=[3e9, 2e9, 4]"],
    ["camera.frequency=abc"], ["camera.frequency_list=230e9"], ["camera.frequency_list=[]"],
    ["camera.frequency_list=[1e9, x]"], ["camera.frequency_list=[1e9, -2e9]"], ["output.image=png"],
    ["output.block_size=0"], ["plasma.beta_c=0"], ["noequals"],
    ["camera.frequency=1e9", "camera.frequency_list=[2e9]"],
    ["camera.frequency_list=[1e9,2e9]", "camera.frequency_list=[3e9, 3e9]"],
])
def test_config_errors_match_reference(built, cfg, over):
    """The same config and overrides give the reference's own parser (host/io/config.hpp, compiled into its CPU
    build) and ours the same error text."""
    ours = _run(built, [cfg] + over)
    ref = subprocess.run([REF_FP64, cfg] + over, capture_output=True, text=True)
    assert ours.returncode == 1 and ref.returncode == 1
    what = ref.stderr.strip().split("ref_render: ", 1)[1]
    assert what in ours.stderr


@pytest.mark.skipif(not os.path.exists(REF_FP64), reason="the reference's CPU build (oracle/_ref) is not built here")
def test_config_file_errors_match_reference(built, tmp_path, cfg):
    text = open(cfg).read()
    bad = tmp_path / "bad.toml"
    for variant in (text.replace("[camera]", "[camera"), text + "\n[camera]\ninclination = 3\n",
                    text.replace("mass = ", "#mass = ").replace("rt_outer = ", "#rt_outer = "),
                    text.replace("mass = ", "mass ")):
        bad.write_text(variant)
        ours = _run(built, [str(bad)])
        ref = subprocess.run([REF_FP64, str(bad)], capture_output=True, text=True)
        assert ours.returncode == 1 and ref.returncode == 1
        assert ref.stderr.strip().split("ref_render: ", 1)[1] in ours.stderr


def test_config_file_errors(built, tmp_path, cfg):
    text = open(cfg).read()
    bad = tmp_path / "bad.toml"
    bad.write_text(text.replace("[camera]", "[camera"))
    assert "bad section header" in _run(built, [str(bad)]).stderr
    bad.write_text(text + "\n[camera]\ninclination = 3\n")
    assert "duplicate key camera.inclination" in _run(built, [str(bad)]).stderr
    bad.write_text(text.replace("mass = ", "#mass = ").replace("rt_outer = ", "#rt_outer = "))
    assert "missing required key(s): black_hole.mass plasma.rt_outer" in _run(built, [str(bad)]).stderr
    bad.write_text(text.replace("frequency = 230000000000.0", 'frequency = 230e9 # "quoted # is not a comment"'))
    assert parsed(built, [str(bad)])["frequencies"] == [230e9]
    r = _run(built, ["--help"])
    assert r.returncode == 0 and "usage:" in r.stderr
    assert "Cannot open file" in _run(built, [str(tmp_path / "missing.toml")]).stderr


def _fake_render(W, H, F, seed=0):
    rng = np.random.default_rng(seed)
    res = rng.random((W, H, F, 6))
    res[..., :4] *= 1e-20
    res[1, 2, 0, 0] = np.nan  # one non-finite pixel, skipped by the flux
    return res


def test_hdf5_image_layout(built, tmp_path):
    W, H, bs = 20, 30, 10
    p = P.make_params(img_width=W, img_height=H, frequencies=[86e9, 230e9], fov_x=30.0, fov_y=45.0)
    res = _fake_render(W, H, 2)
    flux = P.write_output(res, p, str(tmp_path), "hdf5", bs)
    assert np.allclose(flux, P.flux(res, p), rtol=1e-12, atol=0)
    f = H5File(str(tmp_path / "img_data.h5"))
    names = sorted(n for n, _ in f.root_group())
    fs = ["%e" % nu for nu in (86e9, 230e9)]
    expect = sorted(["alpha", "beta"] + [q + s for s in fs for q in ("I", "Q", "U", "V", "tau", "tauF")])
    assert names == expect
    nbj, nblocks = H // bs, (W // bs) * (H // bs)
    b = np.arange(nblocks)[:, None]
    q = np.arange(bs * bs)[None, :]
    ii, jj = (b // nbj) * bs + q // bs, (b % nbj) * bs + q % bs
    for fi, s in enumerate(fs):
        for k, name in enumerate(("I", "Q", "U", "V")):
            got = f.read(name + s)
            assert got.shape == (nblocks, bs * bs) and got.dtype == np.float64
            np.testing.assert_array_equal(got, res[ii, jj, fi, k] * 1e23)
        np.testing.assert_array_equal(f.read("tau" + s), res[ii, jj, fi, 4])
        np.testing.assert_array_equal(f.read("tauF" + s), res[ii, jj, fi, 5])
    np.testing.assert_allclose(f.read("alpha"), -15.0 + (ii + 0.5) * 30.0 / W, rtol=0, atol=1e-14)
    np.testing.assert_allclose(f.read("beta"), -22.5 + (jj + 0.5) * 45.0 / H, rtol=0, atol=1e-14)
    assert (tmp_path / "spectrum.dat").exists() and not (tmp_path / "image.dat").exists()


def test_text_outputs_and_hdf5_fallback(built, tmp_path):
    W, H = 12, 8
    p = P.make_params(img_width=W, img_height=H, frequencies=[230e9])
    res = _fake_render(W, H, 1, seed=3)
    P.write_output(res, p, str(tmp_path), "hdf5", 5)  # 5 does not divide 12: text image instead
    assert not (tmp_path / "img_data.h5").exists()
    rows = np.loadtxt(str(tmp_path / "image.dat"))
    assert rows.shape == (W * H, 8)
    unit = P.pixel_solid_angle(p) * 1e23
    np.testing.assert_allclose(rows[:, 2], res[..., 0, 0].reshape(-1) * unit, rtol=1e-14)
    L = 6.674e-8 * p.mass * 1.989e33 / 2.99792458e10 ** 2
    arcsec = 206265.0 * L / (p.distance * 3.086e21)
    np.testing.assert_allclose(rows[::H, 0], (-20.0 + (np.arange(W) + 0.5) * 40.0 / W) * arcsec, rtol=1e-14)
    spec = np.loadtxt(str(tmp_path / "spectrum.dat"))
    assert spec[0] == 230e9
    np.testing.assert_allclose(spec[1:5], P.flux(res, p)[0], rtol=1e-14)
    ok = np.isfinite(res[..., 0, :4].sum(-1))
    np.testing.assert_allclose(spec[5], res[..., 0, 4][ok].mean(), rtol=1e-14)
