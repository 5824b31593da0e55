"""The parity cases shared by the golden-fixture script, the tests and the smoke check.

Snapshots are generated by phx_gen_snapshot from the arguments below.  `cfg1` is the reference-sized CPU-runnable
case (base grid 64x32x32 in 8^3 blocks, base + 2 refinement levels, seed 0); `small` is a little k-j-i-ordered
(non-Morton) snapshot with one refinement level.
"""
from __future__ import annotations

SNAPSHOTS = {
    "cfg1": {"gen_args": ["--seed", "0", "--base", "64", "32", "32", "--nlevels", "3"], "nlevels": 3, "sfc": True},
    "small": {"gen_args": ["--seed", "3", "--base", "32", "16", "16", "--nlevels", "2", "--sfc", "0", "--nws", "0"],
              "nlevels": 2, "sfc": False},
}

# config.toml keys of each case (the rest are the reference's defaults, input/config.toml)
CASES = {
    # config 1: 64x64, inclination 10 deg, 230 GHz, m_unit 1.2e18
    "cfg1": dict(snapshot="cfg1", inclination=10.0, img_width=64, img_height=64, frequencies=[230e9],
                 m_unit=1.2e18),
    # optically and Faraday thick, three frequencies, position angle
    "thick": dict(snapshot="cfg1", inclination=60.0, img_width=32, img_height=32, frequencies=[86e9, 230e9, 345e9],
                  m_unit=1e19, pa=30.0),
    # non-square image from below the equator with a camera azimuth, k-j-i ordered snapshot
    "edge": dict(snapshot="small", inclination=163.0, img_width=16, img_height=12, frequencies=[345e9],
                 m_unit=3e18, phi=45.0, fov_x=30.0, fov_y=24.0),
}

DEFAULTS = dict(inclination=50.0, img_width=200, img_height=200, fov_x=40.0, fov_y=40.0, r_cam=1e4, t_init=0.0,
                pa=0.0, phi=0.0, mass=4.14e6, distance=8.127, stepsize=0.01, max_steps=10000, horizon_margin=0.01,
                max_order=100, m_unit=1e18, r_low=1.0, r_high=1.0, beta_c=1.0, sigma_cut=1.0, thetae_min=1e-3,
                thetae_max=100.0, rt_outer=50.0)


def case_params(name):
    """Full render parameters of a case (config key names; `frequencies` a list)."""
    c = dict(DEFAULTS)
    c.update({k: v for k, v in CASES[name].items() if k != "snapshot"})
    return c


def write_config(path, case, dump, grid, outdir):
    """A config.toml with the case's keys, in the reference's format (input/config.toml)."""
    c = dict(DEFAULTS)
    c.update({k: v for k, v in case.items() if k != "snapshot"})
    snap = SNAPSHOTS[case["snapshot"]]
    fr = c["frequencies"]
    freq_line = f"frequency = {fr[0]!r}" if len(fr) == 1 else "frequency_list = [" + ", ".join(repr(f) for f in fr) + "]"
    text = f"""[visual]
show_header = false
[output]
dir = "{outdir}"
image = "none"
[camera]
inclination = {c['inclination']!r}
img_width = {c['img_width']}
img_height = {c['img_height']}
fov_x = {c['fov_x']!r}
fov_y = {c['fov_y']!r}
r_cam = {c['r_cam']!r}
t_init = {c['t_init']!r}
pa = {c['pa']!r}
phi = {c['phi']!r}
{freq_line}
[black_hole]
mass = {c['mass']!r}
distance = {c['distance']!r}
[integration]
stepsize = {c['stepsize']!r}
max_steps = {c['max_steps']}
horizon_margin = {c['horizon_margin']!r}
max_order = {c['max_order']}
[plasma]
m_unit = {c['m_unit']!r}
r_low = {c['r_low']!r}
r_high = {c['r_high']!r}
beta_c = {c['beta_c']!r}
sigma_cut = {c['sigma_cut']!r}
thetae_min = {c['thetae_min']!r}
thetae_max = {c['thetae_max']!r}
rt_outer = {c['rt_outer']!r}
[grmhd]
dump_file = "{dump}"
grid_file = "{grid}"
gpu_decode = false
nspin = 3
bpol = 1
sfc = {'true' if snap['sfc'] else 'false'}
nlevels = {snap['nlevels']}
"""
    with open(path, "w") as f:
        f.write(text)
