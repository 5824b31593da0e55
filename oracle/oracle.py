"""ctypes front end of the FP64 CPU oracle (oracle/phx_oracle.c) -- TEST INFRASTRUCTURE ONLY.

The oracle restates the reference renderer's CPU path (nohgz/phoenix src/core/, src/host/io/bhac_io.hpp) in C at
FP64.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libphx_oracle.so")
MAX_FREQS = 32


class OrcParams(C.Structure):
    _fields_ = [
        ("inclination", C.c_double), ("fov_x", C.c_double), ("fov_y", C.c_double), ("r_cam", C.c_double),
        ("t_init", C.c_double), ("pa", C.c_double), ("phi_cam", C.c_double),
        ("img_width", C.c_int32), ("img_height", C.c_int32), ("nfreqs", C.c_int32),
        ("frequencies", C.c_double * MAX_FREQS),
        ("mass", C.c_double), ("distance", C.c_double), ("stepsize", C.c_double), ("max_steps", C.c_int32),
        ("horizon_margin", C.c_double), ("max_order", C.c_int32),
        ("m_unit", C.c_double), ("r_low", C.c_double), ("r_high", C.c_double), ("beta_c", C.c_double),
        ("sigma_cut", C.c_double), ("thetae_min", C.c_double), ("thetae_max", C.c_double), ("rt_outer", C.c_double),
        ("nspin", C.c_int32), ("bpol", C.c_int32), ("nlevels", C.c_int32), ("sfc", C.c_int32),
    ]


# The keys of the reference's default config (input/config.toml) that the render reads, with their values.
DEFAULTS = dict(
    inclination=50.0, img_width=200, img_height=200, fov_x=40.0, fov_y=40.0, r_cam=1e4, t_init=0.0, pa=0.0,
    phi_cam=0.0, frequencies=(230e9,), mass=4.14e6, distance=8.127, stepsize=0.01, max_steps=10000,
    horizon_margin=0.01, max_order=100, m_unit=1e18, r_low=1.0, r_high=1.0, beta_c=1.0, sigma_cut=1.0,
    thetae_min=1e-3, thetae_max=100.0, rt_outer=50.0, nspin=3, bpol=1, nlevels=-1, sfc=1,
)


def make_params(**kw) -> OrcParams:
    d = dict(DEFAULTS)
    d.update(kw)
    p = OrcParams()
    for name, _ in OrcParams._fields_:
        if name in ("frequencies", "nfreqs"):
            continue
        setattr(p, name, d[name])
    freqs = list(d["frequencies"])
    if not 1 <= len(freqs) <= MAX_FREQS:
        raise ValueError("1..32 frequencies")
    p.nfreqs = len(freqs)
    for i, f in enumerate(freqs):
        p.frequencies[i] = f
    return p


def build(force: bool = False) -> str:
    """Compile the oracle library (gcc, FP64, OpenMP) into oracle/_build/."""
    src = os.path.join(HERE, "phx_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(HERE, "phx_oracle.h"))):
        os.makedirs(BUILD, exist_ok=True)
        subprocess.check_call(["gcc", "-O3", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-Wall", "-Wextra", src,
                               "-o", LIB_PATH, "-lm"])
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        L.orc_load.restype = C.c_void_p
        L.orc_load.argtypes = [C.c_char_p, C.c_char_p, C.POINTER(OrcParams), C.c_char_p, C.c_int]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_render.restype = C.c_double
        L.orc_render.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int]
        for name, rt in [("orc_nleafs", C.c_int32), ("orc_nlevels", C.c_int32)]:
            getattr(L, name).restype = rt
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_level_dims.argtypes = [C.c_void_p, C.c_int32, C.c_void_p]
        for name in ("orc_level_map",):
            getattr(L, name).restype = C.POINTER(C.c_int32)
            getattr(L, name).argtypes = [C.c_void_p, C.c_int32]
        for name in ("orc_lb", "orc_dxc", "orc_prim"):
            getattr(L, name).restype = C.POINTER(C.c_double)
            getattr(L, name).argtypes = [C.c_void_p]
        L.orc_scalars.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_pixel_solid_angle.restype = C.c_double
        L.orc_pixel_solid_angle.argtypes = [C.c_void_p]
        L.orc_bessel_ratios.argtypes = [C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_metric_dd.argtypes = [C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        L.orc_metric_uu.argtypes = [C.c_double, C.c_double, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """A BHAC snapshot loaded and decoded by the oracle, ready to render pixels at FP64 on the CPU."""

    def __init__(self, dump: str, grid: str, **params):
        self.params = make_params(**params)
        err = C.create_string_buffer(512)
        self._h = lib().orc_load(dump.encode(), grid.encode(), C.byref(self.params), err, 512)
        if not self._h:
            raise RuntimeError("oracle: " + err.value.decode())
        self.nfreqs = self.params.nfreqs
        self.width, self.height = self.params.img_width, self.params.img_height

    def close(self):
        if self._h:
            lib().orc_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def render(self, pixels=None, threads: int = 0):
        """Render pixel indices i*H+j (default: all, row-major).
        Returns (out[n, nfreqs, 6] float64, stats[n, 3] int64, seconds)."""
        if pixels is None:
            pixels = np.arange(self.width * self.height, dtype=np.int32)
        pixels = np.ascontiguousarray(pixels, dtype=np.int32)
        n = pixels.size
        out = np.zeros((n, self.nfreqs, 6), dtype=np.float64)
        stats = np.zeros((n, 3), dtype=np.int64)
        secs = lib().orc_render(self._h, pixels.ctypes.data, n, out.ctypes.data, stats.ctypes.data, threads)
        return out, stats, secs

    def solid_angle(self) -> float:
        return lib().orc_pixel_solid_angle(self._h)

    def flux(self, out_full):
        """Total Stokes flux [Jy] per frequency of a full image (host/io/output.hpp:43-53)."""
        return flux_from(out_full, self.solid_angle())

    def tables(self):
        L = lib()
        nl = L.orc_nleafs(self._h)
        nlev = L.orc_nlevels(self._h)
        sc = np.zeros(16)
        L.orc_scalars(self._h, sc.ctypes.data)
        cells = int(sc[15])
        maps = []
        for lv in range(nlev):
            dims = np.zeros(3, dtype=np.int32)
            L.orc_level_dims(self._h, lv, dims.ctypes.data)
            n = int(np.prod(dims))
            maps.append(np.ctypeslib.as_array(L.orc_level_map(self._h, lv), shape=(n,)).copy().reshape(dims))
        return dict(
            nleafs=nl, nlevels=nlev, scalars=sc, level_maps=maps,
            lb=np.ctypeslib.as_array(L.orc_lb(self._h), shape=(nl, 3)).copy(),
            dxc=np.ctypeslib.as_array(L.orc_dxc(self._h), shape=(nl, 3)).copy(),
            prim=np.ctypeslib.as_array(L.orc_prim(self._h), shape=(nl, cells, 8)).copy(),
        )


def flux_from(out_full, solid_angle: float):
    """out_full[npix, nfreqs, 6] -> flux[nfreqs, 4] in Jy, skipping pixels with a non-finite Stokes sum."""
    iquv = out_full[..., :4]
    ok = np.isfinite(iquv.sum(axis=-1))
    return np.where(ok[..., None], iquv, 0.0).sum(axis=0) * solid_angle * 1e23


def bessel_ratios(x: float):
    r10, r02 = C.c_double(), C.c_double()
    lib().orc_bessel_ratios(x, C.byref(r10), C.byref(r02))
    return r10.value, r02.value
