"""ctypes binding of the C ABI in include/phoenix_b200.h (libphoenix_b200.so, built in-tree by phoenix_b200.build).

There is no fallback: if the library is missing or cannot be loaded, importing the render entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_build", "libphoenix_b200.so")

MAX_FREQS = 32
MAX_LEVELS = 16

PHX_OK, PHX_E_INVALID, PHX_E_IO, PHX_E_CUDA, PHX_E_TIMEOUT, PHX_E_UNSUPPORTED = 0, -1, -2, -3, -4, -5
PREC_FP32, PREC_FP64, PREC_MIXED = 0, 1, 2
PRECISIONS = {"fp32": PREC_FP32, "fp64": PREC_FP64, "mixed": PREC_MIXED}
SNAP_F64_PRIMS = 1
SNAP_GPU_DECODE = 2
NOALLOC_MAX_JOBS = 1 << 20
NUM_COUNTERS = 16
CTR = dict(queue=0, steps=1, nplasma=2, bad=3, scans=4, fp64_steps=5, fp64_ops=6, rays=7)

# Every symbol include/phoenix_b200.h declares.
EXPORTS = ["phx_default_params", "phx_snapshot_create", "phx_snapshot_load", "phx_snapshot_destroy",
           "phx_bhac_read", "phx_bhac_describe", "phx_bhac_free", "phx_snapshot_bytes", "phx_schedule_morton", "phx_schedule_tiles", "phx_default_pixel_order", "phx_render", "phx_render_async", "phx_render_noalloc", "phx_write_output", "phx_last_error",
           "phx_version", "phx_default_batch_options", "phx_batch_create", "phx_batch_launch", "phx_batch_run",
           "phx_batch_result", "phx_batch_device_result", "phx_batch_tuning", "phx_batch_destroy",
           "phx_default_server_options", "phx_server_create", "phx_server_submit", "phx_server_poll",
           "phx_server_wait", "phx_server_result", "phx_server_stats", "phx_server_destroy",
           "phx_snapshot_info", "phx_snapshot_download", "phx_spectrum_async", "phx_batch_spectrum",
           "phx_measure_fp32_peak"]
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3
TUNE_MAX_CANDIDATES = 16


class PhxFreqOut(C.Structure):
    _fields_ = [("IQUV", C.c_double * 4), ("tau", C.c_double), ("tauF", C.c_double)]


class PhxSpectrum(C.Structure):
    _fields_ = [("IQUV", C.c_double * 4), ("tau_mean", C.c_double), ("tauF_mean", C.c_double),
                ("n_flux", C.c_int64), ("n_tau", C.c_int64)]


class PhxSnapshotDesc(C.Structure):
    _fields_ = [
        ("nleafs", C.c_int32), ("nx", C.c_int32 * 3), ("ng", C.c_int32 * 3), ("nlevels", C.c_int32),
        ("a", C.c_double), ("hslope", C.c_double), ("gam", C.c_double),
        ("x_lo", C.c_double * 3), ("x_hi", C.c_double * 3),
        ("lb", C.c_void_p), ("dxc", C.c_void_p), ("prim_f32", C.c_void_p), ("prim_f64", C.c_void_p),
        ("level_map", C.c_void_p),
    ]


class PhxReadOptions(C.Structure):
    _fields_ = [("nspin", C.c_int32), ("bpol", C.c_int32), ("sfc", C.c_int32), ("nlevels", C.c_int32)]


class PhxRenderParams(C.Structure):
    _fields_ = [
        ("inclination", C.c_double), ("fov_x", C.c_double), ("fov_y", C.c_double), ("r_cam", C.c_double),
        ("t_init", C.c_double), ("pa", C.c_double), ("phi", C.c_double),
        ("img_width", C.c_int32), ("img_height", C.c_int32), ("nfreqs", C.c_int32),
        ("frequencies", C.c_double * MAX_FREQS),
        ("mass", C.c_double), ("distance", C.c_double),
        ("stepsize", C.c_double), ("max_steps", C.c_int32), ("horizon_margin", C.c_double), ("max_order", C.c_int32),
        ("m_unit", C.c_double), ("r_low", C.c_double), ("r_high", C.c_double), ("beta_c", C.c_double),
        ("sigma_cut", C.c_double), ("thetae_min", C.c_double), ("thetae_max", C.c_double), ("rt_outer", C.c_double),
        ("precision", C.c_int32), ("r_fp64", C.c_double), ("tau_fp64", C.c_double),
        ("block", C.c_int32), ("period", C.c_int32), ("blocks_per_sm", C.c_int32), ("refill_lanes", C.c_int32),
    ]


class PhxRenderInfo(C.Structure):
    _fields_ = [
        ("device", C.c_char * 256), ("sms", C.c_int32), ("blocks", C.c_int32), ("block", C.c_int32),
        ("regs", C.c_int32), ("local_bytes", C.c_int32), ("upload_s", C.c_double), ("kernel_s", C.c_double),
        ("steps", C.c_int64), ("nplasma", C.c_int64), ("bad", C.c_int64), ("scans", C.c_int64),
        ("fp64_steps", C.c_int64), ("fp64_ops", C.c_int64),
    ]

    def as_dict(self):
        d = {name: getattr(self, name) for name, _ in self._fields_}
        d["device"] = self.device.decode()
        return d


class PhxBatchItem(C.Structure):
    _fields_ = [("snapshot", C.c_void_p), ("params", PhxRenderParams), ("jobs", C.c_void_p), ("njobs", C.c_int64)]


class PhxBatchOptions(C.Structure):
    _fields_ = [("tile_rays", C.c_int32), ("blocks_per_sm", C.c_int32), ("period", C.c_int32),
                ("autotune", C.c_int32), ("sample_stride", C.c_int32), ("keep_order", C.c_int32),
                ("tile_shape", C.c_int32), ("lane_setup", C.c_int32), ("refill_lanes", C.c_int32)]


class PhxBatchTuning(C.Structure):
    _fields_ = [
        ("blocks_per_sm", C.c_int32), ("period", C.c_int32), ("tile_rays", C.c_int32),
        ("grid", C.c_int32), ("block", C.c_int32), ("regs", C.c_int32), ("local_bytes", C.c_int32),
        ("ncand", C.c_int32), ("cand_blocks_per_sm", C.c_int32 * TUNE_MAX_CANDIDATES),
        ("cand_period", C.c_int32 * TUNE_MAX_CANDIDATES), ("cand_ms", C.c_double * TUNE_MAX_CANDIDATES),
        ("tile_shape", C.c_int32), ("cand_tile_shape", C.c_int32 * TUNE_MAX_CANDIDATES),
        ("nitems", C.c_int64), ("ntiles", C.c_int64), ("nrays", C.c_int64), ("device_bytes", C.c_int64),
        ("refill_lanes", C.c_int32), ("cand_refill_lanes", C.c_int32 * TUNE_MAX_CANDIDATES),
    ]

    def as_dict(self):
        n = self.ncand
        d = {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("cand_")}
        d["candidates"] = [dict(blocks_per_sm=self.cand_blocks_per_sm[i], period=self.cand_period[i],
                                refill_lanes=self.cand_refill_lanes[i], tile_shape=self.cand_tile_shape[i],
                                ms=self.cand_ms[i]) for i in range(n)]
        return d


class PhxSnapshotInfo(C.Structure):
    _fields_ = [("nleafs", C.c_int64), ("cells", C.c_int32), ("nlevels", C.c_int32), ("nx", C.c_int32 * 3),
                ("ng", C.c_int32 * 3), ("a", C.c_double), ("hslope", C.c_double), ("gam", C.c_double),
                ("x_lo", C.c_double * 3), ("x_hi", C.c_double * 3), ("has_f64_prims", C.c_int32),
                ("gpu_decoded", C.c_int32), ("bytes", C.c_int64), ("read_s", C.c_double), ("decode_s", C.c_double),
                ("upload_s", C.c_double)]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if hasattr(v, "__len__") else v
        return d


class PhxServerOptions(C.Structure):
    _fields_ = [
        ("memory_budget", C.c_int64), ("arena_bytes", C.c_int64), ("precision", C.c_int32), ("max_freqs", C.c_int32),
        ("tile_rays", C.c_int32), ("period", C.c_int32), ("blocks_per_sm", C.c_int32), ("max_items", C.c_int32),
        ("max_tiles", C.c_int64), ("idle_ns", C.c_int32), ("idle_limit", C.c_int64), ("linger_ms", C.c_double),
        ("poll_us", C.c_int32), ("publish_chunk", C.c_int32), ("backlog_rays", C.c_int64), ("small_rays", C.c_int64),
        ("refill_lanes", C.c_int32),
    ]


class PhxRequestTiming(C.Structure):
    _fields_ = [("submitted_s", C.c_double), ("admitted_s", C.c_double), ("done_s", C.c_double),
                ("rays", C.c_int64), ("steps", C.c_int64), ("nplasma", C.c_int64), ("bad", C.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PhxServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("submitted", "completed", "inflight", "pending", "generations", "rays",
                                         "steps", "snapshot_bytes", "table_bytes", "arena_bytes", "arena_used",
                                         "job_table_bytes")] + [("grid", C.c_int32), ("regs", C.c_int32),
                                                                ("idle_exits", C.c_int64), ("retries", C.c_int64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class PhxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"phoenix_b200 error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """The loaded native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not found: build it with `python -m phoenix_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    L.phx_default_params.argtypes = [P(PhxRenderParams)]
    L.phx_default_params.restype = None
    L.phx_snapshot_create.argtypes = [P(PhxSnapshotDesc), C.c_int32, P(C.c_void_p)]
    L.phx_snapshot_load.argtypes = [C.c_char_p, C.c_char_p, P(PhxReadOptions), C.c_int32, P(C.c_void_p)]
    L.phx_snapshot_destroy.argtypes = [C.c_void_p]
    L.phx_snapshot_destroy.restype = None
    L.phx_bhac_read.argtypes = [C.c_char_p, C.c_char_p, P(PhxReadOptions), C.c_int32, P(C.c_void_p)]
    L.phx_bhac_describe.argtypes = [C.c_void_p, P(PhxSnapshotDesc)]
    L.phx_bhac_free.argtypes = [C.c_void_p]
    L.phx_bhac_free.restype = None
    L.phx_snapshot_bytes.argtypes = [C.c_void_p]
    L.phx_snapshot_bytes.restype = C.c_int64
    L.phx_schedule_morton.argtypes = [C.c_int32, C.c_int32, C.c_void_p]
    L.phx_schedule_tiles.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    L.phx_default_pixel_order.argtypes = [C.c_void_p]
    L.phx_default_pixel_order.restype = C.c_int
    L.phx_render.argtypes = [C.c_void_p, P(PhxRenderParams), C.c_void_p, C.c_int64, C.c_void_p, P(PhxRenderInfo)]
    L.phx_render_async.argtypes = [C.c_void_p, P(PhxRenderParams), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]
    L.phx_render_noalloc.argtypes = [C.c_void_p, P(PhxRenderParams), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.phx_write_output.argtypes = [P(PhxRenderParams), C.c_void_p, C.c_char_p, C.c_char_p, C.c_int32, C.c_void_p]
    L.phx_write_output.restype = C.c_int
    L.phx_last_error.restype = C.c_char_p
    L.phx_version.restype = C.c_char_p
    L.phx_default_batch_options.argtypes = [P(PhxBatchOptions)]
    L.phx_default_batch_options.restype = None
    L.phx_batch_create.argtypes = [P(PhxBatchItem), C.c_int32, P(PhxBatchOptions), P(C.c_void_p)]
    L.phx_batch_launch.argtypes = [C.c_void_p, C.c_void_p]
    L.phx_batch_run.argtypes = [C.c_void_p]
    L.phx_batch_result.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, P(PhxRenderInfo)]
    L.phx_batch_device_result.argtypes = [C.c_void_p, C.c_int32, P(C.c_void_p)]
    L.phx_batch_tuning.argtypes = [C.c_void_p, P(PhxBatchTuning)]
    L.phx_batch_spectrum.argtypes = [C.c_void_p, C.c_int32, P(PhxSpectrum)]
    L.phx_spectrum_async.argtypes = [P(PhxRenderParams), C.c_void_p, C.c_void_p, C.c_void_p]
    L.phx_measure_fp32_peak.argtypes = [C.c_int32, P(C.c_double)]
    L.phx_batch_destroy.argtypes = [C.c_void_p]
    L.phx_batch_destroy.restype = None
    L.phx_snapshot_info.argtypes = [C.c_void_p, P(PhxSnapshotInfo)]
    L.phx_snapshot_info.restype = C.c_int
    L.phx_snapshot_download.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.phx_snapshot_download.restype = C.c_int
    L.phx_default_server_options.argtypes = [P(PhxServerOptions)]
    L.phx_default_server_options.restype = None
    L.phx_server_create.argtypes = [C.c_void_p, C.c_int32, P(PhxServerOptions), P(C.c_void_p)]
    L.phx_server_submit.argtypes = [C.c_void_p, C.c_int32, P(PhxRenderParams), P(C.c_int64)]
    L.phx_server_poll.argtypes = [C.c_void_p, C.c_int64, P(C.c_int32)]
    L.phx_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_double, P(C.c_int32)]
    L.phx_server_result.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, P(PhxRequestTiming)]
    L.phx_server_stats.argtypes = [C.c_void_p, P(PhxServerStats)]
    L.phx_server_destroy.argtypes = [C.c_void_p]
    L.phx_server_destroy.restype = None
    for name in ("phx_server_create", "phx_server_submit", "phx_server_poll", "phx_server_wait", "phx_server_result",
                 "phx_server_stats"):
        getattr(L, name).restype = C.c_int
    for name in ("phx_snapshot_create", "phx_snapshot_load", "phx_bhac_read", "phx_bhac_describe", "phx_schedule_morton",
                 "phx_schedule_tiles", "phx_render", "phx_render_async", "phx_render_noalloc", "phx_batch_create", "phx_batch_launch",
                 "phx_batch_run", "phx_batch_result", "phx_batch_device_result", "phx_batch_tuning",
                 "phx_batch_spectrum", "phx_spectrum_async", "phx_measure_fp32_peak"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(code: int):
    if code != PHX_OK:
        raise PhxError(code, lib().phx_last_error().decode())


def make_params(**kw) -> PhxRenderParams:
    """Render parameters: the reference's config.toml defaults overridden by keyword (config key names;
    `frequencies` is a sequence, `precision` one of fp32 / fp64 / mixed or a PREC_* code)."""
    p = PhxRenderParams()
    lib().phx_default_params(C.byref(p))
    for k, v in kw.items():
        if k == "frequencies" or k == "frequency":
            fr = [float(v)] if np.isscalar(v) else [float(x) for x in v]
            if not 1 <= len(fr) <= MAX_FREQS:
                raise ValueError("1..32 frequencies")
            p.nfreqs = len(fr)
            for i, f in enumerate(fr):
                p.frequencies[i] = f
        elif k == "precision":
            p.precision = PRECISIONS[v] if isinstance(v, str) else int(v)
        elif k in ("img", "resolution"):
            p.img_width = p.img_height = int(v)
        else:
            if not hasattr(p, k):
                raise KeyError(f"unknown render parameter {k}")
            setattr(p, k, v)
    return p


def schedule_morton(width: int, height: int) -> np.ndarray:
    jobs = np.empty(width * height, dtype=np.int32)
    check(lib().phx_schedule_morton(width, height, jobs.ctypes.data))
    return jobs


# pixel orders (PHX_TILE_*): Morton, or w x h tiles (w along i, h along j) in Morton order of the tiles, or 4x8 tiles
# by the distance of their centre from the image centre
TILE_SHAPES = {"morton": 0, "16x2": 1, "32x1": 2, "4x8": 3, "2x16": 4, "center4x8": 5}


def schedule_tiles(width: int, height: int, shape="morton") -> np.ndarray:
    """Pixel job list in the order of a tile shape (a TILE_SHAPES name or PHX_TILE_* number)."""
    code = TILE_SHAPES[shape] if isinstance(shape, str) else int(shape)
    jobs = np.empty(width * height, dtype=np.int32)
    check(lib().phx_schedule_tiles(width, height, code, jobs.ctypes.data))
    return jobs


def default_pixel_order(params) -> int:
    """The library's pixel order (PHX_TILE_*) for an image: 4x8 tiles, centre first."""
    return lib().phx_default_pixel_order(C.byref(params))


def write_output(res, params, outdir: str, image: str = "hdf5", block_size: int = 10):
    """Write img_data.h5 / image*.dat / spectrum.dat like PHOENIX; returns the flux [nfreqs, 4] in Jy."""
    r = np.ascontiguousarray(res, dtype=np.float64)
    if r.size != params.img_width * params.img_height * params.nfreqs * 6:
        raise ValueError("res does not match the image size")
    flux = np.zeros((params.nfreqs, 4))
    check(lib().phx_write_output(C.byref(params), r.ctypes.data, outdir.encode(), image.encode(), block_size,
                                 flux.ctypes.data))
    return flux
