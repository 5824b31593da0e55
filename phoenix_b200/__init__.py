"""PHOENIX-B200: the B200-native raymarch path of the PHOENIX GRRT renderer.

Python front end of the C ABI (include/phoenix_b200.h).  A Snapshot is a BHAC block-AMR GRMHD snapshot resident on
the GPU; Snapshot.render() marches every pixel's null geodesic through it and returns the reference's per-pixel
FreqOut records (I, Q, U, V, tau, tauF) at index (i * img_height + j) * nfreqs + f, like the reference's
device::render (src/device/kernel.cu:284-360).  The work runs in the sm_100a kernels of libphoenix_b200.so; there is
no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native
from .native import (CTR, NUM_COUNTERS, PREC_FP32, PREC_FP64, PREC_MIXED, PhxError, PhxRenderInfo, make_params,
                     TILE_SHAPES, default_pixel_order, schedule_morton, schedule_tiles, write_output)

__all__ = ["Snapshot", "Batch", "Server", "make_params", "schedule_morton", "schedule_tiles", "default_pixel_order", "TILE_SHAPES", "write_output", "flux", "pixel_solid_angle", "device_spectrum", "spectrum_rows", "measure_fp32_peak", "PhxError", "PREC_FP32",
           "PREC_FP64", "PREC_MIXED", "CTR", "NUM_COUNTERS"]

G_GRAV, M_SUN, C_LIGHT, KPC, JANSKY = 6.674e-8, 1.989e33, 2.99792458e10, 3.086e21, 1e23


class Snapshot:
    """A snapshot uploaded once and kept on the device until close()."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def load(cls, dump: str, grid: str, nspin: int = 3, bpol: int = 1, sfc: bool = True, nlevels: int = -1,
             f64_prims: bool = False, gpu_decode: bool = False) -> "Snapshot":
        """Read a BHAC dump + grid file (config.toml [grmhd] keys) and make it resident; the cells are decoded on the
        host, or on the GPU while the dump streams in (gpu_decode)."""
        L = native.lib()
        opt = native.PhxReadOptions(nspin, bpol, 1 if sfc else 0, nlevels)
        h = C.c_void_p()
        flags = (native.SNAP_F64_PRIMS if f64_prims else 0) | (native.SNAP_GPU_DECODE if gpu_decode else 0)
        native.check(L.phx_snapshot_load(dump.encode(), grid.encode(), C.byref(opt), flags, C.byref(h)))
        return cls(h.value)

    def info(self) -> dict:
        i = native.PhxSnapshotInfo()
        native.check(native.lib().phx_snapshot_info(self._h, C.byref(i)))
        return i.as_dict()

    def download(self, f64: bool = False):
        """The device primitives as numpy arrays [nleafs, cells, 8] (FP32, and FP64 when asked)."""
        i = self.info()
        shape = (i["nleafs"], i["cells"], 8)
        pf = np.empty(shape, np.float32)
        pd = np.empty(shape, np.float64) if f64 else None
        native.check(native.lib().phx_snapshot_download(self._h, pf.ctypes.data, pd.ctypes.data if f64 else None))
        return (pf, pd) if f64 else pf

    @classmethod
    def from_arrays(cls, *, nx, ng, nlevels, a, hslope, gam, x_lo, x_hi, lb, dxc, prim_f32, level_maps,
                    prim_f64=None) -> "Snapshot":
        """Upload a decoded snapshot given as numpy arrays (lb, dxc: [nleafs, 3] float64; prim: [nleafs, cells, 8];
        level_maps: nlevels int32 arrays)."""
        L = native.lib()
        lb = np.ascontiguousarray(lb, dtype=np.float64)
        dxc = np.ascontiguousarray(dxc, dtype=np.float64)
        pf = np.ascontiguousarray(prim_f32, dtype=np.float32)
        pd = None if prim_f64 is None else np.ascontiguousarray(prim_f64, dtype=np.float64)
        maps = [np.ascontiguousarray(m, dtype=np.int32) for m in level_maps]
        ptrs = (C.c_void_p * len(maps))(*[m.ctypes.data for m in maps])
        d = native.PhxSnapshotDesc()
        d.nleafs = lb.shape[0]
        d.nlevels = nlevels
        for k in range(3):
            d.nx[k], d.ng[k], d.x_lo[k], d.x_hi[k] = nx[k], ng[k], x_lo[k], x_hi[k]
        d.a, d.hslope, d.gam = a, hslope, gam
        d.lb, d.dxc, d.prim_f32 = lb.ctypes.data, dxc.ctypes.data, pf.ctypes.data
        d.prim_f64 = pd.ctypes.data if pd is not None else None
        d.level_map = C.cast(ptrs, C.c_void_p)
        h = C.c_void_p()
        native.check(L.phx_snapshot_create(C.byref(d), native.SNAP_F64_PRIMS if pd is not None else 0, C.byref(h)))
        return cls(h.value)

    @property
    def handle(self):
        return self._h

    def nbytes(self) -> int:
        return native.lib().phx_snapshot_bytes(self._h)

    def render(self, params=None, jobs=None, out=None, **kw):
        """Render; returns (res[img_width, img_height, nfreqs, 6] float64, info dict).  `jobs`: pixel indices
        i * img_height + j (default every pixel, in the library's default pixel order); pixels outside `jobs` keep `out`'s values."""
        p = params if params is not None else make_params(**kw)
        W, H, F = p.img_width, p.img_height, p.nfreqs
        res = out if out is not None else np.zeros((W, H, F, 6), dtype=np.float64)
        if res.shape != (W, H, F, 6) or res.dtype != np.float64 or not res.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (W, H, nfreqs, 6)")
        info = PhxRenderInfo()
        if jobs is None:
            jp, nj = None, 0
        else:
            jobs = np.ascontiguousarray(jobs, dtype=np.int32)
            jp, nj = jobs.ctypes.data, jobs.size
        native.check(native.lib().phx_render(self._h, C.byref(p), jp, nj, res.ctypes.data, C.byref(info)))
        return res, info.as_dict()

    def render_async(self, params, d_jobs: int, njobs: int, d_res: int, d_counters: int, d_pixstats: int = 0,
                     stream: int = 0):
        """Launch on a CUDA stream with device pointers (e.g. torch tensors' data_ptr()); allocates nothing."""
        native.check(native.lib().phx_render_async(self._h, C.byref(params), d_jobs or None, njobs, d_res,
                                                   d_pixstats or None, d_counters, stream or None))

    def close(self):
        if self._h and self._h.value:
            native.lib().phx_snapshot_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many images (any mix of snapshots, resolutions, cameras, frequencies and plasma parameters, one precision)
    rendered by one persistent, graph-captured launch of the queue kernel.  items: (snapshot, params) or
    (snapshot, params, jobs) tuples."""

    def __init__(self, items, tile_rays=32, blocks_per_sm=0, period=0, autotune=False, sample_stride=16,
                 keep_order=False, tile_shape=0, lane_setup=False, refill_lanes=0):
        L = native.lib()
        n = len(items)
        arr = (native.PhxBatchItem * n)()
        self._keep = []
        self.params = []
        for k, it in enumerate(items):
            snap, p = it[0], it[1]
            jobs = it[2] if len(it) > 2 else None
            arr[k].snapshot = snap.handle.value
            arr[k].params = p
            if jobs is not None:
                j = np.ascontiguousarray(jobs, dtype=np.int32)
                self._keep.append(j)
                arr[k].jobs, arr[k].njobs = j.ctypes.data, j.size
            self.params.append(p)
        o = native.PhxBatchOptions(tile_rays, blocks_per_sm, period, 1 if autotune else 0, sample_stride,
                                   1 if keep_order else 0, tile_shape, 1 if lane_setup else 0, refill_lanes)
        h = C.c_void_p()
        native.check(L.phx_batch_create(arr, n, C.byref(o), C.byref(h)))
        self._h = h

    def launch(self, stream: int = 0):
        """Replay the captured launch on a CUDA stream (asynchronous)."""
        native.check(native.lib().phx_batch_launch(self._h, stream or None))

    def run(self):
        """Launch on the batch's own stream and wait."""
        native.check(native.lib().phx_batch_run(self._h))

    def result(self, item: int):
        p = self.params[item]
        res = np.zeros((p.img_width, p.img_height, p.nfreqs, 6), dtype=np.float64)
        info = PhxRenderInfo()
        native.check(native.lib().phx_batch_result(self._h, item, res.ctypes.data, C.byref(info)))
        return res, info.as_dict()

    def spectrum(self, item: int) -> np.ndarray:
        """Item's per-frequency totals reduced on the device: rows (I, Q, U, V [Jy], mean tau, mean tauF)."""
        p = self.params[item]
        spec = (native.PhxSpectrum * p.nfreqs)()
        native.check(native.lib().phx_batch_spectrum(self._h, item, spec))
        return spectrum_rows(spec)

    def device_result(self, item: int) -> int:
        ptr = C.c_void_p()
        native.check(native.lib().phx_batch_device_result(self._h, item, C.byref(ptr)))
        return ptr.value

    def tuning(self) -> dict:
        t = native.PhxBatchTuning()
        native.check(native.lib().phx_batch_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def close(self):
        if self._h and self._h.value:
            native.lib().phx_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching render server over resident snapshots (one precision; thread-safe).  Requests are
    admitted by device memory and merged into one running queue kernel while earlier requests are on the GPU."""

    def __init__(self, snapshots, precision="fp32", **opts):
        L = native.lib()
        o = native.PhxServerOptions()
        L.phx_default_server_options(C.byref(o))
        o.precision = native.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        for k, v in opts.items():
            if not hasattr(o, k):
                raise KeyError(f"unknown server option {k}")
            setattr(o, k, v)
        self._snaps = list(snapshots)
        arr = (C.c_void_p * len(self._snaps))(*[sn.handle.value for sn in self._snaps])
        h = C.c_void_p()
        native.check(L.phx_server_create(arr, len(self._snaps), C.byref(o), C.byref(h)))
        self._h = h
        self._params = {}

    def submit(self, snapshot: int, params) -> int:
        rid = C.c_int64()
        native.check(native.lib().phx_server_submit(self._h, snapshot, C.byref(params), C.byref(rid)))
        self._params[rid.value] = params
        return rid.value

    def poll(self, rid: int) -> int:
        st = C.c_int32()
        native.check(native.lib().phx_server_poll(self._h, rid, C.byref(st)))
        return st.value

    def wait(self, rid: int, timeout: float = 0.0) -> int:
        st = C.c_int32()
        native.check(native.lib().phx_server_wait(self._h, rid, timeout, C.byref(st)))
        return st.value

    def result(self, rid: int):
        """(res[img_width, img_height, nfreqs, 6], timing dict) of a finished request; releases it."""
        p = self._params.pop(rid)
        res = np.zeros((p.img_width, p.img_height, p.nfreqs, 6), dtype=np.float64)
        t = native.PhxRequestTiming()
        native.check(native.lib().phx_server_result(self._h, rid, res.ctypes.data, C.byref(t)))
        return res, t.as_dict()

    def stats(self) -> dict:
        st = native.PhxServerStats()
        native.check(native.lib().phx_server_stats(self._h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if self._h and self._h.value:
            native.lib().phx_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def spectrum_rows(spec) -> np.ndarray:
    """PhxSpectrum records as rows (I, Q, U, V [Jy], mean tau, mean tauF)."""
    return np.array([list(r.IQUV) + [r.tau_mean, r.tauF_mean] for r in spec], dtype=np.float64)


def device_spectrum(params, d_res: int, d_spec: int, stream: int = 0):
    """phx_spectrum_async on device pointers: nfreqs PhxSpectrum records (64 bytes each) into d_spec."""
    native.check(native.lib().phx_spectrum_async(C.byref(params), d_res, d_spec, stream or None))


def measure_fp32_peak(repeats: int = 5) -> float:
    """The current GPU's measured FP32 FMA issue rate [TFLOP/s] (phx_measure_fp32_peak)."""
    v = C.c_double()
    native.check(native.lib().phx_measure_fp32_peak(repeats, C.byref(v)))
    return v.value


def pixel_solid_angle(p) -> float:
    """Solid angle of one pixel [sr] (core/geometry/camera.hpp:28-32)."""
    L = G_GRAV * p.mass * M_SUN / C_LIGHT / C_LIGHT
    d = p.distance * KPC
    return (p.fov_x / p.img_width * L / d) * (p.fov_y / p.img_height * L / d)


def flux(res, params) -> np.ndarray:
    """Total Stokes flux [Jy] per frequency (host/io/output.hpp:43-53): pixels with a non-finite I+Q+U+V skipped."""
    r = res.reshape(-1, params.nfreqs, 6)[..., :4]
    ok = np.isfinite(r.sum(axis=-1))
    return np.where(ok[..., None], r, 0.0).sum(axis=0) * pixel_solid_angle(params) * JANSKY
