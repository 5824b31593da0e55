"""Host-side parts of the product that run without a GPU: the C ABI surface, the BHAC reader, the job schedule."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from phoenix_b200 import native
from tests.conftest import ROOT


def test_library_exports_every_declared_symbol(built):
    header = open(os.path.join(ROOT, "include", "phoenix_b200.h")).read()
    declared = set(re.findall(r"\b(phx_[a-z0-9_]+)\s*\(", header))
    assert declared == set(native.EXPORTS)
    L = C.CDLL(built["lib"])
    for name in declared:
        assert hasattr(L, name), name


def test_version_and_errors(built):
    L = native.lib()
    assert b"sm_100a" in L.phx_version()
    h = C.c_void_p()
    rc = L.phx_bhac_read(b"/nonexistent/dump.dat", b"/nonexistent/grid.in", None, 0, C.byref(h))
    assert rc == native.PHX_E_IO
    assert b"cannot open grid file" in L.phx_last_error()


def _schedule_reference_order(W, H):
    """host::jobs::schedule(morton=true) restated: sort i*H+j by the interleave of i (even bits) and j (odd bits)."""
    keys = []
    for i in range(W):
        for j in range(H):
            z = 0
            for b in range(16):
                z |= ((i >> b) & 1) << (2 * b) | ((j >> b) & 1) << (2 * b + 1)
            keys.append((z, i * H + j))
    return np.array([v for _, v in sorted(keys)], dtype=np.int32)


@pytest.mark.parametrize("wh", [(1, 1), (8, 4), (13, 7), (64, 64)])
def test_morton_schedule(built, wh):
    assert np.array_equal(native.schedule_morton(*wh), _schedule_reference_order(*wh))


@pytest.mark.parametrize("shape,tw,th", [("16x2", 16, 2), ("32x1", 32, 1), ("4x8", 4, 8), ("2x16", 2, 16)])
@pytest.mark.parametrize("wh", [(1, 1), (13, 7), (64, 64), (96, 40)])
def test_tile_schedules(built, shape, tw, th, wh):
    """Every pixel once; the image cut into tw x th tiles (j fastest inside one), the tiles in Morton order."""
    W, H = wh
    jobs = native.schedule_tiles(W, H, shape)
    assert np.array_equal(np.sort(jobs), np.arange(W * H))
    nti, ntj = -(-W // tw), -(-H // th)
    want = []
    for t in _schedule_reference_order(nti, ntj):
        ti, tj = divmod(int(t), ntj)
        want += [i * H + j for i in range(ti * tw, min(W, (ti + 1) * tw)) for j in range(tj * th, min(H, (tj + 1) * th))]
    assert np.array_equal(jobs, np.array(want, dtype=np.int32))
    assert np.array_equal(native.schedule_tiles(W, H, "morton"), native.schedule_morton(W, H))
    with pytest.raises(native.PhxError):
        native.schedule_tiles(W, H, 9)


@pytest.mark.parametrize("wh", [(1, 1), (13, 7), (64, 64), (96, 40), (100, 260), (512, 512)])
def test_center_first_schedule(built, wh):
    """4x8 tiles in 32x32-pixel blocks: blocks nearest the image centre first (ties in Morton order), the tiles of a
    block in Morton order, pixels j-fastest inside a tile."""
    W, H = wh
    tw, th, B = 4, 8, 32
    jobs = native.schedule_tiles(W, H, "center4x8")
    assert np.array_equal(np.sort(jobs), np.arange(W * H))
    nti, ntj = -(-W // tw), -(-H // th)
    nbi, nbj = -(-W // B), -(-H // B)

    def d2(b):
        bi, bj = divmod(int(b), nbj)
        ci = 0.5 * (bi * B + min(W, (bi + 1) * B)) - 0.5 * W
        cj = 0.5 * (bj * B + min(H, (bj + 1) * B)) - 0.5 * H
        return ci * ci + cj * cj

    rank = {int(b): r for r, b in enumerate(sorted(_schedule_reference_order(nbi, nbj), key=d2))}  # stable
    tiles = sorted(_schedule_reference_order(nti, ntj),
                   key=lambda t: rank[(int(t) // ntj) * tw // B * nbj + (int(t) % ntj) * th // B])
    want = []
    for t in tiles:
        ti, tj = divmod(int(t), ntj)
        want += [i * H + j for i in range(ti * tw, min(W, (ti + 1) * tw)) for j in range(tj * th, min(H, (tj + 1) * th))]
    assert np.array_equal(jobs, np.array(want, dtype=np.int32))


def test_default_pixel_order(built):
    """Centre-first blocks up to 6 rays per lane of a full grid (148 SMs x 512 lanes here: no GPU), Morton beyond."""
    c, m = native.TILE_SHAPES["center4x8"], native.TILE_SHAPES["morton"]
    lanes = 148 * 512
    for side, want in ((64, c), (512, c), (674, c), (675, m), (1024, m), (2048, m)):
        assert (side * side <= 6 * lanes) == (want == c)
        assert native.default_pixel_order(native.make_params(img=side)) == want, side
    assert native.lib().phx_default_pixel_order(None) == m


def _read_host(dump, grid, spec, f64=True):
    L = native.lib()
    opt = native.PhxReadOptions(3, 1, 1 if spec["sfc"] else 0, spec["nlevels"])
    h = C.c_void_p()
    native.check(L.phx_bhac_read(dump.encode(), grid.encode(), C.byref(opt), native.SNAP_F64_PRIMS if f64 else 0,
                                 C.byref(h)))
    d = native.PhxSnapshotDesc()
    native.check(L.phx_bhac_describe(h, C.byref(d)))
    return h, d


@pytest.mark.parametrize("name", ["cfg1", "small"])
def test_reader_matches_oracle(snapshots, name):
    """Leaf geometry and leaf maps bit-exact; primitives within FP64 rounding of the oracle's decode."""
    from oracle.oracle import Oracle
    dump, grid, spec = snapshots[name]
    o = Oracle(dump, grid, nlevels=spec["nlevels"], sfc=1 if spec["sfc"] else 0)
    t = o.tables()
    h, d = _read_host(dump, grid, spec)
    try:
        n = d.nleafs
        assert n == t["nleafs"] and d.nlevels == t["nlevels"]
        lb = np.ctypeslib.as_array(C.cast(d.lb, C.POINTER(C.c_double)), shape=(n, 3))
        dxc = np.ctypeslib.as_array(C.cast(d.dxc, C.POINTER(C.c_double)), shape=(n, 3))
        assert np.array_equal(lb, t["lb"]) and np.array_equal(dxc, t["dxc"])
        maps = C.cast(d.level_map, C.POINTER(C.c_void_p))
        for L, ref in enumerate(t["level_maps"]):
            m = np.ctypeslib.as_array(C.cast(maps[L], C.POINTER(C.c_int32)), shape=(ref.size,)).reshape(ref.shape)
            assert np.array_equal(m, ref)
        cells = d.nx[0] * d.nx[1] * d.nx[2]
        p64 = np.ctypeslib.as_array(C.cast(d.prim_f64, C.POINTER(C.c_double)), shape=(n, cells, 8))
        p32 = np.ctypeslib.as_array(C.cast(d.prim_f32, C.POINTER(C.c_float)), shape=(n, cells, 8))
        ref = t["prim"]
        scale = np.abs(ref).max(axis=(0, 1))
        assert np.all(np.abs(p64 - ref).max(axis=(0, 1)) <= 1e-13 * scale)
        assert np.array_equal(p32, p64.astype(np.float32))
        sc = t["scalars"]
        assert d.a == sc[0] and d.hslope == sc[1] and d.gam == sc[2]
        assert list(d.x_lo) == list(sc[7:10]) and list(d.x_hi) == list(sc[10:13])
    finally:
        native.lib().phx_bhac_free(h)


def test_reader_rejects_truncated_dump(snapshots, tmp_path):
    dump, grid, spec = snapshots["small"]
    data = open(dump, "rb").read()
    bad = tmp_path / "trunc.dat"
    tail = 40 + 3 * 4 + 4 * 8  # footer, nx[3], neqpar[4]
    bad.write_bytes(data[: len(data) // 3] + data[-tail:])  # trailer intact, body short
    L = native.lib()
    h = C.c_void_p()
    opt = native.PhxReadOptions(3, 1, 0, spec["nlevels"])
    rc = L.phx_bhac_read(str(bad).encode(), grid.encode(), C.byref(opt), 0, C.byref(h))
    assert rc == native.PHX_E_IO
    assert b"short read" in L.phx_last_error() or b"grid mismatch" in L.phx_last_error()


def test_reader_rejects_wrong_sfc(snapshots):
    dump, grid, spec = snapshots["cfg1"]
    L = native.lib()
    h = C.c_void_p()
    opt = native.PhxReadOptions(3, 1, 0, spec["nlevels"])  # the dump is Morton-ordered
    rc = L.phx_bhac_read(dump.encode(), grid.encode(), C.byref(opt), 0, C.byref(h))
    if rc == native.PHX_OK:  # a forest read in the wrong order can still parse; the leaves then differ
        L.phx_bhac_free(h)
    else:
        assert rc == native.PHX_E_IO


def test_make_params_rejects_unknown_keys(built):
    with pytest.raises(KeyError):
        native.make_params(no_such_key=1)
    p = native.make_params(frequencies=[86e9, 230e9], precision="mixed", img=32)
    assert p.nfreqs == 2 and p.precision == native.PREC_MIXED and p.img_width == p.img_height == 32


def test_ctypes_structs_match_the_header(tmp_path):
    """Size and field offsets of every struct the Python binding mirrors, as gcc lays out include/phoenix_b200.h."""
    import subprocess
    structs = {"PhxRenderParams": native.PhxRenderParams, "PhxRenderInfo": native.PhxRenderInfo,
               "PhxSnapshotDesc": native.PhxSnapshotDesc, "PhxReadOptions": native.PhxReadOptions,
               "PhxFreqOut": native.PhxFreqOut, "PhxBatchItem": native.PhxBatchItem,
               "PhxBatchOptions": native.PhxBatchOptions, "PhxBatchTuning": native.PhxBatchTuning,
               "PhxServerOptions": native.PhxServerOptions, "PhxRequestTiming": native.PhxRequestTiming,
               "PhxServerStats": native.PhxServerStats, "PhxSnapshotInfo": native.PhxSnapshotInfo}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "phoenix_b200.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name} {field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for name, cls in structs.items():
        assert got[(name, "size")] == C.sizeof(cls), name
        for field, _ in cls._fields_:
            assert got[(name, field)] == getattr(cls, field).offset, (name, field)
