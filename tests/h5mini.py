"""Minimal HDF5 reader for the tests (no HDF5 library exists on this machine).

Follows the HDF5 File Format Specification (version 3.0) for what a classic-format file holds: superblock version 0
or 1 (possibly behind a user block), groups stored as symbol tables (v1 B-tree of symbol-table nodes plus a local
heap), version-1 object headers, and datasets with a dataspace, a datatype and a contiguous or compact layout.  It
reads the datasets of the root group.  Checked against a file written by libhdf5 (scipy's MATLAB 7.3 test data).
"""
from __future__ import annotations

import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    pass


class H5File:
    def __init__(self, path_or_bytes):
        self.b = open(path_or_bytes, "rb").read() if isinstance(path_or_bytes, str) else bytes(path_or_bytes)
        off = 0
        while True:  # the superblock sits at 0, 512, 1024, 2048, ...
            if self.b[off:off + 8] == SIG:
                break
            off = 512 if off == 0 else off * 2
            if off >= len(self.b):
                raise H5Error("no HDF5 signature")
        self.base = off
        sb = self.b[off:]
        self.sb_version = sb[8]
        if self.sb_version not in (0, 1):
            raise H5Error(f"superblock version {self.sb_version} not supported")
        self.so, self.sl = sb[13], sb[14]  # sizes of offsets and lengths
        if (self.so, self.sl) != (8, 8):
            raise H5Error("only 8-byte offsets and lengths are supported")
        self.leaf_k, self.internal_k = struct.unpack_from("<HH", sb, 16)
        p = 24 if self.sb_version == 0 else 28
        base_addr, _fs, eof, _drv = struct.unpack_from("<4Q", sb, p)
        if base_addr != self.base:
            raise H5Error(f"base address {base_addr} is not the superblock offset {self.base}")
        self.eof = eof
        root = p + 32
        _name_off, self.root_header, cache_type = struct.unpack_from("<QQI", sb, root)
        self.root_btree = self.root_heap = None
        if cache_type == 1:
            self.root_btree, self.root_heap = struct.unpack_from("<QQ", sb, root + 24)
        # libhdf5 records the end-of-file address as an absolute offset (it equals the file size even behind a user
        # block); a file without a user block has both readings agree
        if eof != len(self.b):
            raise H5Error(f"end-of-file address {eof} does not match the file size {len(self.b)}")

    # addresses are relative to the superblock
    def at(self, addr, n):
        a = self.base + addr
        if addr == UNDEF or a + n > len(self.b):
            raise H5Error(f"address {addr:#x} (+{n}) outside the file")
        return self.b[a:a + n]

    def heap(self, addr):
        h = self.at(addr, 32)
        if h[:4] != b"HEAP" or h[4] != 0:
            raise H5Error("bad local heap")
        size, _free, data = struct.unpack_from("<QQQ", h, 8)
        return self.at(data, size)

    def messages(self, addr):
        h = self.at(addr, 16)
        version, _r, nmsg, _refc, size = struct.unpack_from("<BBHII", h, 0)
        if version != 1:
            raise H5Error(f"object header version {version} not supported")
        body = self.at(addr + 16, size)
        out, p = [], 0
        while len(out) < nmsg and p + 8 <= len(body):
            mtype, msize, flags = struct.unpack_from("<HHB", body, p)
            out.append((mtype, body[p + 8:p + 8 + msize], flags))
            p += 8 + msize
            if msize % 8:
                raise H5Error("message size not a multiple of 8")
        if len(out) != nmsg:
            raise H5Error("header message count mismatch")
        return out

    def group_entries(self, btree_addr, heap_addr):
        names = self.heap(heap_addr)
        entries = []

        def walk(addr):
            node = self.at(addr, 24)
            if node[:4] != b"TREE" or node[4] != 0:
                raise H5Error("bad group B-tree node")
            level, used = node[5], struct.unpack_from("<H", node, 6)[0]
            body = self.at(addr + 24, (2 * self.internal_k + 1) * 8 + 2 * self.internal_k * 8)
            for i in range(used):
                child = struct.unpack_from("<Q", body, 8 + 16 * i)[0]
                if level > 0:
                    walk(child)
                else:
                    snod = self.at(child, 8 + 2 * self.leaf_k * 40)
                    if snod[:4] != b"SNOD" or snod[4] != 1:
                        raise H5Error("bad symbol table node")
                    n = struct.unpack_from("<H", snod, 6)[0]
                    for e in range(n):
                        name_off, hdr = struct.unpack_from("<QQ", snod, 8 + 40 * e)
                        end = names.index(b"\0", name_off)
                        entries.append((names[name_off:end].decode(), hdr))

        walk(btree_addr)
        return entries

    def root_group(self):
        btree, heap = self.root_btree, self.root_heap
        if btree is None:
            for mtype, data, _ in self.messages(self.root_header):
                if mtype == 0x11:
                    btree, heap = struct.unpack_from("<QQ", data, 0)
        if btree is None:
            raise H5Error("root group has no symbol table")
        return self.group_entries(btree, heap)

    def dataset(self, hdr):
        shape = dtype = layout = None
        for mtype, data, _ in self.messages(hdr):
            if mtype == 0x1:  # dataspace
                version, ndims, flags = data[0], data[1], data[2]
                off = 8 if version == 1 else 4
                shape = struct.unpack_from("<%dQ" % ndims, data, off)
            elif mtype == 0x3:  # datatype
                cls, version = data[0] & 0x0F, data[0] >> 4
                bits = data[1] | (data[2] << 8) | (data[3] << 16)
                size = struct.unpack_from("<I", data, 4)[0]
                order = ">" if bits & 1 else "<"
                if cls == 1:
                    dtype = np.dtype(order + "f%d" % size)
                elif cls == 0:
                    dtype = np.dtype(order + ("i" if bits & 8 else "u") + "%d" % size)
                else:
                    dtype = ("class", cls, version)
            elif mtype == 0x8:  # layout
                version = data[0]
                if version in (1, 2):  # dimensionality, class, 5 reserved bytes, address, 4-byte dimensions
                    ndims, lclass = data[1], data[2]
                    if lclass != 1:
                        raise H5Error("only contiguous version-1/2 layouts are supported")
                    addr = struct.unpack_from("<Q", data, 8)[0]
                    dims = struct.unpack_from("<%dI" % ndims, data, 16)
                    layout = ("contiguous", addr, None, dims)
                    continue
                lclass = data[1]
                if version != 3:
                    raise H5Error("layout message version %d" % version)
                if lclass == 1:
                    addr, size = struct.unpack_from("<QQ", data, 2)
                    layout = ("contiguous", addr, size)
                elif lclass == 0:
                    size = struct.unpack_from("<H", data, 2)[0]
                    layout = ("compact", data[4:4 + size])
                else:
                    layout = ("chunked",)
        return shape, dtype, layout

    def read(self, name):
        entries = dict(self.root_group())
        shape, dtype, layout = self.dataset(entries[name])
        if not isinstance(dtype, np.dtype):
            raise H5Error(f"{name}: unsupported datatype {dtype}")
        n = int(np.prod(shape)) * dtype.itemsize
        if layout[0] == "contiguous":
            if layout[2] is not None and layout[2] != n:
                raise H5Error(f"{name}: layout size {layout[2]} != {n}")
            raw = self.at(layout[1], n)
        elif layout[0] == "compact":
            raw = layout[1]
        else:
            raise H5Error(f"{name}: chunked layout not supported")
        return np.frombuffer(raw, dtype=dtype).reshape(shape)
