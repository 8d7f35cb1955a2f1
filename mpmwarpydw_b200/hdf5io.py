"""Reading the reference's HDF5 domain files without h5py.

The reference's driver reads its input domain with h5py (runMPMYDW.py:20-23,
69-82, 195-275): datasets ``x`` (3, N), ``particle_volume`` (N) and optional
per-particle material arrays in the root group, written by h5py with its
defaults (exampleDomains/createInputHDF5.py).  Those files use the original
HDF5 layout, which this module reads:

  * superblock version 0 or 1 (any offset / length size);
  * the root group as a symbol table: a version-1 B-tree of group nodes over
    symbol-table nodes (SNOD), names in a local heap (HEAP);
  * version-1 object headers (with continuation blocks) holding the
    dataspace, datatype and data-layout messages of each dataset;
  * contiguous or compact storage of fixed-point and IEEE floating-point
    data, either byte order.

Chunked or filtered (compressed) datasets, version-2 superblocks and
link-message groups raise ``NotImplementedError`` with the dataset's name.
The layout follows the published HDF5 File Format Specification, version 2.
"""
from __future__ import annotations

import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"


class HDF5File:
    """Root-group datasets of an HDF5 file: ``keys()``, ``f[name]`` (numpy)."""

    def __init__(self, path):
        self.path = path
        with open(path, "rb") as fh:
            self.buf = fh.read()
        b = self.buf
        if b[:8] != SIGNATURE:
            raise ValueError(f"{path}: not an HDF5 file")
        version = b[8]
        if version not in (0, 1):
            raise NotImplementedError(f"{path}: superblock version {version} (0 and 1 are read)")
        self.so, self.sl = b[13], b[14]
        pos = 24 + (4 if version == 1 else 0)
        self.base = self._addr(pos)
        pos += 4 * self.so                      # base, free-space, end-of-file, driver addresses
        root = self._symbol_entry(pos)
        if root["cache_type"] != 1:
            raise NotImplementedError(f"{path}: the root group is not a symbol-table group")
        self.datasets = {}
        heap = self._local_heap(root["heap"])
        for name, ohdr in self._group_entries(root["btree"], heap):
            self.datasets[name] = ohdr

    # ---- primitive readers ------------------------------------------------
    def _uint(self, pos, size):
        return int.from_bytes(self.buf[pos:pos + size], "little")

    def _addr(self, pos):
        return self._uint(pos, self.so)

    def _symbol_entry(self, pos):
        so = self.so
        e = {"name_off": self._uint(pos, so), "ohdr": self._addr(pos + so), "cache_type": self._uint(pos + 2 * so, 4)}
        scratch = pos + 2 * so + 8
        e["btree"], e["heap"] = self._addr(scratch), self._addr(scratch + so)
        e["size"] = 2 * so + 24
        return e

    def _local_heap(self, addr):
        if self.buf[addr:addr + 4] != b"HEAP":
            raise ValueError(f"{self.path}: bad local heap at {addr}")
        p = addr + 8 + 2 * self.sl
        return self.base + self._addr(p)

    def _name(self, heap_data, off):
        s = heap_data + off
        e = self.buf.index(b"\0", s)
        return self.buf[s:e].decode()

    def _group_entries(self, btree, heap_data):
        b = self.buf
        if b[btree:btree + 4] != b"TREE":
            raise ValueError(f"{self.path}: bad B-tree node at {btree}")
        ntype, level, used = b[btree + 4], b[btree + 5], self._uint(btree + 6, 2)
        if ntype != 0:
            raise ValueError(f"{self.path}: B-tree node type {ntype} in a group")
        pos = btree + 8 + 2 * self.so          # signature, type, level, entries, two siblings
        out = []
        for k in range(used):
            pos += self.sl                      # key k (a heap offset)
            child = self.base + self._addr(pos)
            pos += self.so
            if level > 0:
                out += self._group_entries(child, heap_data)
                continue
            if b[child:child + 4] != b"SNOD":
                raise ValueError(f"{self.path}: bad symbol-table node at {child}")
            nsym = self._uint(child + 6, 2)
            q = child + 8
            for _ in range(nsym):
                e = self._symbol_entry(q)
                out.append((self._name(heap_data, e["name_off"]), self.base + e["ohdr"]))
                q += e["size"]
        return out

    def _messages(self, addr):
        b = self.buf
        if b[addr] != 1:
            raise NotImplementedError(f"{self.path}: object header version {b[addr]} (1 is read)")
        nmsg = self._uint(addr + 2, 2)
        size = self._uint(addr + 8, 4)
        blocks = [(addr + 16, size)]
        msgs = []
        while blocks and len(msgs) < nmsg:
            start, length = blocks.pop(0)
            p = start
            while p + 8 <= start + length and len(msgs) < nmsg:
                mtype, msize = self._uint(p, 2), self._uint(p + 2, 2)
                data = p + 8
                if mtype == 0x10:               # continuation
                    blocks.append((self.base + self._addr(data), self._uint(data + self.so, self.sl)))
                msgs.append((mtype, data, msize))
                p = data + msize
        return msgs

    # ---- datasets ---------------------------------------------------------
    def keys(self):
        return list(self.datasets)

    def __contains__(self, name):
        return name in self.datasets

    def __getitem__(self, name):
        if name not in self.datasets:
            raise KeyError(name)
        shape, dtype, layout = None, None, None
        for mtype, p, size in self._messages(self.datasets[name]):
            if mtype == 0x1:
                shape = self._dataspace(p)
            elif mtype == 0x3:
                dtype = self._datatype(p, name)
            elif mtype == 0x8:
                layout = (p, size)
            elif mtype == 0xB:
                raise NotImplementedError(f"{self.path}: dataset {name} is filtered (compressed)")
        if shape is None or dtype is None or layout is None:
            raise ValueError(f"{self.path}: dataset {name} lacks a dataspace, datatype or layout message")
        count = int(np.prod(shape)) if shape else 1
        raw = self._layout_bytes(layout[0], name, count * dtype.itemsize)
        return np.frombuffer(raw, dtype=dtype, count=count).reshape(shape).copy()

    def _dataspace(self, p):
        b = self.buf
        version, ndim = b[p], b[p + 1]
        if version == 1:
            q = p + 8
        elif version == 2:
            q = p + 4
        else:
            raise NotImplementedError(f"{self.path}: dataspace version {version}")
        return tuple(self._uint(q + i * self.sl, self.sl) for i in range(ndim))

    def _datatype(self, p, name):
        b = self.buf
        cls = b[p] & 0x0F
        bits = b[p + 1]
        size = self._uint(p + 4, 4)
        order = ">" if bits & 1 else "<"
        if cls == 0:                            # fixed point
            kind = "i" if bits & 0x08 else "u"
            if size not in (1, 2, 4, 8):
                raise NotImplementedError(f"{self.path}: {name}: {size}-byte integers")
            return np.dtype(f"{order}{kind}{size}")
        if cls == 1:                            # IEEE floating point
            if size not in (2, 4, 8):
                raise NotImplementedError(f"{self.path}: {name}: {size}-byte floats")
            return np.dtype(f"{order}f{size}")
        raise NotImplementedError(f"{self.path}: {name}: datatype class {cls}")

    def _layout_bytes(self, p, name, nbytes):
        b = self.buf
        version = b[p]
        if version == 3:
            cls = b[p + 1]
            if cls == 0:                        # compact
                size = self._uint(p + 2, 2)
                return b[p + 4:p + 4 + size]
            if cls == 1:                        # contiguous
                addr = self._addr(p + 2)
                if addr == (1 << (8 * self.so)) - 1:
                    return bytes(nbytes)        # never written: fill value 0
                return b[self.base + addr:self.base + addr + nbytes]
            raise NotImplementedError(f"{self.path}: dataset {name} is chunked")
        if version in (1, 2):
            ndim, cls = b[p + 1], b[p + 2]
            q = p + 8
            if cls == 1:
                addr = self._addr(q)
                return b[self.base + addr:self.base + addr + nbytes]
            if cls == 0:
                q += 4 * ndim
                size = self._uint(q, 4)
                return b[q + 4:q + 4 + size]
            raise NotImplementedError(f"{self.path}: dataset {name} is chunked")
        raise NotImplementedError(f"{self.path}: data layout version {version}")


def read_domain(path):
    """The reference's domain datasets of an HDF5 file as a dict of arrays."""
    f = HDF5File(path)
    return {k: f[k] for k in f.keys()}
