"""A NetCDF classic writer (64-bit offset, "CDF-2") whose variables are written in place.

The element-wise output files (core/output/element-wise/io/ElementIO_NetCDF.cpp) hold arrays
[element, na, GLL, channel, time] that grow along their last axis while the time loop runs.
The whole header (dimensions and variables, all of fixed size) is written when the file is
created, every variable gets its place in the file, and each block of records is then
stored through a memory map of its variable, so only one block is ever held on the host.
The layout follows the NetCDF classic format specification (big-endian, names and data
padded to four bytes, `begin` as a 64-bit offset); the NetCDF library and scipy read it.
"""
from __future__ import annotations

import struct

import numpy as np

_NC_DIMENSION, _NC_VARIABLE = 0x0A, 0x0B
_TYPES = {np.dtype("S1"): (2, 1), np.dtype(np.int32): (4, 4), np.dtype(np.float32): (5, 4),
          np.dtype(np.float64): (6, 8)}
_BIG = {2: "S1", 4: ">i4", 5: ">f4", 6: ">f8"}


def _name(s):
    b = s.encode()
    return struct.pack(">i", len(b)) + b + b"\0" * (-len(b) % 4)


class NC3File:
    """dims: list of (name, length); variables added with add(name, dims, dtype) before
    create(); after create() each variable is a writable memory map (var(name))."""

    def __init__(self, path):
        self.path = path
        self.dims = []
        self.vars = []
        self._maps = {}

    def dim(self, name, length):
        for k, (n, ln) in enumerate(self.dims):
            if n == name:
                if ln != length:
                    raise ValueError("dimension %s defined with two lengths" % name)
                return k
        self.dims.append((name, int(length)))
        return len(self.dims) - 1

    def add(self, name, dims, dtype):
        """dims: list of (name, length)."""
        ids = [self.dim(n, ln) for n, ln in dims]
        self.vars.append((name, ids, np.dtype(dtype)))

    def create(self):
        shapes = [tuple(self.dims[i][1] for i in ids) for _, ids, _ in self.vars]
        sizes = []
        for (name, ids, dt), shp in zip(self.vars, shapes):
            n = int(np.prod(shp, dtype=np.int64)) * _TYPES[dt][1]
            sizes.append(n + (-n % 4))

        def header(begins):
            h = [b"CDF\x02", struct.pack(">i", 0)]
            if self.dims:
                h.append(struct.pack(">ii", _NC_DIMENSION, len(self.dims)))
                for n, ln in self.dims:
                    h += [_name(n), struct.pack(">i", ln)]
            else:
                h.append(struct.pack(">ii", 0, 0))
            h.append(struct.pack(">ii", 0, 0))                      # no global attributes
            if self.vars:
                h.append(struct.pack(">ii", _NC_VARIABLE, len(self.vars)))
                for (name, ids, dt), sz, b in zip(self.vars, sizes, begins):
                    h += [_name(name), struct.pack(">i", len(ids))]
                    h += [struct.pack(">i", i) for i in ids]
                    h.append(struct.pack(">ii", 0, 0))              # no variable attributes
                    h.append(struct.pack(">iIq", _TYPES[dt][0], min(sz, 0xFFFFFFFF), b))
            else:
                h.append(struct.pack(">ii", 0, 0))
            return b"".join(h)

        hlen = len(header([0] * len(self.vars)))
        begins, pos = [], hlen
        for sz in sizes:
            begins.append(pos)
            pos += sz
        with open(self.path, "wb") as f:
            f.write(header(begins))
            f.truncate(pos)
        for (name, ids, dt), shp, b in zip(self.vars, shapes, begins):
            if int(np.prod(shp, dtype=np.int64)) == 0:
                self._maps[name] = np.zeros(shp, _BIG[_TYPES[dt][0]])
            else:
                self._maps[name] = np.memmap(self.path, dtype=_BIG[_TYPES[dt][0]], mode="r+", offset=b,
                                             shape=shp)

    def var(self, name):
        return self._maps[name]

    def flush(self):
        for m in self._maps.values():
            if isinstance(m, np.memmap):
                m.flush()

    def close(self):
        self.flush()
        self._maps.clear()
