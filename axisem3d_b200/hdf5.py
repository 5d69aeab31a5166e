"""A small read-only HDF5 reader: the subset that netCDF-4 (the format of Exodus meshes written
by the salvus mesher) uses, with nothing beyond numpy and zlib.

The reference reads its meshes through the NetCDF C library (`NetCDF_Reader::open`,
`readMatrix`, `readString`, `src/shared/io/netcdf/NetCDF_Reader.cpp`). No HDF5 or NetCDF
library is available to this package, so the file format is read directly, following the
published HDF5 File Format Specification (version 3.0):

- superblock versions 0-3 (the root group by its symbol-table entry or object header address);
- object headers version 1 and version 2 ("OHDR"), with continuation blocks;
- groups stored as symbol tables (v1 B-tree of type 0, "SNOD" nodes, local heap) and groups
  stored as compact link messages;
- dataspace (simple and scalar), datatype (fixed-point, floating-point, fixed-length string),
  data layout versions 1-4 (compact, contiguous, chunked through a v1 B-tree of type 1, and
  the version-4 single-chunk index), filter pipeline (deflate, shuffle, fletcher32 skipped);
- attributes (messages 0x000C) with the datatypes above.

Anything else (dense link or attribute storage in fractal heaps, the other version-4 chunk
indices, variable-length data, compound types) raises `NotImplementedError` naming it, only
when the object that needs it is read.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    """A malformed or unsupported HDF5 file."""


class _Dtype:
    """Parsed datatype message: a numpy dtype, or None with `kind` naming what it is."""

    def __init__(self, np_dtype, kind, size):
        self.np = np_dtype
        self.kind = kind
        self.size = size


class Dataset:
    """One dataset: shape, datatype and the messages needed to read its values."""

    def __init__(self, f: "File", name: str, msgs: dict):
        self._f = f
        self.name = name
        self.shape = msgs.get("shape", ())
        self._dtype = msgs.get("dtype")
        self._layout = msgs.get("layout")
        self._filters = msgs.get("filters", [])
        self.attrs = msgs.get("attrs", {})

    @property
    def dtype(self):
        return self._dtype.np if self._dtype is not None else None

    def read(self) -> np.ndarray:
        """All values, as a numpy array of `shape` (C order)."""
        f, dt, lay = self._f, self._dtype, self._layout
        if dt is None or dt.np is None:
            raise NotImplementedError("HDF5 datatype %r of dataset %s" % (getattr(dt, "kind", None), self.name))
        if lay is None:
            raise H5Error("dataset %s has no layout message" % self.name)
        shape = tuple(self.shape)
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * dt.size
        cls = lay["class"]
        if cls == 0:                                           # compact
            raw = lay["data"][:nbytes]
        elif cls == 1:                                         # contiguous
            if lay["addr"] == UNDEF or n == 0:
                raw = bytes(nbytes)                            # never written: fill value 0
            else:
                raw = f._buf[lay["addr"]:lay["addr"] + nbytes]
        elif cls == 2:                                         # chunked
            return self._read_chunked(shape, dt)
        else:
            raise NotImplementedError("HDF5 layout class %d (dataset %s)" % (cls, self.name))
        if len(raw) < nbytes:
            raise H5Error("dataset %s: data runs past the end of the file" % self.name)
        return np.frombuffer(raw, dtype=dt.np, count=n).reshape(shape).copy()

    def _unfilter(self, raw: bytes, mask: int, esize: int) -> bytes:
        for i, flt in reversed(list(enumerate(self._filters))):
            if mask & (1 << i):
                continue
            fid = flt[0]
            if fid == 1:                                       # deflate
                raw = zlib.decompress(raw)
            elif fid == 2:                                     # shuffle
                a = np.frombuffer(raw, dtype=np.uint8)
                ne = len(a) // esize
                head = a[:ne * esize].reshape(esize, ne).T.reshape(-1)
                raw = head.tobytes() + a[ne * esize:].tobytes()
            elif fid == 3:                                     # fletcher32: drop the checksum
                raw = raw[:-4]
            else:
                raise NotImplementedError("HDF5 filter %d (dataset %s)" % (fid, self.name))
        return raw

    def _read_chunked(self, shape, dt) -> np.ndarray:
        lay = self._layout
        cdims = lay["chunk"]
        rank = len(shape)
        out = np.zeros(shape, dtype=dt.np)
        if rank == 0 or 0 in shape:
            return out
        csize = int(np.prod(cdims)) * dt.size
        lay.setdefault("nbytes", csize)
        for offs, size, mask, addr in self._f._chunks(lay, rank):
            raw = self._f._buf[addr:addr + size]
            if self._filters:
                raw = self._unfilter(raw, mask, dt.size)
            if len(raw) < csize:
                raise H5Error("dataset %s: short chunk at %s" % (self.name, offs))
            chunk = np.frombuffer(raw, dtype=dt.np, count=int(np.prod(cdims))).reshape(cdims)
            dst = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
            src = tuple(slice(0, d.stop - d.start) for d in dst)
            out[dst] = chunk[src]
        return out


class File:
    """An HDF5 file opened for reading; `datasets` maps '/'-joined names to `Dataset`s."""

    def __init__(self, path: str):
        with open(path, "rb") as fh:
            self._buf = fh.read()
        b = self._buf
        # the superblock sits at 0, 512, 1024, ...
        base = 0
        while b[base:base + 8] != _SIG:
            base = 512 if base == 0 else 2 * base
            if base >= len(b):
                raise H5Error("%s: no HDF5 signature" % path)
        ver = b[base + 8]
        if ver in (0, 1):
            self.so, self.sl = b[base + 13], b[base + 14]
            o = base + 24 + (4 if ver == 1 else 0)
            self._check_sizes()
            o += 4 * self.so                                   # base, free space, EOF, driver
            _, ohdr = self._u(o, self.so), self._u(o + self.so, self.so)
            root = ohdr
        elif ver in (2, 3):
            self.so, self.sl = b[base + 9], b[base + 10]
            self._check_sizes()
            o = base + 12 + 3 * self.so
            root = self._u(o, self.so)
        else:
            raise NotImplementedError("HDF5 superblock version %d" % ver)
        self.datasets: dict[str, Dataset] = {}
        self.attrs: dict = {}
        self._walk(root, "", set())

    # ---------------- low-level helpers ----------------
    def _check_sizes(self):
        if self.so != 8 or self.sl != 8:
            raise NotImplementedError("HDF5 offset/length sizes %d/%d" % (self.so, self.sl))

    def _u(self, o, n):
        return int.from_bytes(self._buf[o:o + n], "little")

    def _cstr(self, o):
        e = self._buf.index(b"\0", o)
        return self._buf[o:e].decode("utf-8", "replace")

    # ---------------- object headers ----------------
    def _messages(self, addr):
        """(type, data bytes) of every message of the object header at `addr`."""
        b = self._buf
        out = []
        if b[addr:addr + 4] == b"OHDR":
            flags = b[addr + 5]
            o = addr + 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
            nsz = 1 << (flags & 3)
            size0 = self._u(o, nsz)
            o += nsz
            blocks = [(o, o + size0, True)]
            hdr = 4 + (2 if flags & 0x04 else 0)              # type, size, flags [, order]
            while blocks:
                s, e, _ = blocks.pop(0)
                while e - s >= hdr:                            # a shorter tail is a gap
                    mtype, msize, mflags = b[s], self._u(s + 1, 2), b[s + 3]
                    s += hdr
                    data = b[s:s + msize]
                    s += msize
                    if mtype == 0x10:
                        caddr = int.from_bytes(data[0:8], "little")
                        clen = int.from_bytes(data[8:16], "little")
                        if b[caddr:caddr + 4] != b"OCHK":
                            raise H5Error("bad continuation block")
                        blocks.append((caddr + 4, caddr + clen - 4, False))
                    else:
                        out.append((mtype, data, mflags))
            return out
        if b[addr] != 1:
            raise NotImplementedError("HDF5 object header version %d" % b[addr])
        nmsg = self._u(addr + 2, 2)
        hsize = self._u(addr + 8, 4)
        blocks = [(addr + 16, addr + 16 + hsize)]
        count = 0
        while blocks and count < nmsg:
            s, e = blocks.pop(0)
            while s + 8 <= e and count < nmsg:
                mtype, msize, mflags = self._u(s, 2), self._u(s + 2, 2), b[s + 4]
                data = b[s + 8:s + 8 + msize]
                s += 8 + msize
                count += 1
                if mtype == 0x10:
                    blocks.append((int.from_bytes(data[0:8], "little"),
                                   int.from_bytes(data[0:8], "little") + int.from_bytes(data[8:16], "little")))
                else:
                    out.append((mtype, data, mflags))
        return out

    # ---------------- message decoders ----------------
    @staticmethod
    def _dataspace(d):
        ver, rank, flags = d[0], d[1], d[2]
        if ver == 1:
            o = 8
        elif ver == 2:
            if d[3] == 2:                                      # null dataspace
                return None
            o = 4
        else:
            raise NotImplementedError("HDF5 dataspace version %d" % ver)
        return tuple(int.from_bytes(d[o + 8 * i:o + 8 * i + 8], "little") for i in range(rank))

    @staticmethod
    def _datatype(d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = int.from_bytes(d[4:8], "little")
        order = ">" if bits & 1 else "<"
        if cls == 0:                                           # fixed-point
            signed = bool(bits & 0x08)
            return _Dtype(np.dtype("%s%s%d" % (order, "i" if signed else "u", size)), "int", size)
        if cls == 1:                                           # floating-point
            if size not in (2, 4, 8):
                raise NotImplementedError("HDF5 float of %d bytes" % size)
            return _Dtype(np.dtype("%sf%d" % (order, size)), "float", size)
        if cls == 3:                                           # fixed-length string
            return _Dtype(np.dtype("S%d" % size), "string", size)
        if cls == 4:                                           # bitfield
            return _Dtype(np.dtype("%su%d" % (order, size)), "bitfield", size)
        names = {2: "time", 5: "opaque", 6: "compound", 7: "reference", 8: "enum", 9: "variable-length", 10: "array"}
        return _Dtype(None, names.get(cls, "class %d" % cls), size)

    def _layout(self, d, rank):
        ver = d[0]
        if ver in (1, 2):
            nd, cls = d[1], d[2]
            o = 8
            addr = UNDEF
            if cls != 0:
                addr = int.from_bytes(d[o:o + 8], "little")
                o += 8
            dims = [int.from_bytes(d[o + 4 * i:o + 4 * i + 4], "little") for i in range(nd)]
            o += 4 * nd
            if cls == 2:
                return {"class": 2, "index": "btree1", "addr": addr, "chunk": dims[:-1]}
            if cls == 1:
                return {"class": 1, "addr": addr}
            sz = int.from_bytes(d[o:o + 4], "little")
            return {"class": 0, "data": d[o + 4:o + 4 + sz]}
        if ver == 3:
            cls = d[1]
            if cls == 0:
                sz = int.from_bytes(d[2:4], "little")
                return {"class": 0, "data": d[4:4 + sz]}
            if cls == 1:
                return {"class": 1, "addr": int.from_bytes(d[2:10], "little")}
            if cls == 2:
                nd = d[2]
                addr = int.from_bytes(d[3:11], "little")
                dims = [int.from_bytes(d[11 + 4 * i:15 + 4 * i], "little") for i in range(nd)]
                return {"class": 2, "index": "btree1", "addr": addr, "chunk": dims[:-1]}
        if ver == 4:
            cls = d[1]
            if cls == 0:
                sz = int.from_bytes(d[2:4], "little")
                return {"class": 0, "data": d[4:4 + sz]}
            if cls == 1:
                return {"class": 1, "addr": int.from_bytes(d[2:10], "little")}
            if cls == 2:
                flags, nd, w = d[2], d[3], d[4]
                o = 5
                dims = [int.from_bytes(d[o + w * i:o + w * i + w], "little") for i in range(nd)]
                o += w * nd
                itype = d[o]
                o += 1
                if itype == 1:                                 # single chunk
                    lay = {"class": 2, "index": "single", "chunk": dims[:-1]}
                    if flags & 2:
                        lay["fsize"] = int.from_bytes(d[o:o + 8], "little")
                        lay["fmask"] = int.from_bytes(d[o + 8:o + 12], "little")
                        o += 12
                    lay["addr"] = int.from_bytes(d[o:o + 8], "little")
                    return lay
                raise NotImplementedError("HDF5 version-4 chunk index type %d" % itype)
        raise NotImplementedError("HDF5 data layout version %d" % ver)

    @staticmethod
    def _filters(d):
        ver, n = d[0], d[1]
        out = []
        if ver == 1:
            o = 8
            for _ in range(n):
                fid, nlen, flags, nval = struct.unpack_from("<HHHH", d, o)
                o += 8 + nlen
                vals = struct.unpack_from("<%dI" % nval, d, o)
                o += 4 * nval + (4 if nval % 2 else 0)
                out.append((fid, flags, vals))
        else:
            o = 2
            for _ in range(n):
                fid = struct.unpack_from("<H", d, o)[0]
                o += 2
                nlen = 0
                if fid >= 256:
                    nlen = struct.unpack_from("<H", d, o)[0]
                    o += 2
                flags, nval = struct.unpack_from("<HH", d, o)
                o += 4 + nlen
                vals = struct.unpack_from("<%dI" % nval, d, o)
                o += 4 * nval
                out.append((fid, flags, vals))
        return out

    def _attribute(self, d):
        ver = d[0]
        nlen, tlen, slen = struct.unpack_from("<HHH", d, 2)
        o = 8 + (1 if ver == 3 else 0)
        pad = (lambda n: (n + 7) & ~7) if ver == 1 else (lambda n: n)
        name = d[o:o + nlen].split(b"\0")[0].decode("utf-8", "replace")
        o += pad(nlen)
        dt = self._datatype(d[o:o + tlen])
        o += pad(tlen)
        shape = self._dataspace(d[o:o + slen])
        o += pad(slen)
        if dt.np is None or shape is None:
            return name, None
        n = int(np.prod(shape)) if shape else 1
        val = np.frombuffer(d[o:o + n * dt.size], dtype=dt.np, count=n).reshape(shape)
        if dt.kind == "string":
            return name, b"".join(val.reshape(-1).tolist()).split(b"\0")[0].decode("utf-8", "replace")
        return name, val.copy()

    # ---------------- groups ----------------
    def _walk(self, addr, prefix, seen):
        if addr in seen:
            return
        seen.add(addr)
        msgs = self._messages(addr)
        info = {"attrs": {}}
        links = []
        is_group = False
        for mtype, d, _ in msgs:
            if mtype == 0x01:
                info["shape"] = self._dataspace(d)
            elif mtype == 0x03:
                info["dtype"] = self._datatype(d)
            elif mtype == 0x08:
                info["layout_raw"] = d
            elif mtype == 0x0B:
                info["filters"] = self._filters(d)
            elif mtype == 0x0C:
                k, v = self._attribute(d)
                info["attrs"][k] = v
            elif mtype == 0x11:
                is_group = True
                links += self._symbol_table(int.from_bytes(d[0:8], "little"), int.from_bytes(d[8:16], "little"))
            elif mtype == 0x06:
                is_group = True
                links.append(self._link(d))
            elif mtype == 0x02:
                is_group = True
                fheap = int.from_bytes(d[2 + (8 if d[1] & 1 else 0):][:8], "little")
                if fheap != UNDEF:
                    raise NotImplementedError("HDF5 dense link storage (group %s)" % (prefix or "/"))
        if is_group:
            if not prefix:
                self.attrs = info["attrs"]
            for name, child in links:
                if child is not None:
                    self._walk(child, prefix + "/" + name if prefix else name, seen)
            return
        if "layout_raw" in info:
            info["layout"] = self._layout(info.pop("layout_raw"), len(info.get("shape") or ()))
            self.datasets[prefix] = Dataset(self, prefix, info)

    def _link(self, d):
        flags = d[1]
        o = 2
        ltype = 0
        if flags & 0x08:
            ltype = d[o]
            o += 1
        if flags & 0x04:
            o += 8
        if flags & 0x10:
            o += 1
        w = 1 << (flags & 3)
        nlen = int.from_bytes(d[o:o + w], "little")
        o += w
        name = d[o:o + nlen].decode("utf-8", "replace")
        o += nlen
        if ltype != 0:
            return name, None                                  # soft / external links are not followed
        return name, int.from_bytes(d[o:o + 8], "little")

    def _symbol_table(self, btree, heap):
        b = self._buf
        if b[heap:heap + 4] != b"HEAP":
            raise H5Error("bad local heap")
        data = int.from_bytes(b[heap + 24:heap + 32], "little")
        out = []

        def node(addr):
            if b[addr:addr + 4] == b"TREE":
                level, used = b[addr + 5], self._u(addr + 6, 2)
                o = addr + 24 + 8                              # first key
                for _ in range(used):
                    node(self._u(o, 8))
                    o += 16
            elif b[addr:addr + 4] == b"SNOD":
                nsym = self._u(addr + 6, 2)
                o = addr + 8
                for _ in range(nsym):
                    noff, ohdr = self._u(o, 8), self._u(o + 8, 8)
                    out.append((self._cstr(data + noff), ohdr))
                    o += 40
            else:
                raise H5Error("bad group B-tree node")

        node(btree)
        return out

    # ---------------- chunk indices ----------------
    def _chunks(self, lay, rank):
        """(offsets, stored size, filter mask, address) of every stored chunk."""
        if lay["index"] == "single":
            # an unfiltered single chunk is stored whole; its size is the chunk's
            size = lay.get("fsize", lay.get("nbytes", 0))
            yield (0,) * rank, size, lay.get("fmask", 0), lay["addr"]
            return
        b = self._buf
        if lay["addr"] == UNDEF:
            return
        stack = [lay["addr"]]
        ksize = 8 + 8 * (rank + 1)
        while stack:
            addr = stack.pop()
            if b[addr:addr + 4] != b"TREE" or b[addr + 4] != 1:
                raise H5Error("bad chunk B-tree node")
            level, used = b[addr + 5], self._u(addr + 6, 2)
            o = addr + 24
            for _ in range(used):
                size, mask = self._u(o, 4), self._u(o + 4, 4)
                offs = tuple(self._u(o + 8 + 8 * i, 8) for i in range(rank))
                child = self._u(o + ksize, 8)
                if level > 0:
                    stack.append(child)
                else:
                    yield offs, size, mask, child
                o += ksize + 8


def open_file(path: str) -> File:
    return File(path)
