"""Reader for the JLD2 impurity files that ``setup_LDGA`` and ``readConfig`` load
(runHelpers.jl:87-112, IO.jl:68-88; ``jldopen(f, "r")`` with ``f["key"]``).

JLD2 (JLD2.jl, here files written by version 0.1.1 of its format) stores data in an HDF5 container:
a 512-byte text preamble, an HDF5 version-2 superblock whose addresses are relative to a base
address of 512, version-2 object headers ("OHDR" with Fletcher-style checksums that this reader does
not verify), groups as link messages, and datasets with a dataspace, a datatype (plain or a shared
reference to a committed datatype in the ``_types`` group) and a compact or contiguous layout.
This module implements that subset of the published HDF5 file format specification in NumPy;
it needs no HDF5 library (none is installed).

Supported values: scalars and N-d arrays of IEEE floats, integers and Bool, complex numbers (the
committed ``Base.Complex{T}`` compound of ``re``/``im``), and plain compounds of those.  Julia arrays
are column-major: an HDF5 dataspace lists the dimensions in reverse, so an array of HDF5 shape
(d_n, ..., d_1) is returned as a Fortran-ordered array of shape (d_1, ..., d_n), exactly what Julia
sees.  Anything else (strings, references, chunked or compressed data) raises
``NotImplementedError`` naming the key.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

_SIG = b"\x89HDF\r\n\x1a\n"
_UNDEF = 0xFFFFFFFFFFFFFFFF


@dataclass
class _Msg:
    type: int
    flags: int
    data: bytes


@dataclass
class _Header:
    msgs: list = field(default_factory=list)


class JLD2File:
    """A read-only view of a JLD2 file: ``keys()``, ``haskey``, ``f["name"]`` (root datasets)."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self._d = fh.read()
        d = self._d
        pos = d.find(_SIG, 0, 4096)
        if pos < 0:
            raise ValueError(f"{path}: no HDF5 superblock (not a JLD2 file)")
        ver = d[pos + 8]
        if ver not in (2, 3):
            raise NotImplementedError(f"{path}: HDF5 superblock version {ver}")
        so, sl = d[pos + 9], d[pos + 10]
        if so != 8 or sl != 8:
            raise NotImplementedError(f"{path}: offsets of {so} / lengths of {sl} bytes")
        base, _ext, _eof, root = struct.unpack_from("<4Q", d, pos + 12)
        self._base = base
        self._headers: dict[int, _Header] = {}
        self._links = self._group_links(root)

    # ------------------------------------------------------------------ object headers
    def _header(self, addr: int) -> _Header:
        if addr in self._headers:
            return self._headers[addr]
        h = _Header()
        self._read_chunk(self._base + addr, h, first=True)
        self._headers[addr] = h
        return h

    def _read_chunk(self, off: int, h: _Header, first: bool, length: int = 0) -> None:
        d = self._d
        if first:
            if d[off:off + 4] != b"OHDR":
                raise NotImplementedError(f"object header at {off}: not a version-2 header")
            flags = d[off + 5]
            p = off + 6
            if flags & 0x20:
                p += 16                                   # access/modification/change/birth times
            if flags & 0x10:
                p += 4                                    # attribute phase change values
            nsz = 1 << (flags & 3)
            size = int.from_bytes(d[p:p + nsz], "little")
            p += nsz
            end = p + size
            self._hflags = flags
        else:
            if d[off:off + 4] != b"OCHK":
                raise NotImplementedError(f"continuation block at {off}: bad signature")
            p = off + 4
            end = off + length - 4                        # checksum at the end
        flags = self._hflags
        while p + 4 <= end:
            mtype = d[p]
            msize = struct.unpack_from("<H", d, p + 1)[0]
            mflags = d[p + 3]
            p += 4
            if flags & 0x04:
                p += 2                                    # creation order
            data = d[p:p + msize]
            p += msize
            if mtype == 0x10:                             # continuation
                caddr, clen = struct.unpack_from("<QQ", data, 0)
                self._read_chunk(self._base + caddr, h, first=False, length=clen)
            elif mtype != 0:
                h.msgs.append(_Msg(mtype, mflags, data))

    # ------------------------------------------------------------------ groups
    def _group_links(self, addr: int) -> dict[str, int]:
        links: dict[str, int] = {}
        for m in self._header(addr).msgs:
            if m.type == 0x06:
                name, target = self._link(m.data)
                if target is not None:
                    links[name] = target
            elif m.type == 0x11:
                raise NotImplementedError("version-1 (symbol table) groups")
        return links

    @staticmethod
    def _link(b: bytes):
        p = 0
        if b[p] != 1:
            raise NotImplementedError(f"link message version {b[p]}")
        flags = b[p + 1]
        p += 2
        ltype = 0
        if flags & 0x08:
            ltype = b[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        nsz = 1 << (flags & 3)
        n = int.from_bytes(b[p:p + nsz], "little")
        p += nsz
        name = b[p:p + n].decode("utf-8")
        p += n
        if ltype != 0:
            return name, None                             # soft / external links are not followed
        return name, struct.unpack_from("<Q", b, p)[0]

    def keys(self) -> list[str]:
        return [k for k in self._links if not k.startswith("_")]

    def haskey(self, key: str) -> bool:
        return key in self._links

    __contains__ = haskey

    def __getitem__(self, key: str):
        if key not in self._links:
            raise KeyError(key)
        try:
            return self._dataset(self._links[key])
        except NotImplementedError as e:
            raise NotImplementedError(f"{key}: {e}") from None

    # ------------------------------------------------------------------ datasets
    def _dataset(self, addr: int):
        space = dtype = layout = None
        for m in self._header(addr).msgs:
            if m.type == 0x01:
                space = self._dataspace(m.data)
            elif m.type == 0x03:
                dtype = self._shared_or_inline_type(m)
            elif m.type == 0x08:
                layout = m.data
        if dtype is None or layout is None:
            raise NotImplementedError("object without datatype or layout (a group or an empty value)")
        if space is None:
            space = ()
        if space == "null":
            return None
        raw = self._layout_bytes(layout, int(np.prod(space, dtype=np.int64)) * dtype.itemsize)
        arr = np.frombuffer(raw, dtype=dtype, count=int(np.prod(space, dtype=np.int64)))
        arr = _finish(arr)
        if space == ():
            return arr[0].item() if arr.dtype.kind in "fiucb" else arr[0]
        # HDF5 lists Julia's dimensions slowest first: reverse them for the Fortran view
        return np.asfortranarray(arr.reshape(space).transpose())

    @staticmethod
    def _dataspace(b: bytes):
        ver, rank, flags = b[0], b[1], b[2]
        if ver == 1:
            p = 8
            stype = 1 if rank > 0 else 0
        elif ver == 2:
            stype = b[3]
            p = 4
        else:
            raise NotImplementedError(f"dataspace version {ver}")
        if stype == 2:
            return "null"
        return tuple(struct.unpack_from(f"<{rank}Q", b, p)) if rank else ()

    def _shared_or_inline_type(self, m: _Msg) -> np.dtype:
        if m.flags & 0x02:                                # shared: a committed datatype
            ver, stype = m.data[0], m.data[1]
            if ver == 3 and stype == 2:
                target = struct.unpack_from("<Q", m.data, 2)[0]
            elif ver in (1, 2):
                target = struct.unpack_from("<Q", m.data, 8 if ver == 1 else 2)[0]
            else:
                raise NotImplementedError(f"shared message version {ver} type {stype}")
            for tm in self._header(target).msgs:
                if tm.type == 0x03:
                    return _datatype(tm.data)[0]
            raise NotImplementedError("committed datatype without a datatype message")
        return _datatype(m.data)[0]

    def _layout_bytes(self, b: bytes, nbytes: int) -> bytes:
        ver, cls = b[0], b[1]
        if ver not in (3, 4):
            raise NotImplementedError(f"data layout version {ver}")
        if cls == 0:                                      # compact: the data sits in the header
            size = struct.unpack_from("<H", b, 2)[0]
            return b[4:4 + size][:nbytes]
        if cls == 1:                                      # contiguous
            addr, size = struct.unpack_from("<QQ", b, 2)
            if addr == _UNDEF:
                return bytes(nbytes)
            off = self._base + addr
            return self._d[off:off + min(size, nbytes)]
        raise NotImplementedError("chunked (possibly compressed) data layout")


def _datatype(b: bytes, p: int = 0):
    """Decode an HDF5 datatype message at ``b[p:]``; returns (numpy dtype, bytes consumed)."""
    cv = b[p]
    cls, ver = cv & 0x0F, cv >> 4
    bits = b[p + 1] | (b[p + 2] << 8) | (b[p + 3] << 16)
    size = struct.unpack_from("<I", b, p + 4)[0]
    q = p + 8
    if bits & 1 and cls in (0, 1):
        raise NotImplementedError("big-endian numbers")
    if cls == 0:                                          # fixed-point
        signed = bool(bits & 0x08)
        dt = np.dtype(("<i" if signed else "<u") + str(size))
        if size == 1 and not signed:
            dt = np.dtype("u1")
        return dt, q + 4 - p
    if cls == 1:                                          # IEEE float
        if size not in (2, 4, 8):
            raise NotImplementedError(f"{size}-byte float")
        return np.dtype("<f" + str(size)), q + 12 - p
    if cls == 6:                                          # compound
        if ver < 3:
            raise NotImplementedError(f"compound datatype version {ver}")
        nmem = bits & 0xFFFF
        names, formats, offsets = [], [], []
        for _ in range(nmem):
            e = b.index(b"\x00", q)
            name = b[q:e].decode("utf-8")
            q = e + 1
            osz = 1 if size < 256 else 2 if size < 65536 else 3 if size < (1 << 24) else 4
            off = int.from_bytes(b[q:q + osz], "little")
            q += osz
            mdt, used = _datatype(b, q)
            q += used
            names.append(name)
            formats.append(mdt)
            offsets.append(off)
        dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size})
        return dt, q - p
    raise NotImplementedError(f"HDF5 datatype class {cls}")


def _finish(arr: np.ndarray) -> np.ndarray:
    """Complex compounds (re, im) become complex arrays; other compounds stay structured."""
    n = arr.dtype.names
    if n == ("re", "im"):
        f = arr.dtype.fields
        if f["re"][0] == f["im"][0] and f["re"][0].kind == "f":
            out = np.empty(arr.shape, dtype=np.result_type(f["re"][0], np.complex64))
            out.real = arr["re"]
            out.imag = arr["im"]
            return out
    return np.array(arr)


def jldopen(path, mode: str = "r") -> JLD2File:
    """``jldopen(path, "r")`` for reading; writing is not supported."""
    if mode != "r":
        raise NotImplementedError("only reading JLD2 files is supported")
    return JLD2File(path)
