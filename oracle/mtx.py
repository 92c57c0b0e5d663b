"""Pure-Python restatement of the reference's MatrixMarket and binary matrix
I/O (core/base/mtx_io.cpp) — TEST INFRASTRUCTURE ONLY.

The checker for the library's b2s_mtx_* entry points: tests compare both
against the known answers of the reference's own tests
(core/test/base/mtx_io.cpp) and against each other on generated inputs.
Only tests import this module.

Matrix data is ((rows, cols), [(row, col, value), ...]).  value_type is
"f64" or "f32", index_type "i32" or "i64".  Errors raise MtxError with the
reference's StreamError message.
"""
from __future__ import annotations

import math
import re
import struct

import numpy as np


class MtxError(Exception):
    pass


_WS = " \t\n\v\f\r"
# the longest prefix a stream reads as a double / an integer (classic locale)
_DOUBLE = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?")
_BAD_EXP = re.compile(r"[+-]?(?:\d+\.?\d*|\.\d+)[eE](?![+-]?\d)")
_INT = re.compile(r"[+-]?\d+")
_HEADER = re.compile(r"^%%matrixmarket matrix (coordinate|array) "
                     r"(real|integer|complex|pattern) "
                     r"(general|symmetric|skew-symmetric|hermitian)")
_IRANGE = {"i32": (-2**31, 2**31 - 1), "i64": (-2**63, 2**63 - 1)}


def _round(x, value_type):
    if value_type != "f32":
        return float(x)
    with np.errstate(over="ignore"):  # a cast to float32 may overflow to inf
        return float(np.float32(x))


class _Stream:
    """istream-like cursor over a str (mtx_io.cpp reads through operator>>,
    getline and ignore)."""

    def __init__(self, text):
        self.s = text
        self.i = 0

    def getline(self):
        if self.i >= len(self.s):
            return None
        j = self.s.find("\n", self.i)
        if j < 0:
            line, self.i = self.s[self.i:], len(self.s)
        else:
            line, self.i = self.s[self.i:j], j + 1
        return line

    def ignore_line(self):
        j = self.s.find("\n", self.i)
        self.i = len(self.s) if j < 0 else j + 1

    def _skip(self):
        while self.i < len(self.s) and self.s[self.i] in _WS:
            self.i += 1

    def read_int(self, lo, hi):
        self._skip()
        m = _INT.match(self.s, self.i)
        if not m:
            return None
        self.i = m.end()
        v = int(m.group())
        return v if lo <= v <= hi else None

    def read_double(self):
        self._skip()
        if _BAD_EXP.match(self.s, self.i):
            return None
        m = _DOUBLE.match(self.s, self.i)
        if not m:
            return None
        self.i = m.end()
        v = float(m.group())
        # a decimal that overflows sets failbit in the stream (LWG 23);
        # an underflow keeps the correctly rounded tiny value or zero
        return None if math.isinf(v) else v


def read_raw(text, value_type="f64", index_type="i32"):
    """read_raw (mtx_io.cpp:73-81, header :612-659, coordinate :400-440,
    array :462-492, modifiers :252-381)."""
    st = _Stream(text)
    while True:
        line = st.getline()
        if line is None:
            raise MtxError("error when reading the header line")
        if line != "":
            break
    m = _HEADER.search(line.lower())
    if not m:
        raise MtxError("error parsing the header line")
    layout, field, modifier = m.groups()
    while True:
        dims = st.getline()
        if dims is None:
            raise MtxError("error when reading the dimensions line")
        if not dims.startswith("%"):
            break
    ds = _Stream(dims)
    lo, hi = _IRANGE[index_type]
    entries = []

    def entry():
        if field == "complex":
            raise MtxError("trying to read a complex matrix into a real storage type")
        if field == "pattern":
            return 1.0
        v = st.read_double()
        if v is None:
            raise MtxError("error while reading matrix entry")
        return _round(v, value_type)

    def insert(r, c, v):
        entries.append((r, c, v))
        if r != c and modifier != "general":
            entries.append((c, r, -v if modifier == "skew-symmetric" else v))

    def size():
        ds._skip()
        if ds.s[ds.i:ds.i + 1] == "-":
            return None
        return ds.read_int(0, 2**63 - 1)

    if layout == "coordinate":
        n, mcols, nnz = size(), size(), size()
        if None in (n, mcols, nnz):
            raise MtxError("error when determining matrix size, expected: rows cols nnz")
        for i in range(nnz):
            r = st.read_int(lo, hi)
            c = st.read_int(lo, hi) if r is not None else None
            if c is None:
                raise MtxError(f"error when reading coordinates of matrix entry {i}")
            insert(r - 1, c - 1, entry())
            st.ignore_line()
    else:
        n, mcols = size(), size()
        if None in (n, mcols):
            raise MtxError("error when determining matrix size, expected: rows cols")
        start = {"general": 0, "symmetric": 0, "hermitian": 0, "skew-symmetric": 1}[modifier]
        for c in range(mcols):
            r0 = 0 if modifier == "general" else c + start
            for r in range(r0, n):
                insert(r, c, entry())
                st.ignore_line()
    # sort_row_major; equal coordinates keep their order
    entries.sort(key=lambda t: (t[0], t[1]))
    return (n, mcols), entries


_VBITS = {"D": ("<d", 8), "S": ("<f", 4), "H": ("<e", 2), "B": (None, 2)}


def read_binary_raw(data, value_type="f64", index_type="i32"):
    """read_binary_raw (mtx_io.cpp:760-927)."""
    if len(data) < 32:
        raise MtxError("failed reading header")
    magic = data[:8]
    _, rows, cols, num = struct.unpack("<4Q", data[:32])
    vt, it = chr(magic[6]), chr(magic[7])
    if magic[:6] != b"GINKGO" or vt not in "DSHBZCXY" or it not in "IL":
        raise MtxError("invalid header magic number")
    imax = 2**31 - 1 if index_type == "i32" else 2**63 - 1
    if rows > imax or cols > imax:
        raise MtxError("cannot read into this format, its index type would overflow")
    if vt in "ZCXY":
        raise MtxError("cannot read into this format, would assign complex to real")
    ifmt, isz = ("<i", 4) if it == "I" else ("<q", 8)
    vfmt, vsz = _VBITS[vt]
    esz = 2 * isz + vsz
    entries = []
    for i in range(num):
        off = 32 + i * esz
        if off + esz > len(data):
            raise MtxError(f"failed reading entry {i}")
        r = struct.unpack_from(ifmt, data, off)[0]
        c = struct.unpack_from(ifmt, data, off + isz)[0]
        if index_type == "i32":
            r = (r + 2**31) % 2**32 - 2**31
            c = (c + 2**31) % 2**32 - 2**31
        if vfmt is None:  # bfloat16: the upper half of a binary32
            v = struct.unpack("<f", b"\0\0" + data[off + 2 * isz:off + esz])[0]
        else:
            v = struct.unpack_from(vfmt, data, off + 2 * isz)[0]
        entries.append((r, c, _round(v, value_type)))
    entries.sort(key=lambda t: (t[0], t[1]))
    return (rows, cols), entries


def read_generic_raw(data, value_type="f64", index_type="i32"):
    """read_generic_raw (mtx_io.cpp:930-941)."""
    if len(data) == 0:
        raise MtxError("failed reading from stream")
    if data[:1] == b"%":
        return read_raw(data.decode("latin-1"), value_type, index_type)
    return read_binary_raw(data, value_type, index_type)


def _g(v):
    return "%g" % v  # the default stream format of a double


def write_raw(size, entries, layout="coordinate"):
    """write_raw (mtx_io.cpp:980-1004; coordinate :442-460, array :494-525)."""
    n, m = size
    out = [f"%%MatrixMarket matrix {layout} real general\n"]
    if layout == "coordinate":
        out.append(f"{n} {m} {len(entries)}\n")
        out += [f"{r + 1} {c + 1} {_g(v)}\n" for r, c, v in entries]
        return "".join(out)
    srt = sorted(entries, key=lambda t: (t[1], t[0]))
    out.append(f"{n} {m}\n")
    pos = 0
    for j in range(m):
        for i in range(n):
            if pos >= len(srt) or (srt[pos][0], srt[pos][1]) != (i, j):
                out.append(_g(0.0) + "\n")
            else:
                out.append(_g(srt[pos][2]) + "\n")
                pos += 1
    return "".join(out)


def write_binary_raw(size, entries, value_type="f64", index_type="i64"):
    """write_binary_raw (mtx_io.cpp:943-978)."""
    vt = "D" if value_type == "f64" else "S"
    it = "I" if index_type == "i32" else "L"
    out = [b"GINKGO" + vt.encode() + it.encode(),
           struct.pack("<3Q", size[0], size[1], len(entries))]
    ifmt = "<i" if it == "I" else "<q"
    vfmt = "<d" if vt == "D" else "<f"
    for r, c, v in entries:
        out.append(struct.pack(ifmt, r) + struct.pack(ifmt, c) + struct.pack(vfmt, v))
    return b"".join(out)
