"""A reader for the msgpack subset a DIALS reflection table uses, for the
tests: decodes the document into Python values, each column as
(type name, row count, raw bytes)."""

from __future__ import annotations

import struct

import numpy as np


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        self.i = 0

    def take(self, n):
        b = self.d[self.i:self.i + n]
        if len(b) != n:
            raise ValueError("truncated")
        self.i += n
        return b

    def uint(self, n):
        return int.from_bytes(self.take(n), "big")

    def value(self):
        t = self.take(1)[0]
        if t < 0x80:
            return t
        if 0x80 <= t <= 0x8f:
            return self.map(t & 0x0f)
        if 0x90 <= t <= 0x9f:
            return [self.value() for _ in range(t & 0x0f)]
        if 0xa0 <= t <= 0xbf:
            return self.take(t & 0x1f).decode()
        if t in (0xc4, 0xc5, 0xc6):
            return bytes(self.take(self.uint({0xc4: 1, 0xc5: 2, 0xc6: 4}[t])))
        if t in (0xcc, 0xcd, 0xce, 0xcf):
            return self.uint({0xcc: 1, 0xcd: 2, 0xce: 4, 0xcf: 8}[t])
        if t in (0xd9, 0xda, 0xdb):
            return self.take(self.uint({0xd9: 1, 0xda: 2, 0xdb: 4}[t])).decode()
        if t in (0xdc, 0xdd):
            return [self.value() for _ in range(self.uint(2 if t == 0xdc else 4))]
        if t in (0xde, 0xdf):
            return self.map(self.uint(2 if t == 0xde else 4))
        raise ValueError(f"msgpack type 0x{t:02x} is not used by reflection tables")

    def map(self, n):
        out = {}
        for _ in range(n):
            k = self.value()
            out[k] = self.value()
        return out


def read(path):
    data = open(path, "rb").read()
    r = _Reader(data)
    doc = r.value()
    if r.i != len(data):
        raise ValueError("trailing bytes")
    name, version, body = doc
    columns = {k: (v[0], v[1][0], v[1][1]) for k, v in body["data"].items()}
    return {"name": name, "version": version, "identifiers": body["identifiers"],
            "nrows": body["nrows"], "columns": columns}


def shoeboxes(raw: bytes, rows: int):
    """The shoebox column as a list of (panel, bbox, data, mask, background)."""
    out, at = [], 0
    for _ in range(rows):
        panel, *bbox = struct.unpack_from("<I6i", raw, at)
        at += 28
        assert raw[at] == 2
        at += 1
        n = (bbox[1] - bbox[0]) * (bbox[3] - bbox[2]) * (bbox[5] - bbox[4])
        shape = (bbox[5] - bbox[4], bbox[3] - bbox[2], bbox[1] - bbox[0])
        data = np.frombuffer(raw, np.float32, n, at).reshape(shape)
        at += 4 * n
        mask = np.frombuffer(raw, np.uint8, n, at).reshape(shape)
        at += n
        bg = np.frombuffer(raw, np.float32, n, at).reshape(shape)
        at += 4 * n
        out.append((panel, bbox, data, mask, bg))
    assert at == len(raw)
    return out
