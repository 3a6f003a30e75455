"""Record-file I/O shared with oracle/ref_harness.cpp (TEST INFRASTRUCTURE ONLY).

A record is a 16-byte NUL-padded name, one type byte ('d' float64 or 'i'
int32), a little-endian int64 element count and the payload.
"""
from __future__ import annotations

import struct
from typing import Dict

import numpy as np


def write_records(path: str, records: Dict[str, object]) -> None:
    with open(path, "wb") as f:
        for name, value in records.items():
            arr = np.asarray(value)
            if arr.dtype.kind in "iub":
                arr, t = np.ascontiguousarray(arr, dtype="<i4").ravel(), b"i"
            else:
                arr, t = np.ascontiguousarray(arr, dtype="<f8").ravel(), b"d"
            f.write(name.encode()[:16].ljust(16, b"\0"))
            f.write(t)
            f.write(struct.pack("<q", arr.size))
            f.write(arr.tobytes())


def read_records(path: str) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos + 25 <= len(data):
        name = data[pos:pos + 16].rstrip(b"\0").decode()
        t = data[pos + 16:pos + 17]
        (count,) = struct.unpack("<q", data[pos + 17:pos + 25])
        pos += 25
        dt, size = ("<f8", 8) if t == b"d" else ("<i4", 4)
        out[name] = np.frombuffer(data[pos:pos + count * size], dtype=dt).copy()
        pos += count * size
    return out
