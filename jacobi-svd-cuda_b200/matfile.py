"""Python codec of the reference's `*.mat` stream format (tooling only).

One record = u64 rows | u64 columns | rows*columns f64, all big-endian,
row-major values; records are concatenated with no file header
(kleedaisuki/jacobi-svd-cuda include/io.hpp:40-51, src/io.cu:1180-1287).
The C++ implementation lives in csrc/io.cpp; this module writes test inputs
and reads outputs of either implementation.
"""
from __future__ import annotations

import numpy as np

_HDR = np.dtype([("rows", ">u8"), ("columns", ">u8")])


def encode(matrices) -> bytes:
    parts = []
    for a in matrices:
        a = np.asarray(a, dtype=np.float64)
        if a.ndim == 1:
            a = a.reshape(1, -1)
        hdr = np.array([(a.shape[0], a.shape[1])], dtype=_HDR)
        parts.append(hdr.tobytes())
        parts.append(np.ascontiguousarray(a).astype(">f8").tobytes())
    return b"".join(parts)


def decode(buf: bytes) -> list[np.ndarray]:
    out = []
    off = 0
    total = len(buf)
    while off < total:
        if total - off < 16:
            raise ValueError("Truncated *.mat header.")
        hdr = np.frombuffer(buf, dtype=_HDR, count=1, offset=off)[0]
        rows, cols = int(hdr["rows"]), int(hdr["columns"])
        off += 16
        nbytes = rows * cols * 8
        if total - off < nbytes:
            raise ValueError("Truncated *.mat payload.")
        vals = np.frombuffer(buf, dtype=">f8", count=rows * cols, offset=off).astype(np.float64)
        out.append(vals.reshape(rows, cols))
        off += nbytes
    return out


def write(path, matrices) -> None:
    with open(path, "wb") as f:
        f.write(encode(matrices))


def read(path) -> list[np.ndarray]:
    with open(path, "rb") as f:
        return decode(f.read())
