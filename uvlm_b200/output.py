"""Reading the per-step state records (`SimpleSimulator.set_sheet_path` / `set_result_path`).

Every record is its byte length (uint64, little endian) followed by one
message of proto/uvlm.proto in the protobuf wire format: AllVortexSheets
{t = 1, wing = 2, wake = 3} with VortexSheet {t = 1, num = 2, rows = 3,
cols = 4, vortices = 5}, or Snapshot2 {t = 1, ..., vortices = 3}; a
VortexRing is {gamma = 1, nodes = 2, nodes0 = 3} and a Point {x, y, z} =
{1, 2, 3}.  The decoder here reads those fields (others are skipped), so any
protobuf implementation of the schema reads the same bytes.
"""
from __future__ import annotations

import struct
from typing import Iterator

import numpy as np


def read_records(path: str) -> Iterator[bytes]:
    """The messages of a record file, in order."""
    with open(path, "rb") as f:
        while True:
            head = f.read(8)
            if not head:
                return
            if len(head) != 8:
                raise ValueError("truncated record header")
            (n,) = struct.unpack("<Q", head)
            body = f.read(n)
            if len(body) != n:
                raise ValueError("truncated record")
            yield body


def _varint(b: bytes, i: int):
    v = shift = 0
    while True:
        c = b[i]
        i += 1
        v |= (c & 0x7F) << shift
        if c < 0x80:
            return v, i
        shift += 7


def fields(b: bytes):
    """(field number, wire type, value) of every field of a message; value is an int (varint), a float
    (64-bit) or the bytes of a length-delimited field."""
    i, n = 0, len(b)
    while i < n:
        key, i = _varint(b, i)
        f, w = key >> 3, key & 7
        if w == 0:
            v, i = _varint(b, i)
        elif w == 1:
            (v,) = struct.unpack_from("<d", b, i)
            i += 8
        elif w == 2:
            ln, i = _varint(b, i)
            v = b[i:i + ln]
            i += ln
        elif w == 5:
            (v,) = struct.unpack_from("<f", b, i)
            i += 4
        else:
            raise ValueError(f"unsupported wire type {w}")
        yield f, w, v


def _point(b: bytes) -> list[float]:
    p = [0.0, 0.0, 0.0]
    for f, _, v in fields(b):
        if 1 <= f <= 3:
            p[f - 1] = v
    return p


def _ring(b: bytes):
    g, nodes = 0.0, []
    for f, _, v in fields(b):
        if f == 1:
            g = v
        elif f == 2:
            nodes.append(_point(v))
    return g, nodes


def decode_sheet(b: bytes) -> dict:
    """VortexSheet -> {num, rows, cols, rings (n, 4, 3), gammas (n,)}, rings in (n, i, j) order."""
    out = dict(num=0, rows=0, cols=0)
    rings, gammas = [], []
    for f, _, v in fields(b):
        if f in (2, 3, 4):
            out[{2: "num", 3: "rows", 4: "cols"}[f]] = v
        elif f == 5:
            g, nodes = _ring(v)
            rings.append(nodes)
            gammas.append(g)
    out["rings"] = np.array(rings, dtype=np.float64).reshape(-1, 4, 3)
    out["gammas"] = np.array(gammas, dtype=np.float64)
    return out


def decode_all_vortex_sheets(b: bytes) -> dict:
    """AllVortexSheets -> {t, wing, wake} with decode_sheet's dicts."""
    out = dict(t=0.0, wing=None, wake=None)
    for f, _, v in fields(b):
        if f == 1:
            out["t"] = v
        elif f == 2:
            out["wing"] = decode_sheet(v)
        elif f == 3:
            out["wake"] = decode_sheet(v)
    return out


def decode_snapshot2(b: bytes) -> dict:
    """Snapshot2 -> {rings (n, 4, 3), gammas (n,)} (the vortices field)."""
    rings, gammas = [], []
    for f, _, v in fields(b):
        if f == 3:
            g, nodes = _ring(v)
            rings.append(nodes)
            gammas.append(g)
    return dict(rings=np.array(rings, dtype=np.float64).reshape(-1, 4, 3), gammas=np.array(gammas))


def read_sheets(path: str) -> list[dict]:
    """Every AllVortexSheets record of a sheet file."""
    return [decode_all_vortex_sheets(m) for m in read_records(path)]


def read_snapshots(path: str) -> list[dict]:
    """Every Snapshot2 record of a result file."""
    return [decode_snapshot2(m) for m in read_records(path)]


def sheet_to_grid(sheet: dict):
    """A decoded VortexSheet back to the simulator's arrays: nodes (num, rows+1, cols+1, 3) and circulations
    (num, rows, cols) (ring (n, i, j) has nodes p(i,j), p(i,j+1), p(i+1,j+1), p(i+1,j))."""
    num, rows, cols = sheet["num"], sheet["rows"], sheet["cols"]
    g = sheet["gammas"].reshape(num, rows, cols)
    if rows == 0:
        return None, g
    r = sheet["rings"].reshape(num, rows, cols, 4, 3)
    pos = np.zeros((num, rows + 1, cols + 1, 3))
    pos[:, :rows, :cols] = r[..., 0, :]
    pos[:, :rows, cols] = r[:, :, cols - 1, 1, :]
    pos[:, rows, :cols] = r[:, rows - 1, :, 3, :]
    pos[:, rows, cols] = r[:, rows - 1, cols - 1, 2, :]
    return pos, g
