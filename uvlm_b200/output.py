"""Reading the per-step state records (`SimpleSimulator.set_sheet_path` / `set_result_path`).

Every record is its byte length (uint64, little endian) followed by one
message of proto/uvlm.proto in the protobuf wire format: AllVortexSheets
{t = 1, wing = 2, wake = 3} with VortexSheet {t = 1, num = 2, rows = 3,
cols = 4, vortices = 5}, or Snapshot2 {t = 1, ..., vortices = 3}; a
VortexRing is {gamma = 1, nodes = 2, nodes0 = 3} and a Point {x, y, z} =
{1, 2, 3}.  The decoder here reads those fields (others are skipped), so any
protobuf implementation of the schema reads the same bytes.

The legacy simulator (uvlm_b200.legacy) writes one unframed Snapshot2 file
per step instead (src/simulator/simulator.cpp:118-160), with t = 1,
container_shapes = 2 {rows, cols, id, chord = 5, span = 6}, the ring pool
with reference nodes (nodes0 = 3) and morphing_velocities = 4 {center = 1,
nodes = 2, freestream = 3}.
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


def _ring(b: bytes, with_nodes0: bool = False):
    g, nodes, nodes0 = 0.0, [], []
    for f, _, v in fields(b):
        if f == 1:
            g = v
        elif f == 2:
            nodes.append(_point(v))
        elif f == 3 and with_nodes0:
            nodes0.append(_point(v))
    return (g, nodes, nodes0) if with_nodes0 else (g, nodes)


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


def _shape(b: bytes) -> dict:
    out = dict(rows=0, cols=0, id=0, chord=0.0, span=0.0)
    for f, _, v in fields(b):
        if 1 <= f <= 3:
            out[("rows", "cols", "id")[f - 1]] = v
        elif f == 5:
            out["chord"] = v
        elif f == 6:
            out["span"] = v
    return out


def decode_snapshot2(b: bytes) -> dict:
    """Snapshot2 -> {t, container_shapes, rings (n, 4, 3), rings0, gammas (n,), mv_center (m, 3),
    mv_nodes (m, 4, 3), mv_freestream (m, 3)}: container_shapes are dicts {rows, cols, id, chord, span}
    (ContainerShape), rings None when a ring does not carry four nodes, rings0 the rings' reference nodes
    ((n, 4, 3), or None when the rings carry none), and the mv_* arrays the MorphingVelocity records
    {center, nodes, freestream}."""
    out = dict(t=0.0, container_shapes=[])
    rings, rings0, gammas, center, mv_nodes, free = [], [], [], [], [], []
    for f, _, v in fields(b):
        if f == 1:
            out["t"] = v
        elif f == 2:
            out["container_shapes"].append(_shape(v))
        elif f == 3:
            g, nodes, nodes0 = _ring(v, with_nodes0=True)
            rings.append(nodes)
            rings0.append(nodes0)
            gammas.append(g)
        elif f == 4:
            c, nodes, fs = [0.0] * 3, [], [0.0] * 3
            for f2, _, v2 in fields(v):
                if f2 == 1:
                    c = _point(v2)
                elif f2 == 2:
                    nodes.append(_point(v2))
                elif f2 == 3:
                    fs = _point(v2)
            center.append(c)
            mv_nodes.append(nodes)
            free.append(fs)
    # rings without four nodes (a message holding circulations only) leave no ring array
    out["rings"] = np.array(rings, dtype=np.float64).reshape(-1, 4, 3) if all(len(r) == 4 for r in rings) else None
    out["gammas"] = np.array(gammas, dtype=np.float64)
    has0 = bool(rings0) and all(len(r) == 4 for r in rings0)
    out["rings0"] = np.array(rings0, dtype=np.float64).reshape(-1, 4, 3) if has0 else None
    out["mv_center"] = np.array(center, dtype=np.float64).reshape(-1, 3)
    out["mv_nodes"] = np.array(mv_nodes, dtype=np.float64).reshape(len(mv_nodes), -1, 3) if mv_nodes else \
        np.zeros((0, 4, 3))
    out["mv_freestream"] = np.array(free, dtype=np.float64).reshape(-1, 3)
    return out


def read_snapshot2_file(path: str) -> dict:
    """One unframed Snapshot2 file of the legacy simulator (LegacySimulator.SetOutputPath)."""
    with open(path, "rb") as f:
        return decode_snapshot2(f.read())


def snapshot_containers(snap: dict) -> list[dict]:
    """The VortexContainer views of a decoded Snapshot2 (Snapshot2ToContainers, src/proto_adaptor.h:75-89):
    each shape's dict plus `offset`, the index of its first ring in the pool, id x rows x cols
    (VortexContainer::Offset, src/vortex_container.h:55)."""
    return [dict(c, offset=c["id"] * c["rows"] * c["cols"]) for c in snap["container_shapes"]]


def write_legacy_snapshot2(path: str, t: float, shapes, rings, rings0, gammas, mv_center, mv_nodes,
                           mv_freestream) -> None:
    """Write one legacy Snapshot2 file (uvlm_write_legacy_snapshot2): shapes = [(rows, cols, chord, span)],
    container c gets id c; rings0 None writes no reference nodes."""
    import ctypes as C

    from ._capi import check, lib

    P = C.POINTER(C.c_double)

    def arr(a, shape):
        return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))

    n_c = len(shapes)
    rows = (C.c_int64 * max(n_c, 1))(*[int(s[0]) for s in shapes])
    cols = (C.c_int64 * max(n_c, 1))(*[int(s[1]) for s in shapes])
    chord = arr([s[2] for s in shapes], -1)
    span = arr([s[3] for s in shapes], -1)
    r = arr(rings, (-1, 4, 3))
    r0 = None if rings0 is None else arr(rings0, (-1, 4, 3))
    g = arr(gammas, -1)
    c, nd, fs = arr(mv_center, (-1, 3)), arr(mv_nodes, (-1, 4, 3)), arr(mv_freestream, (-1, 3))
    if (r0 is not None and r0.shape != r.shape) or g.shape[0] != r.shape[0] or not (
            c.shape[0] == nd.shape[0] == fs.shape[0]):
        raise ValueError("inconsistent snapshot arrays")
    p = lambda a: a.ctypes.data_as(P) if a is not None and a.size else None  # noqa: E731
    check(lib().uvlm_write_legacy_snapshot2(str(path).encode(), float(t), n_c, rows, cols, p(chord), p(span), p(r),
                                            p(r0), p(g), r.shape[0], p(c), p(nd), p(fs), c.shape[0]))


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
