"""GDSII stream read/write for Design.import_gds / Design.export_gds (beamz/design/core.py:445-553).

The reference goes through gdspy; this module reads and writes the GDSII stream
format itself (big-endian records: 2-byte length, record type, data type, data;
8-byte reals in the format's excess-64 base-16 form).

Writing: one library (user unit 1 um, database unit 1 nm, as the reference's
gdspy library), one cell "main", one BOUNDARY per polygon; a polygon with holes is
written as one boundary that walks the outline, cuts in to each hole, walks it the
other way round and comes back (a keyhole), which the even-odd fill rule reads as
the same region.

Reading: BOUNDARY and PATH elements (path types 0, 1 and 2 as polygons: flush, round
ends drawn flush, ends extended by half the width; joints mitred), SREF and AREF
references flattened with reflection about x, magnification and rotation (the
absolute-magnification/angle flags are read as relative), BOX/TEXT/NODE skipped.
Only the top cells (those no reference points to) are flattened, so a referenced
cell is placed where its references put it and nowhere else.
"""
from __future__ import annotations

import math
import struct
from typing import Dict, List, Tuple

import numpy as np

# record types
HEADER, BGNLIB, LIBNAME, UNITS, ENDLIB, BGNSTR, STRNAME, ENDSTR = 0x00, 0x01, 0x02, 0x03, 0x04, 0x05, 0x06, 0x07
BOUNDARY, PATH, SREF, AREF, TEXT, LAYER, DATATYPE, WIDTH, XY, ENDEL = (0x08, 0x09, 0x0A, 0x0B, 0x0C, 0x0D, 0x0E, 0x0F,
                                                                       0x10, 0x11)
SNAME, COLROW, NODE, STRANS, MAG, ANGLE, PATHTYPE, BOX = 0x12, 0x13, 0x15, 0x1A, 0x1B, 0x1C, 0x21, 0x2D
# data types
NO_DATA, BITARRAY, INT2, INT4, REAL8, ASCII = 0, 1, 2, 3, 5, 6


def real8_encode(v: float) -> bytes:
    """8-byte GDSII real: sign bit, 7-bit exponent of 16 biased by 64, 56-bit fraction."""
    if v == 0:
        return bytes(8)
    sign = 0x80 if v < 0 else 0
    v = abs(float(v))
    exp = 64
    while v >= 1.0:  # scaling by 16 is exact in binary floating point
        v /= 16.0
        exp += 1
    while v < 1.0 / 16.0:
        v *= 16.0
        exp -= 1
    mant = int(round(v * (1 << 56)))
    if mant >= 1 << 56:  # rounded up to 1.0
        mant >>= 4
        exp += 1
    if not 0 <= exp <= 127:
        raise ValueError(f"{v} is outside the GDSII real range")
    return bytes([sign | exp]) + mant.to_bytes(7, "big")


def real8_decode(b: bytes) -> float:
    exp = (b[0] & 0x7F) - 64
    mant = int.from_bytes(b[1:8], "big")
    v = math.ldexp(mant, 4 * exp - 56)
    return -v if b[0] & 0x80 else v


def _record(rtype: int, dtype: int, data: bytes = b"") -> bytes:
    if len(data) % 2:
        data += b"\0"
    if len(data) + 4 > 0xFFFF:
        raise ValueError("GDSII record longer than 65535 bytes")
    return struct.pack(">HBB", len(data) + 4, rtype, dtype) + data


_STAMP = struct.pack(">12h", 2000, 1, 1, 0, 0, 0, 2000, 1, 1, 0, 0, 0)  # fixed: the output is reproducible


def write_gds(path: str, polygons: Dict[int, List[Tuple[np.ndarray, List[np.ndarray]]]], unit=1e-6, precision=1e-9,
              libname="BEAMZ", cellname="main") -> None:
    """Writes {layer: [(outline (n, 2) in metres, [hole (m, 2), ...]), ...]} as BOUNDARY
    elements of one cell; coordinates are rounded to the database unit ``precision``."""
    out = [_record(HEADER, INT2, struct.pack(">h", 600)), _record(BGNLIB, INT2, _STAMP),
           _record(LIBNAME, ASCII, libname.encode()),
           _record(UNITS, REAL8, real8_encode(precision / unit) + real8_encode(precision)),
           _record(BGNSTR, INT2, _STAMP), _record(STRNAME, ASCII, cellname.encode())]
    for layer in sorted(polygons):
        for outline, holes in polygons[layer]:
            pts = _keyhole(np.asarray(outline, dtype=float), [np.asarray(h, dtype=float) for h in holes])
            q = np.rint(pts / precision).astype(np.int64)
            q = np.vstack([q, q[:1]])  # a boundary repeats its first point
            if len(q) > 8191:
                raise ValueError(f"polygon with {len(q)} points exceeds the 8191 points of a GDSII boundary")
            if np.abs(q).max() >= 2 ** 31:
                raise ValueError("coordinate outside the 32-bit GDSII range")
            out += [_record(BOUNDARY, NO_DATA), _record(LAYER, INT2, struct.pack(">h", layer)),
                    _record(DATATYPE, INT2, struct.pack(">h", 0)),
                    _record(XY, INT4, struct.pack(f">{2 * len(q)}i", *q.reshape(-1).tolist())), _record(ENDEL, NO_DATA)]
    out += [_record(ENDSTR, NO_DATA), _record(ENDLIB, NO_DATA)]
    with open(path, "wb") as fh:
        fh.write(b"".join(out))


def _keyhole(outline: np.ndarray, holes: List[np.ndarray]) -> np.ndarray:
    """One point loop for an outline with holes: after outline point 0 it goes to each
    hole's first point, round the hole, and back to outline point 0."""
    if not holes:
        return outline
    pts = [outline[0]]
    for h in holes:
        h = np.asarray(h, dtype=float)
        pts += [h[0], *h[1:], h[0], outline[0]]
    pts += list(outline[1:])
    return np.asarray(pts)


def _parse(data: bytes):
    """Records as (type, payload) pairs."""
    i, n = 0, len(data)
    while i + 4 <= n:
        length, rtype, dtype = struct.unpack(">HBB", data[i:i + 4])
        if length < 4:
            raise ValueError(f"bad GDSII record length {length} at byte {i}")
        payload = data[i + 4:i + length]
        if dtype == INT2:
            val = struct.unpack(f">{len(payload) // 2}h", payload)
        elif dtype == INT4:
            val = struct.unpack(f">{len(payload) // 4}i", payload)
        elif dtype == REAL8:
            val = tuple(real8_decode(payload[k:k + 8]) for k in range(0, len(payload), 8))
        elif dtype == ASCII:
            val = payload.rstrip(b"\0").decode("ascii", "replace")
        elif dtype == BITARRAY:
            val = struct.unpack(">H", payload)[0]
        else:
            val = None
        yield rtype, val
        i += length
        if rtype == ENDLIB:
            break


def _path_polygon(pts: np.ndarray, width: float, pathtype: int) -> np.ndarray:
    """Outline of a path of the given width (mitred joints; type 2 extends both ends
    by half the width, types 0 and 1 end flush)."""
    pts = np.asarray(pts, dtype=float)
    keep = np.r_[True, np.any(np.diff(pts, axis=0) != 0, axis=1)]
    pts = pts[keep]
    if len(pts) < 2 or width == 0:
        return np.zeros((0, 2))
    hw = abs(width) / 2
    d = np.diff(pts, axis=0)
    d /= np.linalg.norm(d, axis=1)[:, None]
    nrm = np.stack([-d[:, 1], d[:, 0]], axis=1)
    if pathtype == 2:
        pts = pts.copy()
        pts[0] -= d[0] * hw
        pts[-1] += d[-1] * hw
    left, right = [pts[0] + nrm[0] * hw], [pts[0] - nrm[0] * hw]
    for k in range(1, len(pts) - 1):
        m = nrm[k - 1] + nrm[k]
        m_len = np.dot(m, nrm[k])
        m = m / m_len if abs(m_len) > 1e-12 else nrm[k]
        left.append(pts[k] + m * hw)
        right.append(pts[k] - m * hw)
    left.append(pts[-1] + nrm[-1] * hw)
    right.append(pts[-1] - nrm[-1] * hw)
    return np.asarray(left + right[::-1])


def read_gds(path: str) -> Dict[Tuple[int, int], List[np.ndarray]]:
    """{(layer, datatype): [polygon (n, 2) in metres, ...]} of the flattened top cells."""
    with open(path, "rb") as fh:
        data = fh.read()
    cells: Dict[str, list] = {}
    order: List[str] = []
    meters = 1e-9
    cur, elem = None, None
    for rtype, val in _parse(data):
        if rtype == UNITS:
            meters = val[1]
        elif rtype == STRNAME:
            cur = cells.setdefault(val, [])
            order.append(val)
        elif rtype in (BOUNDARY, PATH, SREF, AREF):
            elem = {"kind": rtype, "layer": 0, "datatype": 0, "width": 0, "pathtype": 0, "strans": 0, "mag": 1.0,
                    "angle": 0.0, "colrow": (1, 1)}
        elif rtype in (TEXT, NODE, BOX):
            elem = {"kind": None}
        elif elem is not None:
            if rtype == LAYER:
                elem["layer"] = val[0]
            elif rtype == DATATYPE:
                elem["datatype"] = val[0]
            elif rtype == WIDTH:
                elem["width"] = val[0]
            elif rtype == PATHTYPE:
                elem["pathtype"] = val[0]
            elif rtype == XY:
                elem["xy"] = np.asarray(val, dtype=float).reshape(-1, 2)
            elif rtype == SNAME:
                elem["sname"] = val
            elif rtype == STRANS:
                elem["strans"] = val
            elif rtype == MAG:
                elem["mag"] = val[0]
            elif rtype == ANGLE:
                elem["angle"] = val[0]
            elif rtype == COLROW:
                elem["colrow"] = (val[0], val[1])
            elif rtype == ENDEL:
                if elem["kind"] is not None and cur is not None and "xy" in elem:
                    cur.append(elem)
                elem = None
    referenced = {e["sname"] for es in cells.values() for e in es if e["kind"] in (SREF, AREF) and "sname" in e}
    out: Dict[Tuple[int, int], List[np.ndarray]] = {}

    def emit(name, transform, depth):
        if depth > 64:
            raise ValueError("GDSII references nest deeper than 64 levels (a cycle?)")
        for e in cells.get(name, []):
            if e["kind"] == BOUNDARY:
                pts = e["xy"]
                if len(pts) > 1 and np.array_equal(pts[0], pts[-1]):
                    pts = pts[:-1]
                out.setdefault((e["layer"], e["datatype"]), []).append(transform(pts) * meters)
            elif e["kind"] == PATH:
                poly = _path_polygon(e["xy"], e["width"], e["pathtype"])
                if len(poly):
                    out.setdefault((e["layer"], e["datatype"]), []).append(transform(poly) * meters)
            else:
                origins = [e["xy"][0]]
                if e["kind"] == AREF:
                    cols, rows = e["colrow"]
                    p1, p2, p3 = e["xy"][:3]
                    cv, rv = (p2 - p1) / cols, (p3 - p1) / rows
                    origins = [p1 + c * cv + r * rv for r in range(rows) for c in range(cols)]
                th = math.radians(e["angle"])
                rot = np.array([[math.cos(th), -math.sin(th)], [math.sin(th), math.cos(th)]]) * e["mag"]
                flip = np.diag([1.0, -1.0]) if e["strans"] & 0x8000 else np.eye(2)
                lin = rot @ flip
                for o in origins:
                    emit(e["sname"], lambda p, lin=lin, o=o, tr=transform: tr(p @ lin.T + o), depth + 1)

    for name in order:
        if name not in referenced:
            emit(name, lambda p: p, 0)
    return out
