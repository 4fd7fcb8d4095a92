"""GDSII I/O of Design (design/gds.py): the 8-byte real format, a stream built here byte
by byte from the format's record layout (references, arrays, paths), and an
export/import round trip."""
import struct

import numpy as np
import pytest

from beamz_b200.design.gds import read_gds, real8_decode, real8_encode


@pytest.mark.parametrize("v,b", [(1.0, "4110000000000000"), (0.5, "4080000000000000"), (-2.0, "c120000000000000"),
                                 (0.0, "0000000000000000"), (16.0, "4210000000000000")])
def test_real8_known_bytes(v, b):
    assert real8_encode(v).hex() == b
    assert real8_decode(bytes.fromhex(b)) == v


def test_real8_round_trip_is_exact():
    rng = np.random.default_rng(3)
    for v in np.concatenate([10.0 ** rng.uniform(-12, 12, 200) * rng.choice([-1, 1], 200), [1e-3, 1e-9, 1e-6, 90.0]]):
        assert real8_decode(real8_encode(v)) == v


def _rec(rtype, dtype, data=b""):
    if len(data) % 2:
        data += b"\0"
    return struct.pack(">HBB", 4 + len(data), rtype, dtype) + data


def _i2(*v):
    return struct.pack(f">{len(v)}h", *v)


def _i4(*v):
    return struct.pack(f">{len(v)}i", *v)


def _stream():
    """Cell "unit": a 1000 x 500 nm box on layer 3. Cell "top": an SREF of it rotated by
    90 degrees at (5000, 0), a 2 x 1 AREF at (0, 10000) with pitch 2000 in x, and a
    200 nm wide flush PATH on layer 4 from (0, -1000) to (3000, -1000)."""
    stamp = _i2(2000, 1, 1, 0, 0, 0, 2000, 1, 1, 0, 0, 0)
    b = _rec(0x00, 2, _i2(600)) + _rec(0x01, 2, stamp) + _rec(0x02, 6, b"LIB")
    b += _rec(0x03, 5, real8_encode(1e-3) + real8_encode(1e-9))
    b += _rec(0x05, 2, stamp) + _rec(0x06, 6, b"unit")
    b += _rec(0x08, 0) + _rec(0x0D, 2, _i2(3)) + _rec(0x0E, 2, _i2(0))
    b += _rec(0x10, 3, _i4(0, 0, 1000, 0, 1000, 500, 0, 500, 0, 0)) + _rec(0x11, 0)
    b += _rec(0x07, 0)
    b += _rec(0x05, 2, stamp) + _rec(0x06, 6, b"top")
    b += _rec(0x0A, 0) + _rec(0x12, 6, b"unit") + _rec(0x1A, 1, struct.pack(">H", 0))
    b += _rec(0x1C, 5, real8_encode(90.0)) + _rec(0x10, 3, _i4(5000, 0)) + _rec(0x11, 0)
    b += _rec(0x0B, 0) + _rec(0x12, 6, b"unit") + _rec(0x13, 2, _i2(2, 1))
    b += _rec(0x10, 3, _i4(0, 10000, 4000, 10000, 0, 11000)) + _rec(0x11, 0)
    b += _rec(0x09, 0) + _rec(0x0D, 2, _i2(4)) + _rec(0x0E, 2, _i2(0)) + _rec(0x21, 2, _i2(0))
    b += _rec(0x0F, 3, _i4(200)) + _rec(0x10, 3, _i4(0, -1000, 3000, -1000)) + _rec(0x11, 0)
    b += _rec(0x07, 0) + _rec(0x04, 0)
    return b


def _bbox(p):
    return np.round(np.concatenate([p.min(axis=0), p.max(axis=0)]) * 1e9).astype(int).tolist()


def test_read_flattens_references_arrays_and_paths(tmp_path):
    f = tmp_path / "t.gds"
    f.write_bytes(_stream())
    polys = read_gds(str(f))
    assert set(polys) == {(3, 0), (4, 0)}
    boxes = sorted(_bbox(p) for p in polys[(3, 0)])
    assert boxes == [[0, 10000, 1000, 10500], [2000, 10000, 3000, 10500], [4500, 0, 5000, 1000]]
    assert [_bbox(p) for p in polys[(4, 0)]] == [[0, -1100, 3000, -900]]


def test_design_import_gds(bz, tmp_path):
    f = tmp_path / "t.gds"
    f.write_bytes(_stream())
    d = bz.Design.import_gds(str(f), default_depth=0.22e-6)
    assert len(d.layers[3]) == 3 and len(d.layers[4]) == 1
    assert d.is_3d and d.depth == 0.22e-6
    assert all(p in d.structures for p in d.layers[3])


def test_export_import_round_trip(bz, tmp_path):
    from beamz_b200.design.structures import _point_in_path

    si, sin = bz.Material(permittivity=12.25), bz.Material(permittivity=4.0)
    d = bz.Design(width=6e-6, height=4e-6, auto_pml=False)
    d.add(bz.Rectangle(position=(0.5e-6, 1e-6), width=2e-6, height=0.5e-6, material=si))
    d.add(bz.Polygon(vertices=[(3e-6, 1e-6), (4.5e-6, 1e-6), (3.7e-6, 2.5e-6)], material=si))
    d.add(bz.Ring(position=(2e-6, 3e-6), inner_radius=0.3e-6, outer_radius=0.6e-6, material=sin))
    f = tmp_path / "rt.gds"
    d.export_gds(str(f))
    polys = read_gds(str(f))
    assert sorted(polys) == [(0, 0), (1, 0), (2, 0)]  # background, Si, SiN in order of first appearance
    assert len(polys[(1, 0)]) == 2 and len(polys[(2, 0)]) == 1
    assert sorted(_bbox(p) for p in polys[(1, 0)]) == [[500, 1000, 2500, 1500], [3000, 1000, 4500, 2500]]
    ring = [tuple(v) for v in polys[(2, 0)][0]]
    assert not _point_in_path(2e-6, 3e-6, ring)  # the hole
    assert _point_in_path(2e-6 + 0.45e-6, 3e-6, ring)  # the band
    assert not _point_in_path(2e-6 + 0.8e-6, 3e-6, ring)
