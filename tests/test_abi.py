"""The C-ABI library loads and exports every declared symbol; argument checks
return clean errors without touching a GPU."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(bz_\w+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    from beamz_b200 import _native as nat

    declared = _declared()
    assert "bz_step2d" in declared and "bz_rasterize2d" in declared
    missing = [n for n in declared if not hasattr(nat.lib, n)]
    assert not missing, missing
    assert set(nat.EXPORTED) == declared


def test_version_and_error_reporting():
    from beamz_b200 import _native as nat

    assert nat.version().startswith("beamz_b200")
    st = nat._step2d(None, None, None, None, 0, None, None)
    assert st == nat.BZ_ERR_INVALID
    code, msg = nat.last_error()
    assert code == nat.BZ_ERR_INVALID and "NULL" in msg
    with pytest.raises(nat.NativeError):
        nat.check(st)


def test_bad_grid_rejected_before_launch():
    from beamz_b200 import _native as nat

    g = nat.Grid2D()
    g.nx, g.ny, g.pitch, g.n_designs, g.n_comp, g.n_mat, g.dtype = 10, 10, 10, 1, 1, 1, 0
    f = nat.Fields2D()
    assert nat._step2d(C.byref(g), C.byref(f), None, None, 0, None, None) == nat.BZ_ERR_INVALID
    assert "pitch" in nat.last_error()[1]
    g.pitch, g.n_comp = 32, 3
    assert nat._step2d(C.byref(g), C.byref(f), None, None, 0, None, None) == nat.BZ_ERR_INVALID
    assert "n_comp" in nat.last_error()[1]
    assert nat._prepare(None, None, 1, 1, 1, 0, 1.0, 1.0, 1.0, None, None, None) == nat.BZ_ERR_INVALID
    assert nat._raster2d(0, 0, *([None] * 6), 0, None, None, None, None, 0, None, 1.0, 1.0, 1.0,
                         None, None, None, None) == nat.BZ_ERR_INVALID
