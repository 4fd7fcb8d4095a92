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


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes mirror of a header struct has the C struct's size and field offsets
    (a C program built against include/beamz_b200.h prints them)."""
    import shutil
    import subprocess

    from beamz_b200 import _native as nat

    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    pairs = {"Grid2D": "bz_grid2d", "Fields2D": "bz_fields2d", "SourceOps": "bz_source_ops",
             "MonitorOps": "bz_monitor_ops", "Adjoint2D": "bz_adjoint2d", "Gemm": "bz_gemm", "Grid3D": "bz_grid3d",
             "Fields3D": "bz_fields3d", "GatherOps": "bz_gather_ops", "Shape2D": "bz_shape2d",
             "Shape3D": "bz_shape3d", "Pml2D": "bz_pml2d"}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "beamz_b200.h"', "int main(void) {"]
    for py, c in pairs.items():
        lines.append(f'  printf("{py} sizeof %zu\\n", sizeof({c}));')
        for field in getattr(nat, py)._fields_:
            lines.append(f'  printf("{py} {field[0]} %zu\\n", offsetof({c}, {field[0]}));')
    lines += ["  return 0;", "}"]
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    bad = []
    for py, field, value in zip(out[0::3], out[1::3], out[2::3]):
        cls = getattr(nat, py)
        want = C.sizeof(cls) if field == "sizeof" else getattr(cls, field).offset
        if want != int(value):
            bad.append((py, field, int(value), want))
    assert not bad, bad
