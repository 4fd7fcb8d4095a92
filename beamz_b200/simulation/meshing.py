"""Design -> material grids (beamz/simulation/meshing.py:8-925), rasterised on the GPU.

``RegularGrid(design, resolution)`` exposes ``permittivity``, ``permeability`` and
``conductivity`` as float64 NumPy arrays of shape (ny, nx) with
``nx = int(width / resolution)``, like the reference, so callers can edit them
(``np.copyto(grid.permittivity, eps)``) before handing the grid to ``FDTD``.

The host compiles each structure into the record of the fast path the reference
uses for it (``_compile_shapes``: index boxes, interior/boundary split, Python
slice semantics) and tabulates the position-only part of each PML region
(``_compile_pml``); ``bz_rasterize2d`` then evaluates every cell on the device.
"""
from __future__ import annotations

import ctypes as C
from typing import Any

import numpy as np
import torch

from .. import _native as nat
from ..const import EPS_0, MU_0
from ..design.materials import material_triple
from ..design.structures import Rectangle
from ..helpers import display_status

__all__ = ["BaseMeshGrid", "RegularGrid", "RegularGrid3D", "create_mesh", "mesh_2d", "mesh_3d"]


def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("beamz_b200 needs a CUDA GPU (sm_100a); none is visible")
    return torch.device("cuda", torch.cuda.current_device())


def _dev_f64(a) -> torch.Tensor:
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(_device())


def _dev_struct_array(structs, ctype) -> torch.Tensor | None:
    if not structs:
        return None
    arr = (ctype * len(structs))(*structs)
    raw = bytes(C.string_at(C.addressof(arr), C.sizeof(arr)))
    return torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(_device())


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _slice_bounds(start: int, stop: int, n: int) -> tuple[int, int]:
    s, e, _ = slice(start, stop).indices(n)
    return s, max(s, e)


class BaseMeshGrid:
    def __init__(self, design, resolution):
        self.design = design
        self.resolution = resolution
        if self.resolution <= 0:
            raise ValueError("Resolution must be positive")
        if self.design is None:
            raise ValueError("Design cannot be None")


def _is_device(s) -> bool:
    from ..devices.monitors import Monitor
    from ..devices.sources import GaussianSource, ModeSource

    return isinstance(s, (ModeSource, GaussianSource, Monitor))


def _compile_shapes(design, cs: float, gw: int, gh: int, x_centers, y_centers):
    """Per-structure rasteriser records, mirroring the path selection of
    meshing.py:146-482 for every structure after the background."""
    shapes, paths, verts, custom = [], [], [], []
    for s in design.structures[1:]:
        if getattr(s, "is_pml", False) or _is_device(s):
            continue
        mat = getattr(s, "material", None)
        if mat is None:
            continue
        is_custom = hasattr(mat, "get_permittivity")
        bbox = s.get_bounding_box() if hasattr(s, "get_bounding_box") else None
        if bbox is None:
            display_status(f"Warning: structure {type(s).__name__} has no bounding box; skipped", "warning")
            continue
        if len(bbox) == 6:
            min_x, min_y, _, max_x, max_y, _ = bbox
        elif len(bbox) == 4:
            min_x, min_y, max_x, max_y = bbox
        else:
            raise ValueError(f"Invalid bounding box format: {bbox}")
        i0 = max(0, int(min_y / cs) - 1)
        j0 = max(0, int(min_x / cs) - 1)
        i1 = min(gh, int(np.ceil(max_y / cs)) + 1)
        j1 = min(gw, int(np.ceil(max_x / cs)) + 1)
        if i0 >= gh or j0 >= gw or i1 <= 0 or j1 <= 0:
            continue
        rec = nat.Shape2D()
        rec.custom_off = -1
        if not is_custom:
            rec.perm, rec.permb, rec.cond = (float(v) for v in material_triple(mat))
        if isinstance(s, Rectangle) and s.vertices[0][0] - s.position[0] == 0 and s.vertices[0][1] - s.position[1] == 0:
            px, py = s.position[0], s.position[1]
            ri0, rj0 = max(0, int(py / cs)), max(0, int(px / cs))
            rj1 = min(gw, int(np.ceil((px + s.width) / cs)))
            ri1 = min(gh, int(np.ceil((py + s.height) / cs)))
            ii0 = max(0, int((py + 0.25 * cs) / cs))
            ij0 = max(0, int((px + 0.25 * cs) / cs))
            ij1 = min(gw, int(np.floor((px + s.width - 0.25 * cs) / cs)))
            ii1 = min(gh, int(np.floor((py + s.height - 0.25 * cs) / cs)))
            nrows, ncols = ri1 - ri0, rj1 - rj0
            if nrows < 0 or ncols < 0:
                raise ValueError("negative dimensions are not allowed")
            rec.kind = nat.BZ_SHAPE_RECT
            rec.i0, rec.i1, rec.j0, rec.j1 = ri0, ri1, rj0, rj1
            rec.fill = int(ii1 > ii0 and ij1 > ij0)
            if is_custom:  # explicit index loops in the reference (range semantics)
                rec.fi0, rec.fi1, rec.fj0, rec.fj1 = ii0, max(ii0, ii1), ij0, max(ij0, ij1)
            else:  # NumPy slice assignment (slice semantics)
                rec.fi0, rec.fi1 = _slice_bounds(ii0, ii1, gh)
                rec.fj0, rec.fj1 = _slice_bounds(ij0, ij1, gw)
            rec.top = (ii0 - ri0) if ri0 < ii0 else 0
            rec.bottom = slice(ii1 - ri0, None).indices(nrows)[0] if ii1 < ri1 else 1 << 30
            rec.left = (ij0 - rj0) if rj0 < ij0 else 0
            rec.right = slice(ij1 - rj0, None).indices(ncols)[0] if ij1 < rj1 else 1 << 30
            rec.p0, rec.p1 = px, px + s.width
            rec.p2, rec.p3 = py, py + s.height
            if is_custom:
                if rec.fill and not (ri0 <= rec.fi0 and rec.fi1 <= ri1 and rj0 <= rec.fj0 and rec.fj1 <= rj1):
                    raise NotImplementedError("custom-material rectangle whose fill box leaves its cell box")
                rec.custom_off = len(custom)
                for i in range(ri0, ri1):
                    for j in range(rj0, rj1):
                        custom.append(material_triple(mat, x_centers[j], y_centers[i]))
        elif is_custom:
            # the reference only evaluates custom materials on the rectangle path;
            # elsewhere the None material raises and the structure is skipped
            display_status(f"Warning: CustomMaterial on {type(s).__name__} is not rasterised", "warning")
            continue
        elif hasattr(s, "radius"):
            rec.kind = nat.BZ_SHAPE_CIRCLE
            rec.i0, rec.i1, rec.j0, rec.j1 = i0, i1, j0, j1
            rec.p0, rec.p1, rec.p2 = s.position[0], s.position[1], s.radius
            rec.q = 0.3536 * cs
        elif hasattr(s, "inner_radius") and hasattr(s, "outer_radius"):
            rec.kind = nat.BZ_SHAPE_RING
            rec.i0, rec.i1, rec.j0, rec.j1 = i0, i1, j0, j1
            rec.p0, rec.p1, rec.p2, rec.p3 = s.position[0], s.position[1], s.inner_radius, s.outer_radius
            rec.q = 0.3536 * cs
        elif hasattr(s, "point_in_polygon"):
            if not getattr(s, "vertices", None):
                continue  # no exterior path: no sample can be inside
            rec.kind = nat.BZ_SHAPE_POLYGON
            rec.i0, rec.i1, rec.j0, rec.j1 = i0, i1, j0, j1
            rec.path0 = len(paths)
            rings = [s.vertices] + [p for p in getattr(s, "interiors", []) if p]
            rec.npath = len(rings)
            for ring in rings:
                paths.append((len(verts), len(ring)))
                verts.extend((float(v[0]), float(v[1])) for v in ring)
        else:
            raise NotImplementedError(f"cannot rasterise {type(s).__name__} (no point_in_polygon)")
        shapes.append(rec)
    return shapes, paths, verts, custom


def _compile_pml(design, cs: float, gw: int, gh: int, x_centers, y_centers):
    """Loop boxes of meshing.py:484-531 and the position-only PML factors per cell."""
    recs, table = [], []
    off = 0
    for b in design.boundaries:
        if not hasattr(b, "position"):
            continue
        if hasattr(b, "width") and hasattr(b, "height"):
            px, py = b.position
            i0, j0 = max(0, int(py / cs)), max(0, int(px / cs))
            i1 = min(gh, int(np.ceil((py + b.height) / cs)))
            j1 = min(gw, int(np.ceil((px + b.width) / cs)))
        elif hasattr(b, "radius"):
            cx, cy = b.position
            i0, j0 = max(0, int((cy - b.radius) / cs)), max(0, int((cx - b.radius) / cs))
            i1 = min(gh, int(np.ceil((cy + b.radius) / cs)))
            j1 = min(gw, int(np.ceil((cx + b.radius) / cs)))
        else:
            continue
        if i1 <= i0 or j1 <= j0:
            continue
        block = _pml_block(b, x_centers[j0:j1], y_centers[i0:i1])
        rec = nat.Pml2D()
        rec.i0, rec.i1, rec.j0, rec.j1 = i0, i1, j0, j1
        rec.table_off = off
        rec.sigma_factor = float(b.sigma_factor)
        recs.append(rec)
        table.append(block.reshape(-1, 2))
        off += block.shape[0] * block.shape[1]
    tab = np.concatenate(table) if table else np.zeros((0, 2))
    return recs, tab


def _pml_block(b, xs, ys) -> np.ndarray:
    """(profile, frequency_factor) per cell of a boundary's loop box; -1 where the
    boundary returns 0. Rectangle strips are separable (depth depends on one axis),
    so the scalar profile is evaluated once per column or row."""
    out = np.full((len(ys), len(xs), 2), -1.0)
    if getattr(b, "region_type", None) == "rect" and b.orientation in ("left", "right", "top", "bottom"):
        px, py = b.position
        xin = np.array([px <= x <= px + b.width for x in xs])
        yin = np.array([py <= y <= py + b.height for y in ys])
        if b.orientation in ("left", "right"):
            y_any = ys[np.argmax(yin)] if yin.any() else None
            for j, x in enumerate(xs):
                if y_any is None or not xin[j]:
                    continue
                pf = b.profile_factors(x, y_any)
                if pf is not None:
                    out[yin, j] = pf
        else:
            x_any = xs[np.argmax(xin)] if xin.any() else None
            for i, y in enumerate(ys):
                if x_any is None or not yin[i]:
                    continue
                pf = b.profile_factors(x_any, y)
                if pf is not None:
                    out[i, xin] = pf
        return out
    for i, y in enumerate(ys):
        for j, x in enumerate(xs):
            pf = b.profile_factors(x, y) if hasattr(b, "profile_factors") else None
            if pf is not None:
                out[i, j] = pf
    return out


def rasterize_2d(design, cs: float, gw: int, gh: int):
    """eps, mu, sigma float64 (gh, gw) arrays of a 2D design (meshing.py:92-536)."""
    width, height = design.width, design.height
    xc = np.linspace(0.5 * cs, width - 0.5 * cs, gw)
    yc = np.linspace(0.5 * cs, height - 0.5 * cs, gh)
    bg = (1.0, 1.0, 0.0)
    if design.structures and getattr(design.structures[0], "material", None) is not None:
        bg = tuple(float(v) for v in material_triple(design.structures[0].material))
    shapes, paths, verts, custom = _compile_shapes(design, cs, gw, gh, xc, yc)
    pmls, table = _compile_pml(design, cs, gw, gh, xc, yc)
    dev = _device()
    keep: list[Any] = []

    def up(a, dtype=np.float64):
        if a is None or len(a) == 0:
            return None
        t = torch.as_tensor(np.ascontiguousarray(a, dtype=dtype)).to(dev)
        keep.append(t)
        return t

    t_x, t_y = up(xc), up(yc)
    t_off = up(np.array([-0.25, 0, 0.25]) * cs)
    t_cor = up(np.array([-0.4 * cs, 0.4 * cs]))
    t_bg = up(np.array(bg))
    t_shapes = _dev_struct_array(shapes, nat.Shape2D)
    t_paths = up(np.array(paths, dtype=np.int32).reshape(-1, 2), np.int32) if paths else None
    t_verts = up(np.array(verts).reshape(-1, 2)) if verts else None
    t_custom = up(np.array(custom, dtype=np.float64).reshape(-1, 3)) if custom else None
    t_pml = _dev_struct_array(pmls, nat.Pml2D)
    t_tab = up(table) if len(table) else None
    eps = torch.empty((gh, gw), dtype=torch.float64, device=dev)
    mu = torch.empty_like(eps)
    sig = torch.empty_like(eps)
    stream = torch.cuda.current_stream().cuda_stream
    nat.rasterize2d(gw, gh, _ptr(t_x), _ptr(t_y), _ptr(t_off), _ptr(t_cor), _ptr(t_bg), _ptr(t_shapes), len(shapes),
                    _ptr(t_paths), _ptr(t_verts), _ptr(t_custom), _ptr(t_pml), len(pmls), _ptr(t_tab), float(cs),
                    EPS_0, MU_0, eps.data_ptr(), mu.data_ptr(), sig.data_ptr(), stream)
    return to_host(eps), to_host(mu), to_host(sig)


def to_host(t: torch.Tensor) -> np.ndarray:
    """A device grid as a NumPy array in page-locked host memory (the array keeps the
    pinned buffer alive), so that a simulation's upload of it runs at full copy speed."""
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t)
    return h.numpy()


class RegularGrid(BaseMeshGrid):
    """2D material grid of a design at a uniform resolution."""

    def __init__(self, design, resolution):
        super().__init__(design, resolution)
        gw = int(design.width / resolution)
        gh = int(design.height / resolution)
        if gw < 1 or gh < 1:
            raise ValueError(f"design is smaller than one cell at resolution {resolution}")
        self.permittivity, self.permeability, self.conductivity = rasterize_2d(design, resolution, gw, gh)
        self.shape = self.permittivity.shape
        self.dx = resolution
        self.dy = resolution

    def show(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")


class RegularGrid3D(BaseMeshGrid):
    """3D material grid [z, y, x] (meshing.py:569-893); see meshing3d for the two
    rasterisation modes (reference semantics by default, ``extrude=True`` for the
    physically extruded stack)."""

    def __init__(self, design, resolution_xy=None, resolution_z=None, **kwargs):
        from .meshing3d import init_regular_grid_3d

        init_regular_grid_3d(self, design, resolution_xy, resolution_z, **kwargs)

    def get_2d_slice(self, z_index=None, z_position=None):
        if z_index is None and z_position is None:
            z_index = self.shape[0] // 2
        elif z_position is not None:
            z_index = max(0, min(self.shape[0] - 1, int(z_position / self.resolution_z)))
        return {"permittivity": self.permittivity[z_index], "permeability": self.permeability[z_index],
                "conductivity": self.conductivity[z_index]}

    def show(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")


def create_mesh(design, resolution, auto_select=True, force_3d=False):
    if force_3d or (auto_select and design.is_3d and design.depth > 0):
        return RegularGrid3D(design, resolution)
    return RegularGrid(design, resolution)


def mesh_2d(design, resolution):
    return RegularGrid(design, resolution)


def mesh_3d(design, resolution_xy, resolution_z=None):
    return RegularGrid3D(design, resolution_xy, resolution_z)
