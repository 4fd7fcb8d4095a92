"""3D rasterisation (beamz/simulation/meshing.py:569-893) on the GPU.

Reference mode (default) reproduces RegularGrid3D.__rasterize_3d__: every
structure is tested with its polygon at 27 samples per cell (3 x 3 in xy, 3 in z,
z ignored by the inside test) on the layers of its bounding box as the reference
computes it. For Rectangle that box is taken from the vertices, whose z is the
base plane, so a structure covers the ~2 layers around its base plane whatever
its depth; the PML is the 2D set applied to every layer (no z faces).

``extrude=True`` gives the physically intended stack: a structure fills
[z_base, z_base + depth) (its z samples are tested against that range) and a
graded PML is added on the two z faces, with the same profile as the xy faces.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import _native as nat
from ..const import EPS_0, MU_0
from ..design.materials import material_triple
from .meshing import BaseMeshGrid, _compile_pml, _dev_struct_array, _device, _ptr, to_host


def _resolutions(design, resolution_xy, resolution_z):
    if isinstance(design, (int, float)) and resolution_xy is not None and not isinstance(resolution_xy, (int, float)):
        return resolution_xy, design, design  # legacy RegularGrid3D(resolution, design)
    if resolution_xy is None:
        resolution_xy = getattr(design, "resolution", None)
        resolution_z = resolution_xy
    elif resolution_z is None:
        resolution_z = resolution_xy
    return design, resolution_xy, resolution_z


def _layer_weights(s, k0, k1, zc, offs_z, extrude):
    """z samples of each layer counted inside the structure (reference: all of them)."""
    n_zs = len(offs_z)
    if not extrude:
        return [n_zs] * (k1 - k0)
    z_lo = s.position[2] if hasattr(s, "position") and len(s.position) > 2 else (s.vertices[0][2] if s.vertices else 0)
    z_hi = z_lo + (getattr(s, "depth", 0) or 0)
    return [sum(1 for o in offs_z if z_lo <= zc[k] + o < z_hi) for k in range(k0, k1)]


def init_regular_grid_3d(grid, design, resolution_xy=None, resolution_z=None, extrude=False):
    design, rxy, rz = _resolutions(design, resolution_xy, resolution_z)
    BaseMeshGrid.__init__(grid, design, rxy)
    grid.resolution_xy, grid.resolution_z = rxy, rz
    W, H, D = design.width, design.height, design.depth
    gw, gh = int(W / rxy), int(H / rxy)
    gd = int(D / rz) if D > 0 else 1
    if min(gw, gh, gd) < 1:
        raise ValueError("design is smaller than one cell")
    xc = np.linspace(0.5 * rxy, W - 0.5 * rxy, gw)
    yc = np.linspace(0.5 * rxy, H - 0.5 * rxy, gh)
    zc = np.linspace(0.5 * rz, D - 0.5 * rz, gd) if D > 0 else np.array([0.0])
    offs_z = np.array([-0.25, 0, 0.25]) * rz if D > 0 else np.array([0.0])
    bg = (1.0, 1.0, 0.0)
    s0 = design.structures[0] if design.structures else None
    if s0 is not None and getattr(s0, "material", None) is not None:
        m = s0.material
        bg = (float(m.permittivity), float(m.permeability), float(m.conductivity))
    shapes, zw, paths, verts = [], [], [], []
    for s in design.structures[1:]:
        if getattr(s, "is_pml", False):
            continue
        if getattr(s, "material", None) is None:
            continue
        mat = tuple(float(v) for v in material_triple(s.material))
        bb = s.get_bounding_box()
        if len(bb) == 6:
            min_x, min_y, min_z, max_x, max_y, max_z = bb
        else:
            min_x, min_y, max_x, max_y = bb
            min_z = max_z = 0
        if extrude:
            z_lo = s.position[2] if hasattr(s, "position") and len(s.position) > 2 else min_z
            min_z, max_z = z_lo, z_lo + (getattr(s, "depth", 0) or 0)
        i0, j0 = max(0, int(min_y / rxy) - 1), max(0, int(min_x / rxy) - 1)
        k0 = max(0, int(min_z / rz) - 1) if D > 0 else 0
        i1, j1 = min(gh, int(np.ceil(max_y / rxy)) + 1), min(gw, int(np.ceil(max_x / rxy)) + 1)
        k1 = min(gd, int(np.ceil(max_z / rz)) + 1) if D > 0 else 1
        if i0 >= gh or j0 >= gw or k0 >= gd or i1 <= 0 or j1 <= 0 or k1 <= 0:
            continue
        if not (hasattr(s, "point_in_polygon") and getattr(s, "vertices", None)):
            continue
        rec = nat.Shape3D()
        rec.i0, rec.i1, rec.j0, rec.j1, rec.k0, rec.k1 = i0, i1, j0, j1, k0, k1
        rec.perm, rec.permb, rec.cond = mat
        rec.zw_off = len(zw)
        zw.extend(_layer_weights(s, k0, k1, zc, offs_z, extrude))
        rec.path0 = len(paths)
        rings = [s.vertices] + [p for p in getattr(s, "interiors", []) if p]
        rec.npath = len(rings)
        for ring in rings:
            paths.append((len(verts), len(ring)))
            verts.extend((float(v[0]), float(v[1])) for v in ring)
        shapes.append(rec)
    pmls, table = _compile_pml(design, rxy, gw, gh, xc, yc)
    prof_z, sf_z = None, 0.0
    if extrude and D > 0 and design.boundaries:
        ref = next((b for b in design.boundaries if getattr(b, "region_type", "") == "rect"), design.boundaries[0])
        thick = getattr(ref, "width", None) if ref.orientation in ("left", "right") else getattr(ref, "height", None)
        if thick:
            prof_z = np.full((gd, 2), -1.0)
            for k, z in enumerate(zc):
                d = max(1.0 - z / thick if z <= thick else -1.0, (z - (D - thick)) / thick if z >= D - thick else -1.0)
                if d >= 0:
                    prof_z[k] = ref.get_profile(d)[0], 1.0 / (1.0 + ref.get_profile(d)[1])
            sf_z = float(ref.sigma_factor)
    dev = _device()
    keep = []

    def up(a, dtype=np.float64):
        if a is None or len(a) == 0:
            return None
        t = torch.as_tensor(np.ascontiguousarray(a, dtype=dtype)).to(dev)
        keep.append(t)
        return t

    t_x, t_y = up(xc), up(yc)
    t_off = up(np.array([-0.25, 0, 0.25]) * rxy)
    t_bg = up(np.array(bg))
    t_sh = _dev_struct_array(shapes, nat.Shape3D)
    t_zw = up(np.array(zw, dtype=np.int32), np.int32) if zw else None
    t_paths = up(np.array(paths, dtype=np.int32).reshape(-1, 2), np.int32) if paths else None
    t_verts = up(np.array(verts).reshape(-1, 2)) if verts else None
    t_pml = _dev_struct_array(pmls, nat.Pml2D)
    t_tab = up(table) if len(table) else None
    t_pz = up(prof_z) if prof_z is not None else None
    eps = torch.empty((gd, gh, gw), dtype=torch.float64, device=dev)
    mu, sig = torch.empty_like(eps), torch.empty_like(eps)
    nat.rasterize3d(gw, gh, gd, len(offs_z), _ptr(t_x), _ptr(t_y), _ptr(t_off), _ptr(t_bg), _ptr(t_sh), len(shapes),
                    _ptr(t_zw), _ptr(t_paths), _ptr(t_verts), _ptr(t_pml), len(pmls), _ptr(t_tab), _ptr(t_pz), sf_z,
                    float(rxy), EPS_0, MU_0, eps.data_ptr(), mu.data_ptr(), sig.data_ptr(),
                    torch.cuda.current_stream().cuda_stream)
    grid.permittivity, grid.permeability, grid.conductivity = to_host(eps), to_host(mu), to_host(sig)
    grid.shape = grid.permittivity.shape
    grid.dx, grid.dy, grid.dz = rxy, rxy, rz
    grid.extrude = extrude
