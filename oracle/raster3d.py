"""3D host rasteriser (test oracle, see oracle/__init__.py).

Restates beamz/simulation/meshing.py:616-781 (RegularGrid3D.__rasterize_3d__ and
_process_3d_pml) in vectorised float64 NumPy, duck-typed on the design objects so
that it runs on reference designs and on beamz_b200 designs alike:

* cell centres and the 3 x 3 x 3 sample offsets as meshing.py:627-637;
* background fill from the first structure (644-649);
* every structure in painter's order over its index box (meshing.py:679-688), each
  cell blended as ``value * (1 - f) + material * f`` with f = inside samples / 27
  (713-725); the inside test is the even-odd crossing rule of
  beamz/design/structures.py:178-207 on the xy sample, evaluated with the same
  expressions (so the same roundings) as the scalar reference;
* the PML pass: every boundary's conductivity (beamz/design/pml.py:29-62) added
  per cell where positive (757-781), sigma_max from that cell's permittivity.

Two modes:

``extrude=False`` (the reference as written). ``Rectangle.get_bounding_box`` takes
its z range from the vertices, which all sit on the base plane
(structures.py:167-176, 219-231), so only the layers around the base plane are
visited, and the inside test ignores z, so all three z samples of a visited layer
count. The PML is the 2D set replicated over z (no z faces).

``extrude=True`` (the physically intended stack, used by the 3D SOI workload). A
structure's z range is [z_base, z_base + depth) with z_base its position's z (the
base vertex's z for shapes without a 3D position); the index box's z bounds use that
range, and a z sample counts only inside it, so a cell's weight is
(xy samples inside) x (z samples inside) / 27. A graded PML is added on the two z
faces with the profile of the first rectangular xy boundary (same thickness,
polynomial order, alpha_max and sigma_factor): normalised depth
d = 1 - z / t below z = t and d = (z - (D - t)) / t above z = D - t (the larger where
both apply), conductivity sigma_max(eps) * sigma(d) / (1 + alpha(d)), added after the
xy boundaries.
"""
from __future__ import annotations

import numpy as np

EPS_0 = 8.85e-12  # beamz/const.py
MU_0 = 1.256e-6


def _skip(s) -> bool:
    if getattr(s, "is_pml", False):
        return True
    if type(s).__name__ in ("ModeSource", "GaussianSource", "Monitor"):
        return True
    return getattr(s, "material", None) is None


def _xy(v):
    return float(v[0]), float(v[1])


def _inside_path(X, Y, path):
    """Even-odd crossing test of one closed path (structures.py:178-196), elementwise
    over sample arrays X, Y with the reference's expressions."""
    pts = [_xy(v) for v in path]
    n = len(pts)
    inside = np.zeros(X.shape, dtype=bool)
    if n == 0:
        return inside
    p1x, p1y = pts[0]
    for i in range(n + 1):
        p2x, p2y = pts[i % n]
        hit = (Y > min(p1y, p2y)) & (Y <= max(p1y, p2y)) & (X <= max(p1x, p2x))
        if hit.any():
            if p1y != p2y:
                xint = (Y - p1y) * (p2x - p1x) / (p2y - p1y) + p1x
            else:
                xint = np.full(X.shape, p1x)
            cross = hit & ((p1x == p2x) | (X <= xint))
            inside ^= cross
        p1x, p1y = p2x, p2y
    return inside


def _inside(s, X, Y):
    """structures.py:198-207: inside the exterior path and outside every hole."""
    if not getattr(s, "vertices", None):
        return np.zeros(X.shape, dtype=bool)
    ok = _inside_path(X, Y, s.vertices)
    for hole in getattr(s, "interiors", None) or []:
        if hole:
            ok &= ~_inside_path(X, Y, hole)
    return ok


def _material(m):
    return float(m.permittivity), float(m.permeability), float(m.conductivity)


def _z_range(s, bbox, extrude):
    if len(bbox) == 6:
        zmin, zmax = bbox[2], bbox[5]
    else:
        zmin = zmax = 0
    if extrude:
        pos = getattr(s, "position", None)
        if pos is not None and len(pos) > 2:
            zmin = pos[2]
        elif getattr(s, "vertices", None):
            zmin = s.vertices[0][2]
        zmax = zmin + (getattr(s, "depth", 0) or 0)
    return zmin, zmax


def _profile(b, d):
    """pml.py:21-27."""
    d = min(max(d, 0.0), 1.0)
    if d < 0.05:
        sigma = 0.01 * (d / 0.05) ** 2
    else:
        sigma = ((d - 0.05) / 0.95) ** b.polynomial_order
    return sigma, b.alpha_max * d ** 2


def _position_factors(b, x, y):
    """The position-dependent part of pml.py:29-62 at one cell centre: (sigma
    profile, frequency factor), or None where the boundary contributes nothing."""
    if b.region_type == "rect":
        px, py = b.position[0], b.position[1]
        if not (px <= x <= px + b.width and py <= y <= py + b.height):
            return None
        o = b.orientation
        if o == "left":
            dist = 1.0 - (x - px) / b.width
        elif o == "right":
            dist = (x - px) / b.width
        elif o == "top":
            dist = (y - py) / b.height
        elif o == "bottom":
            dist = 1.0 - (y - py) / b.height
        else:
            return None
    else:
        cx, cy = b.position[0], b.position[1]
        r = np.hypot(x - cx, y - cy)
        if r > b.radius:
            return None
        ddx, ddy = x - cx, y - cy
        o = b.orientation
        if (o == "top-left" and (ddx > 0 or ddy < 0)) or (o == "top-right" and (ddx < 0 or ddy < 0)) or \
                (o == "bottom-left" and (ddx > 0 or ddy > 0)) or (o == "bottom-right" and (ddx < 0 or ddy > 0)):
            return None
        dist = r / b.radius
    sp, ap = _profile(b, dist)
    return sp, 1.0 / (1.0 + ap)


def _add_pml(sig, eps, prof, ff, sf, dx):
    """conductivity += sigma_max(eps) * profile * factor where positive (pml.py:44-62,
    meshing.py:772-779); eps and sig broadcast over z."""
    eta = np.sqrt(MU_0 / (EPS_0 * eps))
    smax = 1.2 / (eta * dx)
    smax = smax * sf
    cond = smax * prof
    cond = cond * ff
    pos = cond > 0
    sig[pos] = sig[pos] + cond[pos]


def rasterize3d(design, resolution_xy, resolution_z=None, extrude=False):
    """(eps, mu, sigma) arrays [z, y, x] of a 3D design."""
    rxy = float(resolution_xy)
    rz = float(resolution_z if resolution_z is not None else resolution_xy)
    W, H, D = design.width, design.height, design.depth
    gw, gh = int(W / rxy), int(H / rxy)
    gd = int(D / rz) if D > 0 else 1
    xc = np.linspace(0.5 * rxy, W - 0.5 * rxy, gw)
    yc = np.linspace(0.5 * rxy, H - 0.5 * rxy, gh)
    zc = np.linspace(0.5 * rz, D - 0.5 * rz, gd) if D > 0 else np.array([0.0])
    off = np.array([-0.25, 0, 0.25]) * rxy
    offz = np.array([-0.25, 0, 0.25]) * rz if D > 0 else np.array([0.0])
    n_samples = 9 * len(offz)
    eps, mu, sig = np.ones((gd, gh, gw)), np.ones((gd, gh, gw)), np.zeros((gd, gh, gw))
    if design.structures and getattr(design.structures[0], "material", None) is not None:
        e0, m0, c0 = _material(design.structures[0].material)
        eps.fill(e0)
        mu.fill(m0)
        sig.fill(c0)
    for s in design.structures[1:]:
        if _skip(s):
            continue
        mat = _material(s.material)
        bb = s.get_bounding_box()
        if bb is None:
            continue
        min_x, min_y = (bb[0], bb[1])
        max_x, max_y = (bb[3], bb[4]) if len(bb) == 6 else (bb[2], bb[3])
        min_z, max_z = _z_range(s, bb, extrude)
        i0, j0 = max(0, int(min_y / rxy) - 1), max(0, int(min_x / rxy) - 1)
        k0 = max(0, int(min_z / rz) - 1) if D > 0 else 0
        i1, j1 = min(gh, int(np.ceil(max_y / rxy)) + 1), min(gw, int(np.ceil(max_x / rxy)) + 1)
        k1 = min(gd, int(np.ceil(max_z / rz)) + 1) if D > 0 else 1
        if i0 >= gh or j0 >= gw or k0 >= gd or i1 <= 0 or j1 <= 0 or k1 <= 0:
            continue
        # xy samples inside, per cell of the box (the z test is separable)
        cnt = np.zeros((i1 - i0, j1 - j0), dtype=np.int64)
        for oy in off:
            Y = np.broadcast_to((yc[i0:i1] + oy)[:, None], (i1 - i0, j1 - j0))
            for ox in off:
                X = np.broadcast_to((xc[j0:j1] + ox)[None, :], (i1 - i0, j1 - j0))
                cnt += _inside(s, X, Y)
        if extrude:
            z_lo, z_hi = min_z, max_z
            wz = np.array([sum(1 for o in offz if z_lo <= zc[k] + o < z_hi) for k in range(k0, k1)], dtype=np.int64)
        else:
            wz = np.full(k1 - k0, len(offz), dtype=np.int64)
        n_in = wz[:, None, None] * cnt[None]
        hit = n_in > 0
        if not hit.any():
            continue
        bf = n_in / n_samples
        for a, v in zip((eps, mu, sig), mat):
            box = a[k0:k1, i0:i1, j0:j1]
            box[hit] = box[hit] * (1 - bf[hit]) + v * bf[hit]
    # PML: the boundaries in order, each over the whole grid (zero outside its region)
    # (the reference passes a dt estimate only to switch the frequency factor on)
    first_rect = None
    for b in getattr(design, "boundaries", None) or []:
        if not hasattr(b, "position"):
            continue
        if b.region_type == "rect" and first_rect is None:
            first_rect = b
        prof = np.full((gh, gw), -1.0)
        ff = np.ones((gh, gw))
        for i, y in enumerate(yc):
            for j in _candidate_columns(b, xc, y, rxy):
                pf = _position_factors(b, xc[j], y)
                if pf is not None:
                    prof[i, j], ff[i, j] = pf
        cols = prof >= 0
        if not cols.any():
            continue
        ii, jj = np.nonzero(cols)
        sub_sig = sig[:, ii, jj]
        _add_pml(sub_sig, eps[:, ii, jj], prof[ii, jj][None], ff[ii, jj][None], float(b.sigma_factor), rxy)
        sig[:, ii, jj] = sub_sig
    if extrude and D > 0 and first_rect is not None:
        b = first_rect
        t = b.width if b.orientation in ("left", "right") else b.height
        for k, z in enumerate(zc):
            d = max(1.0 - z / t if z <= t else -1.0, (z - (D - t)) / t if z >= D - t else -1.0)
            if d < 0:
                continue
            sp, ap = _profile(b, d)
            layer = sig[k]
            _add_pml(layer, eps[k], sp, 1.0 / (1.0 + ap), float(b.sigma_factor), rxy)
            sig[k] = layer
    return eps, mu, sig


def _candidate_columns(b, xc, y, cs):
    """Columns whose centres can lie in the boundary's region (a superset; the exact
    test is _position_factors)."""
    if b.region_type == "rect":
        lo, hi = b.position[0], b.position[0] + b.width
        if not (b.position[1] <= y <= b.position[1] + b.height):
            return ()
    else:
        lo, hi = b.position[0] - b.radius, b.position[0] + b.radius
        if abs(y - b.position[1]) > b.radius:
            return ()
    j0 = max(0, int(np.floor(lo / cs)) - 1)
    j1 = min(len(xc), int(np.ceil(hi / cs)) + 1)
    return range(j0, j1)
