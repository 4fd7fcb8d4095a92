"""Geometry primitives (beamz/design/structures.py:6-454).

Vertices are stored as (x, y, z) tuples. The exterior path is made counter-
clockwise (by the sign of its shoelace area) when it has three or more
vertices; hole paths keep their given orientation. These conventions matter to
the rasteriser, which reproduces the reference's per-sample inside tests
exactly, so vertex lists are built with the same NumPy expressions.
"""
from __future__ import annotations

import numpy as np

__all__ = ["Polygon", "Rectangle", "Circle", "Ring", "CircularBend", "Taper"]


def _as_xyz(vertices):
    out = []
    for v in vertices:
        if len(v) == 2:
            out.append((v[0], v[1], 0.0))
        elif len(v) == 3:
            out.append(tuple(v))
        else:
            raise ValueError(f"Vertex must have 2 or 3 coordinates, got {len(v)}")
    return out


def _signed_area2(xy):
    acc = 0
    n = len(xy)
    for i in range(n):
        j = (i + 1) % n
        acc += xy[i][0] * xy[j][1]
        acc -= xy[j][0] * xy[i][1]
    return acc


def _point_in_path(x, y, path):
    """Even-odd ray crossing test of one closed path (structures.py:178-196)."""
    if not path:
        return False
    n = len(path)
    inside = False
    p1x, p1y = path[0][0], path[0][1]
    for i in range(n + 1):
        p2x, p2y = path[i % n][0], path[i % n][1]
        if y > min(p1y, p2y) and y <= max(p1y, p2y) and x <= max(p1x, p2x):
            xinters = (y - p1y) * (p2x - p1x) / (p2y - p1y) + p1x if p1y != p2y else p1x
            if p1x == p2x or x <= xinters:
                inside = not inside
        p1x, p1y = p2x, p2y
    return inside


def _rotated(points, angle_deg, axis, centre):
    a = np.radians(angle_deg)
    ca, sa = np.cos(a), np.sin(a)
    cx, cy, cz = centre
    if axis == "z":
        return [(cx + (v[0] - cx) * ca - (v[1] - cy) * sa, cy + (v[0] - cx) * sa + (v[1] - cy) * ca, v[2])
                for v in points]
    if axis == "x":
        return [(v[0], cy + (v[1] - cy) * ca - (v[2] - cz) * sa, cz + (v[1] - cy) * sa + (v[2] - cz) * ca)
                for v in points]
    if axis == "y":
        return [(cx + (v[0] - cx) * ca + (v[2] - cz) * sa, v[1], cz - (v[0] - cx) * sa + (v[2] - cz) * ca)
                for v in points]
    raise ValueError(f"Invalid rotation axis '{axis}'. Must be 'x', 'y', or 'z'.")


class Polygon:
    def __init__(self, vertices=None, material=None, color=None, optimize=False, interiors=None, depth=0, z=0):
        self.vertices = self._exterior(vertices if vertices is not None else [], z)
        self.interiors = [[(v[0], v[1], v[2] if len(v) > 2 else z) for v in _as_xyz(p)] if p else []
                          for p in (interiors if interiors is not None else [])]
        self.material = material
        self.optimize = optimize
        self.color = color if color is not None else "#5c7ab3"
        self.depth = depth if depth is not None else 0
        self.z = z if z is not None else 0

    @staticmethod
    def _exterior(vertices, z=0):
        if not vertices:
            return []
        v3 = _as_xyz(vertices)
        xy = [(v[0], v[1]) for v in v3]
        if len(xy) >= 3:
            if _signed_area2(xy) < 0:
                xy = xy[::-1]
            # z is re-attached by position in the original list, as the reference does
            v3 = [(x, y, v3[i][2] if len(v3[i]) > 2 else z) for i, (x, y) in enumerate(xy)]
        return v3

    def _centroid(self):
        n = len(self.vertices)
        return (sum(v[0] for v in self.vertices) / n, sum(v[1] for v in self.vertices) / n,
                sum(v[2] for v in self.vertices) / n)

    def shift(self, x, y, z=0):
        if self.vertices:
            self.vertices = [(v[0] + x, v[1] + y, v[2] + z) for v in self.vertices]
        self.interiors = [[(v[0] + x, v[1] + y, v[2] + z) for v in p] for p in self.interiors if p]
        return self

    def scale(self, s_x, s_y=None, s_z=None):
        if s_y is None:
            s_y = s_x
        if s_z is None:
            s_z = 1.0 if s_y != s_x else s_x
        if self.vertices:
            cx, cy, cz = self._centroid()
            f = lambda v: (cx + (v[0] - cx) * s_x, cy + (v[1] - cy) * s_y, cz + (v[2] - cz) * s_z)  # noqa: E731
            self.vertices = [f(v) for v in self.vertices]
            self.interiors = [[f(v) for v in p] for p in self.interiors if p]
        return self

    def rotate(self, angle, axis="z", point=None):
        if self.vertices:
            if point is None:
                centre = self._centroid()
            else:
                centre = (point[0], point[1], point[2] if len(point) > 2 else 0)
            self.vertices = _rotated(self.vertices, angle, axis, centre)
            self.interiors = [_rotated(p, angle, axis, centre) for p in self.interiors if p]
        return self

    def copy(self):
        return Polygon(vertices=list(self.vertices) if self.vertices else [],
                       interiors=[list(p) for p in self.interiors if p], material=self.material, color=self.color,
                       optimize=self.optimize, depth=self.depth, z=self.z)

    def get_bounding_box(self):
        if not self.vertices:
            return (0, 0, 0, 0, 0, 0)
        xs = [v[0] for v in self.vertices]
        ys = [v[1] for v in self.vertices]
        zs = [v[2] for v in self.vertices]
        return (min(xs), min(ys), min(zs), max(xs), max(ys), max(zs))

    def point_in_polygon(self, x, y, z=None):
        if not self.vertices or not _point_in_path(x, y, self.vertices):
            return False
        return not any(p and _point_in_path(x, y, p) for p in self.interiors)

    def add_to_plot(self, *args, **kwargs):
        raise NotImplementedError("plotting is not part of beamz_b200")


def _pos3(position, z=None):
    if len(position) == 2:
        position = (position[0], position[1], 0.0 if z is None else z)
    elif len(position) == 3:
        position = tuple(position) if z is None else (position[0], position[1], z)
    else:
        raise ValueError("Position must be (x,y) or (x,y,z)")
    return position


class Rectangle(Polygon):
    def __init__(self, position=(0, 0, 0), width=1, height=1, depth=1, material=None, color=None, is_pml=False,
                 optimize=False, z=None):
        position = _pos3(position, z)
        x, y, zp = position
        verts = [(x, y, zp), (x + width, y, zp), (x + width, y + height, zp), (x, y + height, zp)]
        super().__init__(vertices=verts, material=material, color=color, optimize=optimize, depth=depth, z=zp)
        self.position = position
        self.width = width
        self.height = height
        self.depth = depth
        self.is_pml = is_pml

    def get_bounding_box(self):
        if not self.vertices:
            x, y, z = self.position
            return (x, y, z, x + self.width, y + self.height, z + self.depth)
        return super().get_bounding_box()

    def shift(self, x, y, z=0):
        self.position = (self.position[0] + x, self.position[1] + y, self.position[2] + z)
        return super().shift(x, y, z)

    def _refit_box(self):
        xs = [v[0] for v in self.vertices]
        ys = [v[1] for v in self.vertices]
        zs = [v[2] for v in self.vertices]
        self.position = (min(xs), min(ys), min(zs))
        return max(xs) - min(xs), max(ys) - min(ys), max(zs) - min(zs)

    def rotate(self, angle, axis="z", point=None):
        super().rotate(angle, axis, point)
        self.width, self.height, self.depth = self._refit_box()
        return self

    def scale(self, s_x, s_y=None, s_z=None):
        if s_y is None:
            s_y = s_x
        if s_z is None:
            s_z = 1.0 if s_y != s_x else s_x
        super().scale(s_x, s_y, s_z)
        self.width *= s_x
        self.height *= s_y
        self.depth *= s_z
        return self

    def copy(self):
        r = Rectangle(self.position, self.width, self.height, self.depth, self.material, self.color, self.is_pml,
                      self.optimize)
        r.vertices = [tuple(v) for v in self.vertices]
        return r


def _circle_points(cx, cy, cz, r, theta):
    return [(cx + r * np.cos(t), cy + r * np.sin(t), cz) for t in theta]


class Circle(Polygon):
    def __init__(self, position=(0, 0), radius=1, points=32, material=None, color=None, optimize=False, depth=0, z=0):
        position = _pos3(position)
        theta = np.linspace(0, 2 * np.pi, points, endpoint=False)
        super().__init__(vertices=_circle_points(*position, radius, theta), material=material, color=color,
                         optimize=optimize, depth=depth, z=z)
        self.position = position
        self.radius = radius
        self.points = points

    def shift(self, x, y, z=0):
        self.position = (self.position[0] + x, self.position[1] + y, self.position[2] + z)
        return super().shift(x, y, z)

    def scale(self, s_x, s_y=None, s_z=None):
        self.radius *= s_x
        theta = np.linspace(0, 2 * np.pi, self.points, endpoint=False)
        self.vertices = _circle_points(*self.position, self.radius, theta)
        return self

    def copy(self):
        return Circle(position=self.position, radius=self.radius, points=self.points, material=self.material,
                      color=self.color, optimize=self.optimize, depth=self.depth, z=self.z)


class Ring(Polygon):
    def __init__(self, position=(0, 0), inner_radius=1, outer_radius=2, material=None, color=None, optimize=False,
                 points=256, depth=0, z=None):
        position = _pos3(position, z)
        theta = np.linspace(0, 2 * np.pi, points, endpoint=False)
        outer = _circle_points(*position, outer_radius, theta)
        inner_cw = _circle_points(*position, inner_radius, theta[::-1])
        super().__init__(vertices=outer, interiors=[inner_cw] if inner_cw else [], material=material, color=color,
                         optimize=optimize, depth=depth, z=position[2])
        self.points = points
        self.position = position
        self.inner_radius = inner_radius
        self.outer_radius = outer_radius

    def shift(self, x, y, z=0):
        self.position = (self.position[0] + x, self.position[1] + y, self.position[2] + z)
        return super().shift(x, y, z)

    def scale(self, s_x, s_y=None, s_z=None):
        self.inner_radius *= s_x
        self.outer_radius *= s_x
        theta = np.linspace(0, 2 * np.pi, self.points, endpoint=False)
        self.vertices = _circle_points(*self.position, self.outer_radius, theta)
        self.interiors = [_circle_points(*self.position, self.inner_radius, theta[::-1])]
        return self

    def copy(self):
        return Ring(position=self.position, inner_radius=self.inner_radius, outer_radius=self.outer_radius,
                    material=self.material, color=self.color, optimize=self.optimize, points=self.points,
                    depth=self.depth, z=self.z)


class CircularBend(Polygon):
    def __init__(self, position=(0, 0), inner_radius=1, outer_radius=2, angle=90, rotation=0, material=None,
                 facecolor=None, optimize=False, points=64, depth=0, z=0):
        position = _pos3(position)
        self.points = points
        self.position = position
        self.inner_radius = inner_radius
        self.outer_radius = outer_radius
        self.angle = angle
        self.rotation = rotation
        super().__init__(vertices=self._arc_vertices(), material=material, color=facecolor, optimize=optimize,
                         depth=depth, z=z)

    def _arc_vertices(self):
        theta = np.linspace(0, np.radians(self.angle), self.points)
        rot = np.radians(self.rotation)
        cx, cy, cz = self.position
        outer = [(cx + self.outer_radius * np.cos(t + rot), cy + self.outer_radius * np.sin(t + rot), cz)
                 for t in theta]
        inner = [(cx + self.inner_radius * np.cos(t + rot), cy + self.inner_radius * np.sin(t + rot), cz)
                 for t in theta[::-1]]
        return outer + inner

    def shift(self, x, y, z=0):
        self.position = (self.position[0] + x, self.position[1] + y, self.position[2] + z)
        return super().shift(x, y, z)

    def rotate(self, angle, axis="z", point=None):
        if axis == "z":
            self.rotation = (self.rotation + angle) % 360
        return super().rotate(angle, axis, point or self.position)

    def scale(self, s_x, s_y=None, s_z=None):
        self.inner_radius *= s_x
        self.outer_radius *= s_x
        self.vertices = self._arc_vertices()
        return self

    def copy(self):
        return CircularBend(self.position, self.inner_radius, self.outer_radius, self.angle, self.rotation,
                            self.material, self.color, self.optimize, self.points, self.depth, self.z)


class Taper(Polygon):
    def __init__(self, position=(0, 0), input_width=1, output_width=0.5, length=1, material=None, color=None,
                 optimize=False, depth=0, z=0):
        position = _pos3(position)
        x, y, zp = position
        verts = [(x, y - input_width / 2, zp), (x + length, y - output_width / 2, zp),
                 (x + length, y + output_width / 2, zp), (x, y + input_width / 2, zp)]
        super().__init__(vertices=verts, material=material, color=color, optimize=optimize, depth=depth, z=zp)
        self.position = position
        self.input_width = input_width
        self.output_width = output_width
        self.length = length

    def rotate(self, angle, axis="z", point=None):
        super().rotate(angle, axis, point)
        xs = [v[0] for v in self.vertices]
        self.position = (min(xs), min(v[1] for v in self.vertices), min(v[2] for v in self.vertices))
        self.length = max(xs) - min(xs)
        return self

    def copy(self):
        t = Taper(self.position, self.input_width, self.output_width, self.length, self.material, self.color,
                  self.optimize, self.depth, self.z)
        t.vertices = [tuple(v) for v in self.vertices]
        return t
