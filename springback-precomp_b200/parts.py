"""Target part shapes of the forming workloads: the height fields z(x, y)
(z <= 0 below the sheet plane) of the four part families the reference's
data generation draws from (python/precomp/geometry/parts.py:63-639):

- TruncatedCone: a circular frustum, `top_radius` where the straight wall,
  extended, meets the sheet plane; fillets at rim and floor;
- EllipticCone: the same over an ellipse, its level sets the ellipse's
  parallel curves (the wall angle the same all round);
- Pyramid: a rectangular frustum whose plan corners are rounded;
- Dome: a spherical cap (ellipsoidal with `aspect` != 1) blended into the
  flange by a rim fillet.

The wall of the three frusta is one C1 profile z = g(w) of the inward
distance w from the nominal opening: flat (z = 0) for w below the rim
fillet, a circular arc, the straight wall at the wall angle, a second arc,
and the flat floor at z = -depth. These formulas are the families'
definitions, so they are the reference's; the code is written from them.
The forming workloads use them to place the sheet and the tools; nothing on
the element loop's path depends on them.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, Sequence, Tuple

import numpy as np


class WallProfile:
    """z = g(w): the polyline through (w_k, z_k) (w increasing), horizontal
    before the first and after the last vertex, each vertex k rounded by a
    circular arc of radius r_k tangent to its two segments."""

    def __init__(self, vertices: Sequence[Tuple[float, float]], radii: Sequence[float]):
        v = np.asarray(vertices, dtype=float)
        if v.ndim != 2 or v.shape[1] != 2 or len(v) < 1 or len(radii) != len(v):
            raise ValueError("one fillet radius per (w, z) vertex")
        if np.any(np.diff(v[:, 0]) <= 0):
            raise ValueError("the vertices' w must increase strictly")
        self.w = v[:, 0].copy()
        self.z = v[:, 1].copy()
        slopes = np.concatenate([[0.0], np.diff(self.z) / np.diff(self.w), [0.0]])
        self.slopes = slopes
        angle = np.arctan(slopes)
        self.arcs = []
        self.tangents = np.zeros(len(v))
        for k, r in enumerate(radii):
            turn = angle[k + 1] - angle[k]
            if r <= 0.0 or abs(turn) < 1e-15:
                self.arcs.append(None)
                continue
            # The arc meets the incoming segment and the outgoing one at a
            # distance T = r tan(|turn| / 2) from the vertex; its centre lies
            # r from the first touch point along the segment's normal, on the
            # side the profile turns to.
            T = r * math.tan(abs(turn) / 2.0)
            self.tangents[k] = T
            a_in, a_out = angle[k], angle[k + 1]
            w0 = self.w[k] - T * math.cos(a_in)
            z0 = self.z[k] - T * math.sin(a_in)
            w1 = self.w[k] + T * math.cos(a_out)
            side = 1.0 if turn > 0 else -1.0
            cw = w0 - side * r * math.sin(a_in)
            cz = z0 + side * r * math.cos(a_in)
            self.arcs.append((w0, w1, cw, cz, r, turn > 0))
        for k in range(1, len(v)):
            seg = math.hypot(self.w[k] - self.w[k - 1], self.z[k] - self.z[k - 1])
            if self.tangents[k - 1] + self.tangents[k] > seg * (1.0 + 1e-12):
                raise ValueError("the fillets of neighbouring corners overlap")

    @property
    def w_first(self) -> float:
        return float(self.w[0] - self.tangents[0])

    @property
    def w_last(self) -> float:
        return float(self.w[-1] + self.tangents[-1])

    def __call__(self, w) -> np.ndarray:
        w = np.asarray(w, dtype=float)
        z = np.interp(w, self.w, self.z)
        for arc in self.arcs:
            if arc is None:
                continue
            w0, w1, cw, cz, r, up = arc
            on = (w >= w0) & (w <= w1)
            if np.any(on):
                root = np.sqrt(np.maximum(r * r - (w[on] - cw) ** 2, 0.0))
                z[on] = cz - root if up else cz + root
        return z


def wall_profile(wall_angle_deg: float, depth: float, top_fillet: float, bottom_fillet: float) -> WallProfile:
    run = depth / math.tan(math.radians(wall_angle_deg))
    return WallProfile([(0.0, 0.0), (run, -depth)], [top_fillet, bottom_fillet])


def ellipse_inward_distance(x, y, a: float, b: float, halvings: int = 100) -> np.ndarray:
    """Signed distance from (x, y) to the ellipse (x/a)^2 + (y/b)^2 = 1,
    positive inside: the closest point by bisection on the one-dimensional
    root of the published method of D. Eberly ("Distance from a point to an
    ellipse, an ellipsoid, or a hyperellipsoid", Geometric Tools), with the
    points on the axes in closed form."""
    x = np.asarray(x, dtype=float)
    y = np.asarray(y, dtype=float)
    x, y = np.broadcast_arrays(x, y)
    swap = b > a
    e0, e1 = (b, a) if swap else (a, b)
    p0 = np.abs(y if swap else x)
    p1 = np.abs(x if swap else y)
    d = np.empty(p0.shape)
    gen = (p0 > 0) & (p1 > 0)
    if np.any(gen):
        z0, z1 = p0[gen] / e0, p1[gen] / e1
        g = z0 * z0 + z1 * z1 - 1.0
        ratio = (e0 / e1) ** 2
        n0 = ratio * z0
        lo = z1 - 1.0
        hi = np.where(g < 0, 0.0, np.hypot(n0, z1) - 1.0)
        for _ in range(halvings):
            mid = 0.5 * (lo + hi)
            f = (n0 / (mid + ratio)) ** 2 + (z1 / (mid + 1.0)) ** 2 - 1.0
            lo = np.where(f > 0, mid, lo)
            hi = np.where(f > 0, hi, mid)
        t = 0.5 * (lo + hi)
        q0 = ratio * p0[gen] / (t + ratio)
        q1 = p1[gen] / (t + 1.0)
        d[gen] = np.hypot(q0 - p0[gen], q1 - p1[gen])
    minor = (p0 == 0) & (p1 > 0)
    d[minor] = np.abs(p1[minor] - e1)
    major = p1 == 0
    if np.any(major):
        pm = p0[major]
        num = e0 * pm
        den = e0 * e0 - e1 * e1
        dm = np.abs(pm - e0)
        inner = num < den
        if np.any(inner):
            s = num[inner] / den
            dm[inner] = np.hypot(e0 * s - pm[inner], e1 * np.sqrt(np.maximum(1.0 - s * s, 0.0)))
        d[major] = dm
    inside = (x / a) ** 2 + (y / b) ** 2 < 1.0
    return np.where(inside, d, -d)


def rounded_rectangle_inward_distance(x, y, half_x: float, half_y: float, corner: float) -> np.ndarray:
    """Inward distance from a rounded rectangle's outline (exact outside it
    and down to `corner` inside; capped there)."""
    qx = np.maximum(np.abs(np.asarray(x, float)) - (half_x - corner), 0.0)
    qy = np.maximum(np.abs(np.asarray(y, float)) - (half_y - corner), 0.0)
    return corner - np.hypot(qx, qy)


@dataclasses.dataclass(frozen=True)
class TruncatedCone:
    top_radius: float
    wall_angle_deg: float
    depth: float
    top_fillet: float = 0.005
    bottom_fillet: float = 0.005
    family = "truncated_cone"

    @property
    def profile(self) -> WallProfile:
        return wall_profile(self.wall_angle_deg, self.depth, self.top_fillet, self.bottom_fillet)

    def height(self, x, y) -> np.ndarray:
        return self.profile(self.top_radius - np.hypot(np.asarray(x, float), np.asarray(y, float)))

    def footprint_radius(self) -> float:
        return self.top_radius - self.profile.w_first

    @classmethod
    def with_footprint(cls, footprint_radius: float, wall_angle_deg: float, depth: float, top_fillet: float,
                       bottom_fillet: float) -> "TruncatedCone":
        """The cone whose rim fillet leaves the sheet plane at `footprint_radius`."""
        t = -wall_profile(wall_angle_deg, depth, top_fillet, bottom_fillet).w_first
        return cls(footprint_radius - t, wall_angle_deg, depth, top_fillet, bottom_fillet)


@dataclasses.dataclass(frozen=True)
class EllipticCone:
    semi_axis_x: float
    semi_axis_y: float
    wall_angle_deg: float
    depth: float
    top_fillet: float = 0.004
    bottom_fillet: float = 0.004
    family = "elliptic_cone"

    @property
    def profile(self) -> WallProfile:
        return wall_profile(self.wall_angle_deg, self.depth, self.top_fillet, self.bottom_fillet)

    def height(self, x, y) -> np.ndarray:
        return self.profile(ellipse_inward_distance(x, y, self.semi_axis_x, self.semi_axis_y))

    def footprint_radius(self) -> float:
        return max(self.semi_axis_x, self.semi_axis_y) - self.profile.w_first


@dataclasses.dataclass(frozen=True)
class Pyramid:
    half_width_x: float
    half_width_y: float
    wall_angle_deg: float
    depth: float
    corner_radius: float
    top_fillet: float = 0.004
    bottom_fillet: float = 0.004
    family = "pyramid"

    @property
    def profile(self) -> WallProfile:
        return wall_profile(self.wall_angle_deg, self.depth, self.top_fillet, self.bottom_fillet)

    def height(self, x, y) -> np.ndarray:
        w = rounded_rectangle_inward_distance(x, y, self.half_width_x, self.half_width_y, self.corner_radius)
        return self.profile(w)

    def footprint_radius(self) -> float:
        t = -self.profile.w_first
        return math.hypot(self.half_width_x - self.corner_radius, self.half_width_y - self.corner_radius) + \
            self.corner_radius + t


@dataclasses.dataclass(frozen=True)
class Dome:
    opening_radius: float
    depth: float
    rim_fillet: float = 0.01
    aspect: float = 1.0
    family = "dome"

    @property
    def sphere_radius(self) -> float:
        a, d = self.opening_radius, self.depth
        return (a * a + d * d) / (2.0 * d) - self.rim_fillet

    def height(self, x, y) -> np.ndarray:
        a, d, f = self.opening_radius, self.depth, self.rim_fillet
        R = self.sphere_radius
        rho = np.hypot(np.asarray(x, float), np.asarray(y, float) / self.aspect)
        # The cap (centre R - d above the pole) meets the rim fillet (centre
        # f below the sheet plane at rho = a) where their circles touch.
        rho_t = a * R / (R + f)
        z = np.zeros_like(rho)
        cap = rho <= rho_t
        z[cap] = (R - d) - np.sqrt(np.maximum(R * R - rho[cap] ** 2, 0.0))
        fil = (rho > rho_t) & (rho < a)
        z[fil] = -f + np.sqrt(np.maximum(f * f - (rho[fil] - a) ** 2, 0.0))
        return z

    def footprint_radius(self) -> float:
        return self.opening_radius * max(1.0, self.aspect)


FAMILIES: Dict[str, type] = {c.family: c for c in (TruncatedCone, EllipticCone, Pyramid, Dome)}
