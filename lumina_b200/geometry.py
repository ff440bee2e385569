"""Dipole-lattice generators (inputs of the solve).

``discretise_primitive`` follows crates/lumina-geometry/src/discretise.rs:27-58:
a cubic lattice centred on the bounding-box midpoint, x = cx + ix*spacing
for ix in [-nx, nx], nx = floor((max - cx)/spacing), kept when
``contains`` holds (primitives.rs:80-212, inclusive comparisons).  The
arithmetic is elementwise IEEE FP64 in the reference's order, so positions are
bit-identical to the reference's.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence

import numpy as np


@dataclass
class Sphere:
    centre: Sequence[float]
    radius: float

    def bounding_box(self):
        c, r = self.centre, self.radius
        return [c[0] - r, c[1] - r, c[2] - r], [c[0] + r, c[1] + r, c[2] + r]

    def contains(self, p: np.ndarray) -> np.ndarray:
        dx = p[:, 0] - self.centre[0]
        dy = p[:, 1] - self.centre[1]
        dz = p[:, 2] - self.centre[2]
        return dx * dx + dy * dy + dz * dz <= self.radius * self.radius


@dataclass
class Cuboid:
    centre: Sequence[float]
    half_extents: Sequence[float]

    def bounding_box(self):
        c, h = self.centre, self.half_extents
        return [c[i] - h[i] for i in range(3)], [c[i] + h[i] for i in range(3)]

    def contains(self, p):
        c, h = self.centre, self.half_extents
        return ((np.abs(p[:, 0] - c[0]) <= h[0]) & (np.abs(p[:, 1] - c[1]) <= h[1])
                & (np.abs(p[:, 2] - c[2]) <= h[2]))


@dataclass
class Ellipsoid:
    centre: Sequence[float]
    semi_axes: Sequence[float]

    def bounding_box(self):
        c, s = self.centre, self.semi_axes
        return [c[i] - s[i] for i in range(3)], [c[i] + s[i] for i in range(3)]

    def contains(self, p):
        c, s = self.centre, self.semi_axes
        dx = (p[:, 0] - c[0]) / s[0]
        dy = (p[:, 1] - c[1]) / s[1]
        dz = (p[:, 2] - c[2]) / s[2]
        return dx * dx + dy * dy + dz * dz <= 1.0


def _unit(a):
    ln = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    return ln, ([a[0] / ln, a[1] / ln, a[2] / ln] if ln > 1e-15 else [0.0, 0.0, 1.0])


@dataclass
class Cylinder:
    base_centre: Sequence[float]
    axis: Sequence[float]
    length: float
    radius: float

    def bounding_box(self):
        _, ax = _unit(self.axis)
        top = [self.base_centre[i] + ax[i] * self.length for i in range(3)]
        lo, hi = [], []
        for i in range(3):
            r_ext = self.radius * math.sqrt(max(1.0 - ax[i] * ax[i], 0.0))
            lo.append(min(self.base_centre[i], top[i]) - r_ext)
            hi.append(max(self.base_centre[i], top[i]) + r_ext)
        return lo, hi

    def contains(self, p):
        ln, ax = _unit(self.axis)
        if ln < 1e-15:
            return np.zeros(p.shape[0], bool)
        dp = p - np.asarray(self.base_centre, np.float64)[None, :]
        proj = dp[:, 0] * ax[0] + dp[:, 1] * ax[1] + dp[:, 2] * ax[2]
        perp = dp[:, 0] * dp[:, 0] + dp[:, 1] * dp[:, 1] + dp[:, 2] * dp[:, 2] - proj * proj
        return (proj >= 0.0) & (proj <= self.length) & (perp <= self.radius * self.radius)


@dataclass
class Helix:
    """Right-handed helical wire (primitives.rs:126-211)."""
    base_centre: Sequence[float]
    axis: Sequence[float]
    radius: float
    pitch: float
    turns: float
    wire_radius: float

    def bounding_box(self):
        _, ax = _unit(self.axis)
        total_h = self.pitch * self.turns
        outer = self.radius + self.wire_radius
        lo, hi = [], []
        for i in range(3):
            r_ext = outer * math.sqrt(max(1.0 - ax[i] * ax[i], 0.0))
            base = self.base_centre[i]
            top = base + total_h * ax[i]
            lo.append(min(base, top) - r_ext - self.wire_radius)
            hi.append(max(base, top) + r_ext + self.wire_radius)
        return lo, hi

    def contains(self, p, chunk=1 << 16):
        ln, ax = _unit(self.axis)
        if ln < 1e-15:
            return np.zeros(p.shape[0], bool)
        seed = [1.0, 0.0, 0.0] if abs(ax[0]) < 0.9 else [0.0, 1.0, 0.0]
        dsa = seed[0] * ax[0] + seed[1] * ax[1] + seed[2] * ax[2]
        ur = [seed[i] - dsa * ax[i] for i in range(3)]
        ul = math.sqrt(ur[0] ** 2 + ur[1] ** 2 + ur[2] ** 2)
        u = [ur[i] / ul for i in range(3)]
        v = [ax[1] * u[2] - ax[2] * u[1], ax[2] * u[0] - ax[0] * u[2], ax[0] * u[1] - ax[1] * u[0]]
        out = np.zeros(p.shape[0], bool)
        two_pi = 2.0 * math.pi
        t_max = two_pi * self.turns
        total_h = self.pitch * self.turns
        for s in range(0, p.shape[0], chunk):
            dp = p[s:s + chunk] - np.asarray(self.base_centre, np.float64)[None, :]
            z = dp[:, 0] * ax[0] + dp[:, 1] * ax[1] + dp[:, 2] * ax[2]
            ok = ~((z < -self.wire_radius) | (z > total_h + self.wire_radius))
            pu = dp[:, 0] * u[0] + dp[:, 1] * u[1] + dp[:, 2] * u[2]
            pv = dp[:, 0] * v[0] + dp[:, 1] * v[1] + dp[:, 2] * v[2]
            tg = z * two_pi / self.pitch if self.pitch > 1e-15 else np.zeros_like(z)
            tg = np.clip(tg, 0.0, t_max)
            t_lo = np.maximum(tg - two_pi, 0.0)
            t_hi = np.minimum(tg + two_pi, t_max)
            best = np.full(z.shape, np.inf)
            for si in range(33):
                t = t_lo + (t_hi - t_lo) * si / 32.0
                cz = t * self.pitch / two_pi
                du = pu - self.radius * np.cos(t)
                dv = pv - self.radius * np.sin(t)
                dz = z - cz
                best = np.minimum(best, dz * dz + du * du + dv * dv)
            out[s:s + chunk] = ok & (best <= self.wire_radius * self.wire_radius)
        return out


def discretise_primitive(prim, spacing: float) -> np.ndarray:
    """Centred cubic lattice clipped to ``prim`` (discretise.rs:27-58)."""
    if not spacing > 0.0:
        raise ValueError("Dipole spacing must be positive")
    lo, hi = prim.bounding_box()
    c = [0.5 * (lo[i] + hi[i]) for i in range(3)]
    n = [int(math.floor((hi[i] - c[i]) / spacing)) for i in range(3)]
    ix = np.arange(-n[0], n[0] + 1, dtype=np.float64)
    iy = np.arange(-n[1], n[1] + 1, dtype=np.float64)
    iz = np.arange(-n[2], n[2] + 1, dtype=np.float64)
    xs = c[0] + ix * spacing
    ys = c[1] + iy * spacing
    zs = c[2] + iz * spacing
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")  # ix outer, iz inner (reference order)
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    return np.ascontiguousarray(pts[prim.contains(pts)])


def cell_centred_cuboid(size: Sequence[float], spacing: float, centre=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Cells of edge ``spacing`` filling a box of ``size`` exactly; one dipole
    at each cell centre (60 x 50 x 10 nm at 1 nm gives 30,000 dipoles)."""
    counts = [int(round(size[i] / spacing)) for i in range(3)]
    axes = [centre[i] - 0.5 * size[i] + (np.arange(counts[i], dtype=np.float64) + 0.5) * spacing
            for i in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    return np.ascontiguousarray(np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1))


def rotation_zyx(rx_deg: float, ry_deg: float, rz_deg: float) -> np.ndarray:
    """R = Rz(rz) Ry(ry) Rx(rx), row-major (scene.rs:548-560 convention)."""
    rx, ry, rz = (math.radians(v) for v in (rx_deg, ry_deg, rz_deg))
    cx, sx, cy, sy, cz, sz = math.cos(rx), math.sin(rx), math.cos(ry), math.sin(ry), math.cos(rz), math.sin(rz)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


_GL16_X = [0.0950125098376374, 0.2816035507792589, 0.4580167776572274, 0.6178762444026438,
           0.7554044083550030, 0.8656312023878318, 0.9445750230732326, 0.9894009349916499]
_GL16_W = [0.1894506104550685, 0.1826034150449236, 0.1691565193950025, 0.1495959888165767,
           0.1246289712555339, 0.0951585116824928, 0.0622535239386479, 0.0271524594117541]


def ellipsoid_depol_factors(semi_axes: Sequence[float]) -> list:
    """Depolarisation factors L_i = (abc/2) int ds / ((s_i^2+s) sqrt(...)),
    16-point Gauss-Legendre after s = s_i^2 (1-u^2)/u^2 (ellipsoid.rs:66-108)."""
    a, b, c = semi_axes
    a2, b2, c2 = a * a, b * b, c * c

    def integrand(si2, u):
        u2 = u * u
        qa = si2 + (a2 - si2) * u2
        qb = si2 + (b2 - si2) * u2
        qc = si2 + (c2 - si2) * u2
        return 2.0 * u2 / math.sqrt(qa * qb * qc)

    def integ(si2):
        s = 0.0
        for x, w in zip(_GL16_X, _GL16_W):
            s += 0.5 * w * integrand(si2, (1.0 + x) * 0.5)
            s += 0.5 * w * integrand(si2, (1.0 - x) * 0.5)
        return s

    pre = a * b * c * 0.5
    return [pre * integ(a2), pre * integ(b2), pre * integ(c2)]
