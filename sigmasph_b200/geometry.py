"""Particle lattices and the analytic regions that carve them (geometry.py of the
reference, :1-561).

The lattice must be laid exactly as the reference lays it -- float64 `arange` per
axis, an 'ij' meshgrid, cast to float32 -- because the particle positions are the
inputs every parity comparison starts from.  The dogbone profile is a circular arc of
radius R from the gauge half-width to the tab half-width:

    w(s) = W_g/2 + R - sqrt(R^2 - s^2)   for |s| <= s_j = sqrt(D (2R - D)),  D = (W_t - W_g)/2
    w(s) = W_t/2                          beyond,            total length 2 (s_j + H_t)

and containment carries an absolute tolerance of 1e-6 W_t so that lattice sites lying on
the profile are kept on both sides alike.
"""
from __future__ import annotations

import numpy as np


def lattice_points(lower, size, diameter, dim=3):
    axes = [np.arange(lower[i], lower[i] + size[i], diameter) for i in range(dim)]
    grid = np.array(np.meshgrid(*axes, sparse=False, indexing="ij"), dtype=np.float32)
    return grid.reshape(dim, -1).T


class _Profile:
    axial = 1          # column of the specimen's long axis
    revolved = False

    def __init__(self, tab_width, tab_height, gauge_width, radius, centre=(0.0, 0.0, 0.0)):
        self.tab_width = float(tab_width)
        self.tab_height = float(tab_height)
        self.gauge_width = float(gauge_width)
        self.radius = float(radius)
        c = np.asarray(centre, dtype=float).ravel()
        self.centre = np.zeros(3)
        self.centre[:len(c)] = c[:3]
        if self.gauge_width <= 0.0 or self.tab_width <= 0.0 or self.tab_height <= 0.0:
            raise ValueError("dogbone: widths and tab height must be positive")
        if self.gauge_width > self.tab_width:
            raise ValueError("dogbone: gauge_width exceeds tab_width")
        self.reduction = 0.5 * (self.tab_width - self.gauge_width)
        if self.radius < self.reduction:
            raise ValueError("dogbone: radius smaller than (tab_width - gauge_width)/2")
        self.shoulder = np.sqrt(self.reduction * (2.0 * self.radius - self.reduction))
        self.total_height = 2.0 * (self.shoulder + self.tab_height)

    def half_width(self, s_abs):
        ds = np.abs(np.asarray(s_abs, dtype=float) - self.centre[self.axial])
        arc = (0.5 * self.gauge_width + self.radius
               - np.sqrt(np.maximum(self.radius ** 2 - np.minimum(ds, self.radius) ** 2, 0.0)))
        return np.where(ds <= self.shoulder, arc, 0.5 * self.tab_width)

    def _tol(self, tol):
        return 1e-6 * self.tab_width if tol is None else float(tol)

    def _in_length(self, p, tol):
        return np.abs(p[:, self.axial] - self.centre[self.axial]) <= 0.5 * self.total_height + tol

    def summary(self):
        return (f"{type(self).__name__}: tab {self.tab_width} x {self.tab_height}, gauge "
                f"{self.gauge_width}, radius {self.radius}, total length {self.total_height:.6g}")


class DogBone2D(_Profile):
    """Plane-strain slab |x - x_c| <= w(y)."""

    def contains(self, points, tol=None):
        tol = self._tol(tol)
        p = np.asarray(points, dtype=float)
        return self._in_length(p, tol) & (np.abs(p[:, 0] - self.centre[0])
                                          <= self.half_width(p[:, 1]) + tol)


class DogBone3D(_Profile):
    """Round bar: the profile revolved about the y axis, hypot(x - x_c, z - z_c) <= w(y)."""
    revolved = True

    def contains(self, points, tol=None):
        tol = self._tol(tol)
        p = np.asarray(points, dtype=float)
        r = np.hypot(p[:, 0] - self.centre[0], p[:, 2] - self.centre[2])
        return self._in_length(p, tol) & (r <= self.half_width(p[:, 1]) + tol)


class DogBoneAxi(_Profile):
    """Meridional half-section for an axisymmetric deck: x axial, y = r >= 0."""
    axial = 0
    revolved = True

    def contains(self, points, tol=None):
        tol = self._tol(tol)
        p = np.asarray(points, dtype=float)
        return (self._in_length(p, tol) & (p[:, 1] >= -tol)
                & (p[:, 1] <= self.half_width(p[:, 0]) + tol))


class GaugeDogBoneAxi(DogBoneAxi):
    """Axisymmetric round bar with a PARALLEL gauge length: a straight section of
    diameter W_g over `gauge_length`, tangent fillets of radius R, and straight heads of
    diameter W_t over `tab_height`.  The reference's profile has no parallel length
    (its two arcs meet at mid-length); this is the host-side shape extension the
    tensile-bar workloads need.  Only the profile differs from DogBoneAxi."""

    def __init__(self, tab_width, tab_height, gauge_width, radius, gauge_length,
                 centre=(0.0, 0.0, 0.0)):
        self.gauge_length = float(gauge_length)
        super().__init__(tab_width, tab_height, gauge_width, radius, centre)
        # fillet: quarter-type arc from the gauge surface to the head surface
        self.total_height = self.gauge_length + 2.0 * (self.shoulder + self.tab_height)

    def half_width(self, s_abs):
        ds = np.abs(np.asarray(s_abs, dtype=float) - self.centre[self.axial])
        half_g = 0.5 * self.gauge_length
        t = np.maximum(ds - half_g, 0.0)
        arc = (0.5 * self.gauge_width + self.radius
               - np.sqrt(np.maximum(self.radius ** 2 - np.minimum(t, self.radius) ** 2, 0.0)))
        return np.where(t <= self.shoulder, arc, 0.5 * self.tab_width)


class GaugeDogBone3D(GaugeDogBoneAxi):
    """The parallel-gauge profile revolved about the y axis (3D round bar)."""
    axial = 1

    def contains(self, points, tol=None):
        tol = self._tol(tol)
        p = np.asarray(points, dtype=float)
        r = np.hypot(p[:, 0] - self.centre[0], p[:, 2] - self.centre[2])
        return self._in_length(p, tol) & (r <= self.half_width(p[:, 1]) + tol)


class Circle2D:
    def __init__(self, radius, centre=(0.0, 0.0, 0.0)):
        self.radius = float(radius)
        c = np.asarray(centre, dtype=float).ravel()
        self.centre = np.zeros(3)
        self.centre[:len(c)] = c[:3]

    def contains(self, points, tol=None):
        tol = 1e-6 * self.radius if tol is None else float(tol)
        p = np.asarray(points, dtype=float)
        return np.hypot(p[:, 0] - self.centre[0], p[:, 1] - self.centre[1]) <= self.radius + tol

    def summary(self):
        return f"circle: radius {self.radius}"


class Sphere3D(Circle2D):
    def contains(self, points, tol=None):
        tol = 1e-6 * self.radius if tol is None else float(tol)
        p = np.asarray(points, dtype=float) - self.centre[None, :]
        return np.sqrt((p[:, :3] ** 2).sum(axis=1)) <= self.radius + tol


class Cylinder3D(Circle2D):
    def __init__(self, radius, axis="x", centre=(0.0, 0.0, 0.0)):
        super().__init__(radius, centre)
        self.axis = "xyz".index(str(axis).lower())

    def contains(self, points, tol=None):
        tol = 1e-6 * self.radius if tol is None else float(tol)
        p = np.asarray(points, dtype=float) - self.centre[None, :]
        k = [a for a in range(3) if a != self.axis]
        return np.hypot(p[:, k[0]], p[:, k[1]]) <= self.radius + tol


def region_from_spec(spec, default_centre):
    """The region of a block's `shape` entry, or None (geometry.py:517-549)."""
    if not spec:
        return None
    kind = str(spec.get("type", "")).lower()
    centre = spec.get("center", default_centre)
    if kind == "circle":
        return Circle2D(spec["radius"], centre)
    if kind == "sphere":
        return Sphere3D(spec["radius"], centre)
    if kind == "cylinder":
        return Cylinder3D(spec["radius"], spec.get("axis", "x"), centre)
    if kind in ("dogbone", "dogbone3d", "dogboneaxi"):
        cls = {"dogbone": DogBone2D, "dogbone3d": DogBone3D, "dogboneaxi": DogBoneAxi}[kind]
        return cls(spec["tabWidth"], spec["tabHeight"], spec["gaugeWidth"], spec["radius"], centre)
    if kind in ("gaugedogboneaxi", "gaugedogbone3d"):
        cls = GaugeDogBoneAxi if kind == "gaugedogboneaxi" else GaugeDogBone3D
        return cls(spec["tabWidth"], spec["tabHeight"], spec["gaugeWidth"], spec["radius"],
                   spec["gaugeLength"], centre)
    raise ValueError(f"unknown block shape {spec.get('type')!r}")
