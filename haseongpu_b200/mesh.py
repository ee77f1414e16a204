"""Extruded triangle-prism gain medium (the legacy HASEonGPU mesh layout).

A 2-D triangle mesh (``points`` [Np, 2], ``triangles`` [T, 3]) is extruded to
``numberOfLevels`` z levels spaced ``thickness`` apart.  Prism (triangle t,
layer l) has index ``t + l * T``; sample point (point p, level l) has index
``p + l * Np`` -- the legacy HostMesh layout whose compatibility fields survive
in the reference at include/core/mesh.hpp:532-539 and whose record names are
pyInclude/openpmd/schema/builtins.py:149-171.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


@dataclass
class PrismMesh:
    points: np.ndarray                     # [Np, 2] float64 (cm)
    triangles: np.ndarray                  # [T, 3] uint32
    numberOfLevels: int
    thickness: float                       # level spacing (cm)
    betaVolume: np.ndarray                 # [(levels-1) * T] excited fraction per prism
    nTot: float                            # doping density (cm^-3)
    crystalTFluo: float                    # fluorescence lifetime (s)
    betaCells: np.ndarray | None = None    # [levels * Np] per sample point (dndt)
    claddingCellTypes: np.ndarray | None = None  # [T]
    claddingNumber: int = 1
    claddingAbsorption: float = 0.0        # cm^-1
    reflectivities: np.ndarray | None = None     # [T, 2]: bottom, top
    refractiveIndices: np.ndarray | None = None  # [4]: bottom in/out, top in/out
    name: str = field(default="prism-mesh", compare=False)

    def __post_init__(self):
        self.points = np.ascontiguousarray(np.asarray(self.points, np.float64).reshape(-1, 2))
        self.triangles = np.ascontiguousarray(np.asarray(self.triangles, np.uint32).reshape(-1, 3))
        self.numberOfLevels = int(self.numberOfLevels)
        self.thickness = float(self.thickness)
        self.betaVolume = np.ascontiguousarray(np.asarray(self.betaVolume, np.float64).ravel())
        if self.numberOfLevels < 2:
            raise ValueError("numberOfLevels must be >= 2")
        if self.betaVolume.size != self.numberOfPrisms:
            raise ValueError(f"betaVolume must have {self.numberOfPrisms} entries, got {self.betaVolume.size}")
        if self.betaCells is not None:
            self.betaCells = np.ascontiguousarray(np.asarray(self.betaCells, np.float64).ravel())
            if self.betaCells.size != self.numberOfSamples:
                raise ValueError(f"betaCells must have {self.numberOfSamples} entries")
        if self.claddingCellTypes is not None:
            self.claddingCellTypes = np.ascontiguousarray(np.asarray(self.claddingCellTypes, np.uint32).ravel())
            if self.claddingCellTypes.size != self.numberOfTriangles:
                raise ValueError("claddingCellTypes must have one entry per triangle")
        if self.reflectivities is not None:
            self.reflectivities = np.ascontiguousarray(np.asarray(self.reflectivities, np.float64).reshape(-1, 2))
            if self.reflectivities.shape[0] != self.numberOfTriangles:
                raise ValueError("reflectivities must be [T, 2]")
        if self.refractiveIndices is not None:
            self.refractiveIndices = np.ascontiguousarray(np.asarray(self.refractiveIndices, np.float64).ravel())
            if self.refractiveIndices.size != 4:
                raise ValueError("refractiveIndices must have 4 entries")

    @property
    def numberOfPoints(self) -> int:
        return int(self.points.shape[0])

    @property
    def numberOfTriangles(self) -> int:
        return int(self.triangles.shape[0])

    @property
    def numberOfPrisms(self) -> int:
        return self.numberOfTriangles * (self.numberOfLevels - 1)

    @property
    def numberOfSamples(self) -> int:
        return self.numberOfPoints * self.numberOfLevels

    def samplePoints(self) -> np.ndarray:
        """[S, 3] sample positions, index p + l * Np."""
        z = np.repeat(np.arange(self.numberOfLevels) * self.thickness, self.numberOfPoints)
        xy = np.tile(self.points, (self.numberOfLevels, 1))
        return np.column_stack([xy, z])

    def triangleAreas(self) -> np.ndarray:
        p = self.points[self.triangles]
        ab = p[:, 1] - p[:, 0]
        ac = p[:, 2] - p[:, 0]
        return 0.5 * np.abs(ab[:, 0] * ac[:, 1] - ab[:, 1] * ac[:, 0])

    def prismVolumes(self) -> np.ndarray:
        return np.tile(self.triangleAreas() * self.thickness, self.numberOfLevels - 1)

    def prismCentroids(self) -> np.ndarray:
        c = self.points[self.triangles].mean(axis=1)
        z = (np.arange(self.numberOfLevels - 1) + 0.5) * self.thickness
        return np.column_stack([np.tile(c, (self.numberOfLevels - 1, 1)), np.repeat(z, self.numberOfTriangles)])

    def withBeta(self, betaVolume, betaCells=None) -> "PrismMesh":
        from dataclasses import replace
        return replace(self, betaVolume=betaVolume, betaCells=self.betaCells if betaCells is None else betaCells)

    @classmethod
    def fromLegacyFixture(cls, path, claddingAbsorption=None) -> "PrismMesh":
        """Load a legacy prism fixture written by tests/golden/make_golden.py."""
        d = np.load(Path(path))
        absorption = claddingAbsorption
        if absorption is None:
            absorption = float(d["claddingAbsorption"]) if "claddingAbsorption" in d.files else 0.0
        return cls(
            points=d["points2d"], triangles=d["triangles"], numberOfLevels=int(d["numberOfLevels"]),
            thickness=float(d["thickness"]), betaVolume=d["betaVolume"], nTot=float(d["nTot"]),
            crystalTFluo=float(d["crystalTFluo"]), betaCells=d["betaCells"],
            claddingCellTypes=d["claddingCellTypes"], claddingNumber=int(d["claddingNumber"]),
            claddingAbsorption=float(absorption), name=Path(path).stem)


def disc_points(radius: float, rings: int, rng: np.random.Generator, jitter: float = 0.25) -> np.ndarray:
    """Points on concentric rings (6k points on ring k), jittered by +-jitter * ring spacing.

    Interior points move uniformly in x and y; the outer ring only moves
    along the circle, so the disc boundary stays on radius ``radius``.
    """
    dr = radius / rings
    pts = [np.zeros((1, 2))]
    for k in range(1, rings + 1):
        n = 6 * k
        phi = 2.0 * np.pi * (np.arange(n) + rng.uniform(-jitter, jitter, n) * (k < rings)) / n
        phi += rng.uniform(0, 2 * np.pi / n)
        r = np.full(n, k * dr)
        ring = np.column_stack([r * np.cos(phi), r * np.sin(phi)])
        if k < rings:
            ring += rng.uniform(-jitter * dr, jitter * dr, size=(n, 2))
        else:
            ring = np.column_stack([radius * np.cos(phi), radius * np.sin(phi)])
        pts.append(ring)
    return np.vstack(pts)


def morton_order(xy: np.ndarray, bits: int = 16) -> np.ndarray:
    """Permutation sorting 2-D positions along a Z-order (Morton) curve."""
    xy = np.asarray(xy, np.float64)
    lo, hi = xy.min(axis=0), xy.max(axis=0)
    q = ((xy - lo) / np.maximum(hi - lo, 1e-300) * ((1 << bits) - 1)).astype(np.uint64)

    def spread(v):
        v = v & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v

    return np.argsort(spread(q[:, 0]) | (spread(q[:, 1]) << np.uint64(1)), kind="stable")


def delaunay_triangles(points: np.ndarray, spatial_order: bool = True) -> np.ndarray:
    """Delaunay triangulation (scipy/Qhull), counter-clockwise, slivers removed.

    With ``spatial_order`` the triangles are numbered along a Morton curve of
    their centroids, so neighbouring prism indices are neighbouring prisms
    (warps then walk nearby rays)."""
    from scipy.spatial import Delaunay

    tri = Delaunay(points).simplices.astype(np.int64)
    p = points[tri]
    cross = (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 1, 1] - p[:, 0, 1]) * (p[:, 2, 0] - p[:, 0, 0])
    tri[cross < 0] = tri[cross < 0][:, [0, 2, 1]]
    keep = np.abs(cross) > 1e-12 * np.max(np.abs(cross))
    tri = tri[keep]
    if spatial_order:
        tri = tri[morton_order(points[tri].mean(axis=1))]
    return tri.astype(np.uint32)


def gaussian_pump_beta(mesh_points, triangles, levels, thickness, waist=0.4, depth=0.5, base=0.05, peak=0.25):
    """beta = base + peak * exp(-r^2 / waist^2) * exp(-z / depth) at each prism centroid."""
    c = np.asarray(mesh_points)[np.asarray(triangles)].mean(axis=1)
    r2 = (c ** 2).sum(axis=1)
    z = (np.arange(levels - 1) + 0.5) * thickness
    beta = base + peak * np.exp(-r2[None, :] / waist ** 2) * np.exp(-z[:, None] / depth)
    return beta.ravel()


def point_beta(mesh_points, levels, thickness, waist=0.4, depth=0.5, base=0.05, peak=0.25):
    r2 = (np.asarray(mesh_points) ** 2).sum(axis=1)
    z = np.arange(levels) * thickness
    return (base + peak * np.exp(-r2[None, :] / waist ** 2) * np.exp(-z[:, None] / depth)).ravel()
