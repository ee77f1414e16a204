"""Tet4 (tetrahedral) gain medium: the mesh of the reference's current,
forward phi-ASE method.

Layout mirrors the reference's ``VolumeTopology`` / ``HostMesh`` for Tet4
cells (include/core/mesh.hpp:144-333; pyInclude/geometry/volume.py:460-509):
``points`` [Np, 3] (cm), ``cells`` [C, 4] point indices, per-cell
``betaVolume``, ``claddingCellTypes`` (cells of type ``claddingNumber`` are
cladding, absorbing with ``claddingAbsorption``), ``nTot`` and
``crystalTFluo``.  Local face f of a cell is the face opposite its vertex f.

Generators: ``fromPrismMesh`` splits every wedge of an extruded prism mesh
into three tetrahedra (the Tet4 twin of a prism mesh, as the reference's
utils/convert_vtk_topology.py:38-52 does), ``ball`` builds a tetrahedral ball
for the analytic sphere-centre check (tests/python/phiAse/test_analyticalSphere.py).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


@dataclass
class TetMesh:
    points: np.ndarray                     # [Np, 3] float64 (cm)
    cells: np.ndarray                      # [C, 4] uint32
    betaVolume: np.ndarray                 # [C] excited fraction per cell
    nTot: float                            # doping density (cm^-3)
    crystalTFluo: float                    # fluorescence lifetime (s)
    claddingCellTypes: np.ndarray | None = None  # [C]
    claddingNumber: int = 1
    claddingAbsorption: float = 0.0        # cm^-1
    name: str = field(default="tet4-mesh", compare=False)
    # Reflecting boundary surfaces (include/core/mesh.hpp:301-332): surface
    # id per local face (> 0 on a boundary face: a reflecting surface), per
    # surface reflectivity and refractive indices inside / outside; ids
    # outside the per-surface arrays fall back to the legacy per-cell
    # ``reflectivities`` [C, 2] (by local face % 2) and ``refractiveIndices``
    # [4] (face % 2 = 0: inside, outside; face % 2 = 1: inside, outside).
    cellFaceBoundaries: np.ndarray | None = None     # [C, 4] int32
    surfaceReflectivities: np.ndarray | None = None  # [S]
    surfaceRefractiveIndexInside: np.ndarray | None = None
    surfaceRefractiveIndexOutside: np.ndarray | None = None
    reflectivities: np.ndarray | None = None         # legacy [C, 2]
    refractiveIndices: np.ndarray | None = None      # legacy [4]

    def __post_init__(self):
        self.points = np.ascontiguousarray(np.asarray(self.points, np.float64).reshape(-1, 3))
        self.cells = np.ascontiguousarray(np.asarray(self.cells, np.uint32).reshape(-1, 4))
        self.betaVolume = np.ascontiguousarray(np.asarray(self.betaVolume, np.float64).ravel())
        if self.cells.size and int(self.cells.max()) >= self.points.shape[0]:
            raise ValueError("cells reference points that do not exist")
        if self.betaVolume.size != self.numberOfCells:
            raise ValueError(f"betaVolume must have {self.numberOfCells} entries, got {self.betaVolume.size}")
        if self.claddingCellTypes is not None:
            self.claddingCellTypes = np.ascontiguousarray(np.asarray(self.claddingCellTypes, np.uint32).ravel())
            if self.claddingCellTypes.size != self.numberOfCells:
                raise ValueError("claddingCellTypes must have one entry per cell")
        if self.cellFaceBoundaries is not None:
            self.cellFaceBoundaries = np.ascontiguousarray(np.asarray(self.cellFaceBoundaries, np.int32).reshape(-1, 4))
            if self.cellFaceBoundaries.shape[0] != self.numberOfCells:
                raise ValueError("cellFaceBoundaries must have one row of 4 surface ids per cell")
        for name in ("surfaceReflectivities", "surfaceRefractiveIndexInside", "surfaceRefractiveIndexOutside",
                     "refractiveIndices"):
            v = getattr(self, name)
            if v is not None:
                setattr(self, name, np.ascontiguousarray(np.asarray(v, np.float64).ravel()))
        if self.reflectivities is not None:
            self.reflectivities = np.ascontiguousarray(np.asarray(self.reflectivities, np.float64).reshape(-1, 2))
            if self.reflectivities.shape[0] != self.numberOfCells:
                raise ValueError("reflectivities must have one row of 2 per cell")
        self.claddingNumber = int(self.claddingNumber)
        self.claddingAbsorption = float(self.claddingAbsorption)
        self.nTot = float(self.nTot)
        self.crystalTFluo = float(self.crystalTFluo)

    @property
    def numberOfPoints(self) -> int:
        return int(self.points.shape[0])

    @property
    def numberOfCells(self) -> int:
        return int(self.cells.shape[0])

    def cellVolumes(self) -> np.ndarray:
        p = self.points[self.cells.astype(np.int64)]
        e = p[:, 1:] - p[:, :1]
        return np.abs(np.einsum("ij,ij->i", e[:, 0], np.cross(e[:, 1], e[:, 2]))) / 6.0

    def cellCenters(self) -> np.ndarray:
        return self.points[self.cells.astype(np.int64)].mean(axis=1)

    def claddingMask(self) -> np.ndarray:
        if self.claddingCellTypes is None:
            return np.zeros(self.numberOfCells, bool)
        return self.claddingCellTypes == self.claddingNumber

    @property
    def numberOfSurfaces(self) -> int:
        return max(0 if v is None else int(v.size) for v in (self.surfaceReflectivities,
                                                             self.surfaceRefractiveIndexInside,
                                                             self.surfaceRefractiveIndexOutside))

    def surfaceArrays(self) -> tuple:
        """Per-surface arrays padded to numberOfSurfaces (None stays None)."""
        n = self.numberOfSurfaces
        out = []
        for v, fill in ((self.surfaceReflectivities, 0.0), (self.surfaceRefractiveIndexInside, 1.0),
                        (self.surfaceRefractiveIndexOutside, 1.0)):
            out.append(None if v is None else np.concatenate([v, np.full(n - v.size, fill)]))
        return tuple(out)

    def boundaryFaces(self) -> np.ndarray:
        """[C, 4] bool: local faces without a neighbour."""
        from collections import Counter

        faces = np.sort(np.stack([np.delete(self.cells, f, axis=1) for f in range(4)], axis=1), axis=2)
        keys = [tuple(k) for k in faces.reshape(-1, 3)]
        count = Counter(keys)
        return np.array([count[k] == 1 for k in keys]).reshape(-1, 4)

    def withBeta(self, betaVolume) -> "TetMesh":
        return TetMesh(self.points, self.cells, betaVolume, self.nTot, self.crystalTFluo, self.claddingCellTypes,
                       self.claddingNumber, self.claddingAbsorption, self.name, self.cellFaceBoundaries,
                       self.surfaceReflectivities, self.surfaceRefractiveIndexInside,
                       self.surfaceRefractiveIndexOutside, self.reflectivities, self.refractiveIndices)

    def withReflectingBoundary(self, reflectivity: float, nInside: float = 1.0, nOutside: float = 1.0) -> "TetMesh":
        """The same mesh with every boundary face on one reflecting surface (id 1)."""
        ids = np.where(self.boundaryFaces(), 1, 0).astype(np.int32)
        m = self.withBeta(self.betaVolume)
        m.cellFaceBoundaries = ids
        m.surfaceReflectivities = np.array([0.0, float(reflectivity)])
        m.surfaceRefractiveIndexInside = np.array([1.0, float(nInside)])
        m.surfaceRefractiveIndexOutside = np.array([1.0, float(nOutside)])
        return m

    @classmethod
    def fromFixture(cls, path, claddingAbsorption=None) -> "TetMesh":
        """Tet4 fixture (.npz with points, cells, betaVolume, claddingCellTypes, ...)."""
        d = np.load(Path(path))
        if claddingAbsorption is None:
            claddingAbsorption = float(d["claddingAbsorption"]) if "claddingAbsorption" in d.files else 0.0
        return cls(d["points"], d["cells"], d["betaVolume"], float(d["nTot"]), float(d["crystalTFluo"]),
                   d["claddingCellTypes"] if "claddingCellTypes" in d.files else None,
                   int(d["claddingNumber"]) if "claddingNumber" in d.files else 1, float(claddingAbsorption),
                   name=Path(path).stem)

    @classmethod
    def fromPrismMesh(cls, prism) -> "TetMesh":
        """Split every wedge (triangle t, layer l) of a PrismMesh into 3 tets.

        With the triangle's vertices ordered by global point index
        v0 < v1 < v2, bottom a_k and top A_k, the tets are
        (a0 a1 a2 A0), (a1 a2 A0 A1), (a2 A0 A1 A2): the quad face between
        v_i < v_j gets the diagonal a_j - A_i, which depends only on the two
        global indices, so neighbouring wedges agree and the Tet4 mesh is
        conforming.  Cells of wedge p = t + l T are 3p, 3p+1, 3p+2 and inherit
        its betaVolume and its triangle's cladding type.
        """
        Np, T, L = prism.numberOfPoints, prism.numberOfTriangles, prism.numberOfLevels
        pts = np.empty((Np * L, 3))
        for lv in range(L):
            pts[lv * Np:(lv + 1) * Np, :2] = prism.points
            pts[lv * Np:(lv + 1) * Np, 2] = lv * prism.thickness
        tri = np.sort(prism.triangles.astype(np.int64), axis=1)
        cells = np.empty((T * (L - 1), 3, 4), np.int64)
        for lv in range(L - 1):
            a = tri + lv * Np
            A = tri + (lv + 1) * Np
            blk = cells[lv * T:(lv + 1) * T]
            blk[:, 0] = np.stack([a[:, 0], a[:, 1], a[:, 2], A[:, 0]], axis=1)
            blk[:, 1] = np.stack([a[:, 1], a[:, 2], A[:, 0], A[:, 1]], axis=1)
            blk[:, 2] = np.stack([a[:, 2], A[:, 0], A[:, 1], A[:, 2]], axis=1)
        clad = None
        if prism.claddingCellTypes is not None:
            clad = np.repeat(np.tile(prism.claddingCellTypes, L - 1), 3)
        out = cls(pts, cells.reshape(-1, 4), np.repeat(prism.betaVolume, 3), prism.nTot, prism.crystalTFluo, clad,
                  prism.claddingNumber, prism.claddingAbsorption, name=f"{prism.name}-tet4")
        if getattr(prism, "reflectivities", None) is not None:
            # bottom face of cell 0 of layer 0 (opposite corner 3) and top face
            # of cell 2 of the last layer (opposite corner 0): surface 1 + 2 t
            # (bottom of triangle t) and 2 + 2 t (top), with the prism's
            # reflectivities and refractive indices
            C = out.numberOfCells
            ids = np.zeros((C, 4), np.int32)
            t = np.arange(T)
            ids[3 * t, 3] = 1 + 2 * t
            ids[3 * ((L - 2) * T + t) + 2, 0] = 2 + 2 * t
            R = np.asarray(prism.reflectivities, np.float64).reshape(T, 2)
            n = np.asarray(prism.refractiveIndices if getattr(prism, "refractiveIndices", None) is not None
                           else [1.0, 1.0, 1.0, 1.0], np.float64)
            out.cellFaceBoundaries = ids
            out.surfaceReflectivities = np.concatenate([[0.0], R.ravel()])
            out.surfaceRefractiveIndexInside = np.concatenate([[1.0], np.tile([n[0], n[2]], T)])
            out.surfaceRefractiveIndexOutside = np.concatenate([[1.0], np.tile([n[1], n[3]], T)])
        return out

    @classmethod
    def ball(cls, radius: float, divisions: int, beta: float, nTot: float, crystalTFluo: float) -> "TetMesh":
        """Tetrahedral ball: the cube [-1, 1]^3 cut into divisions^3 cubes of
        6 tets each (Kuhn split along the main diagonal, conforming), then
        every point p moved radially to p |p|_inf / |p|_2 * radius, which maps
        the cube's surface onto the sphere and fixes the centre.  ``divisions``
        must be even so the centre is a mesh point."""
        n = int(divisions)
        if n < 2 or n % 2:
            raise ValueError("divisions must be an even number >= 2")
        g = np.linspace(-1.0, 1.0, n + 1)
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        p = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        r2 = np.linalg.norm(p, axis=1)
        rinf = np.abs(p).max(axis=1)
        scale = np.where(r2 > 0, rinf / np.where(r2 > 0, r2, 1.0), 0.0)
        pts = p * scale[:, None] * float(radius)

        def idx(i, j, k):
            return (i * (n + 1) + j) * (n + 1) + k

        i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        i, j, k = i.ravel(), j.ravel(), k.ravel()
        corner = {b: idx(i + (b >> 2 & 1), j + (b >> 1 & 1), k + (b & 1)) for b in range(8)}
        # the 6 monotone paths 000 -> 111 through the cube's corners
        paths = [(4, 6), (4, 5), (2, 6), (2, 3), (1, 5), (1, 3)]
        cells = np.concatenate([np.stack([corner[0], corner[a], corner[b], corner[7]], axis=1) for a, b in paths])
        C = cells.shape[0]
        return cls(pts, cells, np.full(C, float(beta)), nTot, crystalTFluo, np.zeros(C, np.uint32), 1, 0.0,
                   name=f"ball-r{radius:g}-n{n}")


def analytic_sphere_centre(gain: float, radius: float, beta: float, nTot: float, crystalTFluo: float) -> float:
    """phi-ASE at the centre of a uniform sphere: N_tot beta/tau expm1(g R)/g
    (tests/python/phiAse/test_analyticalSphere.py:19-28)."""
    if abs(gain) < 1e-12:
        return nTot * beta / crystalTFluo * radius
    return nTot * beta / crystalTFluo * np.expm1(gain * radius) / gain


def beta_from_gain(gain: float, nTot: float, sigmaA: float, sigmaE: float) -> float:
    """beta that gives the gain coefficient g = N_tot (beta (sE + sA) - sA)."""
    return (gain / nTot + sigmaA) / (sigmaA + sigmaE)
