"""Host front end of the forward Tet4 phi-ASE path (include/hase_b200_forward.h).

``TetDeviceMesh`` is one libhase_b200 Tet4 context: the mesh tables resident
on a device, ``calc_phi_ase`` the reference's current calcPhiASE
(include/core/forwardPhiAseEvaluator.hpp:114-178) returning a ``Result`` with
the reference's forward fields (pyInclude/structures.py:7-18): ``phiAse`` and
``relativeStandardError`` per cell, ``totalRays`` the cell's ray visits,
``dndtAse`` and ``droppedRays``.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .simulation import Result
from .tetmesh import TetMesh

TALLY_MODES = {"auto": 0, "global": 1, "shared": 2}


class TetDeviceMesh:
    """A libhase_b200 Tet4 context on one device."""

    def __init__(self, mesh: TetMesh, sigmaA, sigmaE, device: int = 0):
        self.mesh = mesh
        self._keep = []
        sa = self._hold(np.atleast_1d(np.asarray(sigmaA, np.float64)))
        se = self._hold(np.atleast_1d(np.asarray(sigmaE, np.float64)))
        if sa.size != se.size or sa.size == 0:
            raise ValueError("sigmaA and sigmaE must be non-empty and of equal length")
        clad = None if mesh.claddingCellTypes is None else N.ptr(self._hold(mesh.claddingCellTypes), N._u32p)

        def opt(v, t):
            return None if v is None else N.ptr(self._hold(v), t)

        surf = mesh.surfaceArrays()
        desc = N.TetMeshDesc(mesh.numberOfPoints, mesh.numberOfCells, N.ptr(self._hold(mesh.points), N._f64p),
                             N.ptr(self._hold(mesh.cells), N._u32p), N.ptr(self._hold(mesh.betaVolume), N._f64p),
                             clad, int(mesh.claddingNumber), float(mesh.claddingAbsorption), float(mesh.nTot),
                             float(mesh.crystalTFluo), opt(mesh.cellFaceBoundaries, C.POINTER(C.c_int32)),
                             mesh.numberOfSurfaces, *[opt(v, N._f64p) for v in surf],
                             opt(mesh.reflectivities, N._f64p), opt(mesh.refractiveIndices, N._f64p))
        spec = N.SpectrumDesc(sa.size, N.ptr(sa, N._f64p), N.ptr(se, N._f64p))
        handle = C.c_void_p()
        N.check(N.lib().hase_tet_context_create(C.byref(desc), C.byref(spec), int(device), C.byref(handle)))
        self.handle = handle
        self.numberOfWavelengths = sa.size

    def _hold(self, a):
        a = np.ascontiguousarray(a)
        self._keep.append(a)
        return a

    def update_beta(self, betaVolume):
        bv = np.ascontiguousarray(np.asarray(betaVolume, np.float64).ravel())
        if bv.size != self.mesh.numberOfCells:
            raise ValueError("betaVolume size mismatch")
        N.check(N.lib().hase_tet_context_update_beta(self.handle, N.ptr(bv, N._f64p)))

    def calc_phi_ase(self, *, forwardRayCount, maxRays=None, adaptiveSteps=0, relativeStandardErrorThreshold=0.0,
                     monochromatic=False, rngSeed=5489, batches=8, blockSize=0, tallyMode="auto",
                     useReflections=False, reflectionMaxIterations=40, reflectionTolerance=1.0e-4,
                     surfaceReservoirSize=32, divergenceStreak=3) -> Result:
        """The forward solve; with ``useReflections`` the surface-reservoir
        reflection passes run at the mesh's reflecting boundary faces and the
        ``srm*`` fields of the result are filled."""
        n = self.mesh.numberOfCells
        out = Result(phiAse=np.empty(n, np.float32), relativeStandardError=np.empty(n),
                     totalRays=np.empty(n, np.uint32), dndtAse=np.empty(n), droppedRays=np.empty(n, np.uint32))
        if tallyMode not in TALLY_MODES:
            raise ValueError(f"tallyMode must be one of {sorted(TALLY_MODES)}")
        fw = N.ForwardDesc(int(forwardRayCount), int(maxRays if maxRays is not None else forwardRayCount),
                           int(adaptiveSteps), float(relativeStandardErrorThreshold), 1 if monochromatic else 0,
                           int(rngSeed) & 0xFFFFFFFF, int(batches), int(blockSize), TALLY_MODES[tallyMode],
                           1 if useReflections else 0, int(reflectionMaxIterations), float(reflectionTolerance),
                           int(surfaceReservoirSize), int(divergenceStreak))
        r = N.ForwardResultDesc(N.ptr(out.phiAse, N._f32p), N.ptr(out.relativeStandardError, N._f64p),
                                N.ptr(out.dndtAse, N._f64p), N.ptr(out.totalRays, N._u32p),
                                N.ptr(out.droppedRays, N._u32p))
        out.status = N.check(N.lib().hase_tet_calc_phi_ase(self.handle, C.byref(fw), C.byref(r)),
                             allow_warnings=True)
        out.raysTraced = int(r.raysTraced)
        out.crossings = int(r.crossings)
        out.rayMilliseconds = float(r.rayMilliseconds)
        out.totalMilliseconds = float(r.totalMilliseconds)
        out.passes = int(r.launches)
        out.unconvergedSamples = int(r.unconvergedCells)
        out.kernelLaunches = int(r.kernelLaunches)
        out.tallyMode = int(r.tallyMode)
        out.srmStatus = N.SRM_STATUS[r.srmStatus]
        out.srmPasses = int(r.srmPasses)
        out.srmRemainingFraction = float(r.srmRemainingFraction)
        out.srmMaxIterations = int(r.srmMaxIterations)
        out.srmDivergenceStreak = int(r.srmDivergenceStreak)
        out.reflectingFaces = int(r.reflectingFaces)
        return out

    def tables(self):
        C4 = 4 * self.mesh.numberOfCells
        out = {"neighbors": np.empty((self.mesh.numberOfCells, 4), np.int32),
               "neighborFace": np.empty((self.mesh.numberOfCells, 4), np.int32),
               "planes": np.empty((self.mesh.numberOfCells, 4, 4)), "volumes": np.empty(self.mesh.numberOfCells)}
        assert out["planes"].size == 4 * C4
        i32 = C.POINTER(C.c_int32)
        N.check(N.lib().hase_tet_tables(self.handle, N.ptr(out["neighbors"], i32), N.ptr(out["neighborFace"], i32),
                                        N.ptr(out["planes"], N._f64p), N.ptr(out["volumes"], N._f64p)))
        return out

    def trace(self, start_cell, origin, direction, *, wavelength=0, max_segments=64):
        sc = np.ascontiguousarray(np.atleast_1d(np.asarray(start_cell, np.uint32)))
        o = np.ascontiguousarray(np.asarray(origin, np.float64).reshape(-1, 3))
        d = np.ascontiguousarray(np.asarray(direction, np.float64).reshape(-1, 3))
        n = sc.size
        if o.shape[0] != n or d.shape[0] != n:
            raise ValueError("start_cell, origin and direction must describe the same rays")
        out = {"segments": np.empty(n, np.uint32), "cells": np.zeros((n, max_segments), np.uint32),
               "lengths": np.zeros((n, max_segments)), "lnGain": np.empty(n), "endPoint": np.empty((n, 3)),
               "status": np.empty(n, np.int32)}
        i32 = C.POINTER(C.c_int32)
        N.check(N.lib().hase_tet_trace(self.handle, n, N.ptr(sc, N._u32p), N.ptr(o, N._f64p), N.ptr(d, N._f64p),
                                       int(wavelength), int(max_segments), N.ptr(out["segments"], N._u32p),
                                       N.ptr(out["cells"], N._u32p), N.ptr(out["lengths"], N._f64p),
                                       N.ptr(out["lnGain"], N._f64p), N.ptr(out["endPoint"], N._f64p),
                                       N.ptr(out["status"], i32)))
        return out

    def close(self):
        if getattr(self, "handle", None):
            N.lib().hase_tet_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
