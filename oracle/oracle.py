"""ctypes front end of the FP64 CPU oracle (libhase_oracle.so).

TEST INFRASTRUCTURE ONLY.  The tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` use this module as the checker; the product
package never imports it.

Every function takes a *mesh* object with the attributes of
``haseongpu_b200.PrismMesh`` (points, triangles, numberOfLevels, thickness,
betaVolume, betaCells, claddingCellTypes, claddingNumber, claddingAbsorption,
nTot, crystalTFluo, reflectivities, refractiveIndices) and a *spectrum* given
as two sequences ``(sigmaA, sigmaE)``.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libhase_oracle.so"

_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)


class _Mesh(C.Structure):
    _fields_ = [
        ("numberOfPoints", C.c_uint32),
        ("numberOfTriangles", C.c_uint32),
        ("numberOfLevels", C.c_uint32),
        ("points", _f64p),
        ("triangles", _u32p),
        ("thickness", C.c_double),
        ("betaVolume", _f64p),
        ("betaCells", _f64p),
        ("claddingCellTypes", _u32p),
        ("claddingNumber", C.c_uint32),
        ("claddingAbsorption", C.c_double),
        ("nTot", C.c_double),
        ("crystalTFluo", C.c_double),
        ("reflectivities", _f64p),
        ("refractiveIndices", _f64p),
    ]


class _Spectrum(C.Structure):
    _fields_ = [("numberOfWavelengths", C.c_uint32), ("sigmaA", _f64p), ("sigmaE", _f64p)]


class _Experiment(C.Structure):
    _fields_ = [
        ("minRays", C.c_uint32),
        ("maxRays", C.c_uint32),
        ("adaptiveSteps", C.c_uint32),
        ("mseThreshold", C.c_double),
        ("useReflections", C.c_uint32),
        ("seed", C.c_uint32),
        ("minSample", C.c_uint32),
        ("maxSample", C.c_uint32),
        ("nearField", C.c_uint32),
    ]


class _Result(C.Structure):
    _fields_ = [
        ("phiAse", _f64p),
        ("mse", _f64p),
        ("totalRays", _u32p),
        ("dndtAse", _f64p),
        ("droppedRays", _u32p),
        ("gainSum", _f64p),
        ("gainSumSquare", _f64p),
    ]


_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (g++ + OpenMP)."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB_PATH))
        _lib.oracle_ray_map.restype = C.c_uint64
    return _lib


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


class _Keep:
    """Holds the numpy buffers a ctypes structure points into."""

    def __init__(self):
        self.items = []

    def __call__(self, a):
        self.items.append(a)
        return a


def _mesh_struct(mesh, keep):
    pts = keep(np.ascontiguousarray(np.asarray(mesh.points, np.float64).reshape(-1, 2)))
    tri = keep(np.ascontiguousarray(np.asarray(mesh.triangles, np.uint32).reshape(-1, 3)))
    beta = keep(np.ascontiguousarray(np.asarray(mesh.betaVolume, np.float64).ravel()))
    bc = None if getattr(mesh, "betaCells", None) is None else keep(
        np.ascontiguousarray(np.asarray(mesh.betaCells, np.float64).ravel()))
    clad = None if getattr(mesh, "claddingCellTypes", None) is None else keep(
        np.ascontiguousarray(np.asarray(mesh.claddingCellTypes, np.uint32).ravel()))
    refl = None if getattr(mesh, "reflectivities", None) is None else keep(
        np.ascontiguousarray(np.asarray(mesh.reflectivities, np.float64).ravel()))
    ridx = None if getattr(mesh, "refractiveIndices", None) is None else keep(
        np.ascontiguousarray(np.asarray(mesh.refractiveIndices, np.float64).ravel()))
    return _Mesh(
        pts.shape[0], tri.shape[0], int(mesh.numberOfLevels), _ptr(pts, _f64p), _ptr(tri, _u32p),
        float(mesh.thickness), _ptr(beta, _f64p), _ptr(bc, _f64p), _ptr(clad, _u32p),
        int(getattr(mesh, "claddingNumber", 1)), float(getattr(mesh, "claddingAbsorption", 0.0)),
        float(mesh.nTot), float(mesh.crystalTFluo), _ptr(refl, _f64p), _ptr(ridx, _f64p))


def _spectrum_struct(spectrum, keep):
    sa = keep(np.ascontiguousarray(np.atleast_1d(np.asarray(spectrum[0], np.float64))))
    se = keep(np.ascontiguousarray(np.atleast_1d(np.asarray(spectrum[1], np.float64))))
    if sa.shape != se.shape:
        raise ValueError("sigmaA and sigmaE must have the same length")
    return _Spectrum(sa.size, _ptr(sa, _f64p), _ptr(se, _f64p))


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in ctr])
    k = (C.c_uint32 * 2)(*[int(v) & 0xFFFFFFFF for v in key])
    o = (C.c_uint32 * 4)()
    lib().oracle_philox4x32_10(c, k, o)
    return [int(v) for v in o]


def build_tables(points, triangles):
    pts = np.ascontiguousarray(np.asarray(points, np.float64).reshape(-1, 2))
    tri = np.ascontiguousarray(np.asarray(triangles, np.uint32).reshape(-1, 3))
    T = tri.shape[0]
    out = {
        "neighbors": np.empty((T, 3), np.int32), "forbiddenEdge": np.empty((T, 3), np.int32),
        "normalX": np.empty((T, 3)), "normalY": np.empty((T, 3)), "edgeC": np.empty((T, 3)),
        "centerX": np.empty(T), "centerY": np.empty(T), "area": np.empty(T),
    }
    rc = lib().oracle_build_tables(
        pts.shape[0], _ptr(pts, _f64p), T, _ptr(tri, _u32p), _ptr(out["neighbors"], _i32p),
        _ptr(out["forbiddenEdge"], _i32p), _ptr(out["normalX"], _f64p), _ptr(out["normalY"], _f64p),
        _ptr(out["edgeC"], _f64p), _ptr(out["centerX"], _f64p), _ptr(out["centerY"], _f64p),
        _ptr(out["area"], _f64p))
    if rc:
        raise ValueError(f"oracle_build_tables failed ({rc})")
    return out


def trace(mesh, spectrum, start, tri, level, sample, slice_=None, wavelength=0):
    """ln(gain) and straight-line distance of explicit rays (FP64)."""
    keep = _Keep()
    m = _mesh_struct(mesh, keep)
    s = _spectrum_struct(spectrum, keep)
    start = np.ascontiguousarray(np.asarray(start, np.float64).reshape(-1, 3))
    n = start.shape[0]
    tri = np.ascontiguousarray(np.asarray(tri, np.uint32))
    level = np.ascontiguousarray(np.asarray(level, np.uint32))
    sample = np.ascontiguousarray(np.asarray(sample, np.uint32))
    slice_ = np.zeros(n, np.uint32) if slice_ is None else np.ascontiguousarray(np.asarray(slice_, np.uint32))
    ln_gain = np.empty(n)
    dist = np.empty(n)
    dropped = np.empty(n, np.uint32)
    rc = lib().oracle_trace(C.byref(m), C.byref(s), int(wavelength), n, _ptr(start, _f64p), _ptr(tri, _u32p),
                            _ptr(level, _u32p), _ptr(sample, _u32p), _ptr(slice_, _u32p), _ptr(ln_gain, _f64p),
                            _ptr(dist, _f64p), _ptr(dropped, _u32p))
    if rc:
        raise ValueError(f"oracle_trace failed ({rc})")
    return ln_gain, dist, dropped


def importance(mesh, spectrum, sample, slices=1):
    keep = _Keep()
    m = _mesh_struct(mesh, keep)
    s = _spectrum_struct(spectrum, keep)
    P = np.asarray(mesh.triangles).reshape(-1, 3).shape[0] * (int(mesh.numberOfLevels) - 1)
    w = np.empty(slices * P)
    rc = lib().oracle_importance(C.byref(m), C.byref(s), int(sample), int(slices), _ptr(w, _f64p))
    if rc:
        raise ValueError(f"oracle_importance failed ({rc})")
    return w


def ray_map(weights, rays, phase):
    w = np.ascontiguousarray(np.asarray(weights, np.float32))
    q = np.empty(w.size, np.uint32)
    off = np.empty(w.size + 1, np.uint32)
    Q = lib().oracle_ray_map(w.size, _ptr(w, _f32p), int(rays), int(phase) & 0xFFFFFFFF, _ptr(q, _u32p),
                             _ptr(off, _u32p))
    return int(Q), q, off


def phi_ase(mesh, spectrum, *, minRays, maxRays=None, adaptiveSteps=0, mseThreshold=0.0, useReflections=False,
            seed=5489, minSample=0, maxSample=None, weights=None, threads=0, nearField=True):
    """Adaptive backward phi-ASE over samples [minSample, maxSample] (FP64)."""
    keep = _Keep()
    m = _mesh_struct(mesh, keep)
    s = _spectrum_struct(spectrum, keep)
    n_samples_total = np.asarray(mesh.points).reshape(-1, 2).shape[0] * int(mesh.numberOfLevels)
    maxSample = n_samples_total - 1 if maxSample is None else int(maxSample)
    e = _Experiment(int(minRays), int(maxRays if maxRays is not None else minRays), int(adaptiveSteps),
                    float(mseThreshold), 1 if useReflections else 0, int(seed) & 0xFFFFFFFF, int(minSample),
                    maxSample, 1 if nearField else 0)
    n = maxSample - int(minSample) + 1
    out = {
        "phiAse": np.empty(n), "mse": np.empty(n), "totalRays": np.empty(n, np.uint32),
        "dndtAse": np.empty(n), "droppedRays": np.empty(n, np.uint32), "gainSum": np.empty(n),
        "gainSumSquare": np.empty(n),
    }
    r = _Result(*[_ptr(out[k], _u32p if out[k].dtype == np.uint32 else _f64p) for k in
                  ("phiAse", "mse", "totalRays", "dndtAse", "droppedRays", "gainSum", "gainSumSquare")])
    wptr = None
    if weights is not None:
        weights = keep(np.ascontiguousarray(np.asarray(weights, np.float32)))
        wptr = _ptr(weights, _f32p)
    rc = lib().oracle_phi_ase(C.byref(m), C.byref(s), C.byref(e), wptr, int(threads or os.cpu_count() or 1),
                              C.byref(r))
    if rc:
        raise ValueError(f"oracle_phi_ase failed ({rc})")
    return out


# ---- forward Tet4 estimator -------------------------------------------------

class _TetMesh(C.Structure):
    _fields_ = [
        ("numberOfPoints", C.c_uint32),
        ("numberOfCells", C.c_uint32),
        ("points", _f64p),
        ("cells", _u32p),
        ("betaVolume", _f64p),
        ("claddingCellTypes", _u32p),
        ("claddingNumber", C.c_uint32),
        ("claddingAbsorption", C.c_double),
        ("nTot", C.c_double),
        ("crystalTFluo", C.c_double),
        ("cellFaceBoundaries", _i32p),
        ("numberOfSurfaces", C.c_uint32),
        ("surfaceReflectivities", _f64p),
        ("surfaceRefractiveIndexInside", _f64p),
        ("surfaceRefractiveIndexOutside", _f64p),
        ("reflectivities", _f64p),
        ("refractiveIndices", _f64p),
    ]


class _FwdExperiment(C.Structure):
    _fields_ = [
        ("minRays", C.c_uint32),
        ("maxRays", C.c_uint32),
        ("adaptiveSteps", C.c_uint32),
        ("rseThreshold", C.c_double),
        ("seed", C.c_uint32),
        ("batches", C.c_uint32),
        ("useReflections", C.c_uint32),
        ("reflectionMaxIterations", C.c_uint32),
        ("reflectionTolerance", C.c_double),
        ("surfaceReservoirSize", C.c_uint32),
        ("divergenceStreak", C.c_uint32),
    ]


class _FwdResult(C.Structure):
    _fields_ = [
        ("phiAse", _f64p),
        ("relativeStandardError", _f64p),
        ("dndtAse", _f64p),
        ("droppedRays", _u32p),
        ("rayVisits", _u32p),
        ("totalRays", C.c_uint64),
        ("launches", C.c_uint32),
        ("srmStatus", C.c_uint32),
        ("srmPasses", C.c_uint32),
        ("srmRemainingFraction", C.c_double),
    ]


def _tet_struct(mesh, keep):
    pts = keep(np.ascontiguousarray(np.asarray(mesh.points, np.float64).reshape(-1, 3)))
    cells = keep(np.ascontiguousarray(np.asarray(mesh.cells, np.uint32).reshape(-1, 4)))
    beta = keep(np.ascontiguousarray(np.asarray(mesh.betaVolume, np.float64).ravel()))
    clad = None if getattr(mesh, "claddingCellTypes", None) is None else keep(
        np.ascontiguousarray(np.asarray(mesh.claddingCellTypes, np.uint32).ravel()))
    def opt(name, dtype):
        v = getattr(mesh, name, None)
        return None if v is None else keep(np.ascontiguousarray(np.asarray(v, dtype).ravel()))

    bnd = opt("cellFaceBoundaries", np.int32)
    surf = mesh.surfaceArrays() if hasattr(mesh, "surfaceArrays") else (None, None, None)
    surf = [None if v is None else keep(np.ascontiguousarray(v, np.float64)) for v in surf]
    nsurf = max([0] + [v.size for v in surf if v is not None])
    return _TetMesh(pts.shape[0], cells.shape[0], _ptr(pts, _f64p), _ptr(cells, _u32p), _ptr(beta, _f64p),
                    _ptr(clad, _u32p), int(getattr(mesh, "claddingNumber", 1)),
                    float(getattr(mesh, "claddingAbsorption", 0.0)), float(mesh.nTot), float(mesh.crystalTFluo),
                    _ptr(bnd, _i32p), nsurf, *[_ptr(v, _f64p) for v in surf],
                    _ptr(opt("reflectivities", np.float64), _f64p), _ptr(opt("refractiveIndices", np.float64), _f64p))


def tet_tables(mesh):
    keep = _Keep()
    m = _tet_struct(mesh, keep)
    Cn = m.numberOfCells
    out = {"neighbors": np.empty((Cn, 4), np.int32), "neighborFace": np.empty((Cn, 4), np.int32),
           "gradients": np.empty((Cn, 4, 3)), "volumes": np.empty(Cn)}
    rc = lib().oracle_tet_tables(C.byref(m), _ptr(out["neighbors"], _i32p), _ptr(out["neighborFace"], _i32p),
                                 _ptr(out["gradients"], _f64p), _ptr(out["volumes"], _f64p))
    if rc:
        raise ValueError(f"oracle_tet_tables failed ({rc})")
    return out


SRM_STATUS = ("disabled", "converged", "stable", "diverged", "max_iterations")


def forward_phi_ase(mesh, spectrum, *, minRays, maxRays=None, adaptiveSteps=0, rseThreshold=0.0, seed=5489,
                    batches=8, threads=0, useReflections=False, reflectionMaxIterations=40, reflectionTolerance=1e-4,
                    surfaceReservoirSize=32, divergenceStreak=3):
    """Forward Tet4 phi-ASE per cell (FP64), with the surface-reservoir
    reflection passes when ``useReflections``."""
    keep = _Keep()
    m = _tet_struct(mesh, keep)
    s = _spectrum_struct(spectrum, keep)
    n = m.numberOfCells
    out = {"phiAse": np.empty(n), "relativeStandardError": np.empty(n), "dndtAse": np.empty(n),
           "droppedRays": np.empty(n, np.uint32), "rayVisits": np.empty(n, np.uint32)}
    r = _FwdResult(_ptr(out["phiAse"], _f64p), _ptr(out["relativeStandardError"], _f64p),
                   _ptr(out["dndtAse"], _f64p), _ptr(out["droppedRays"], _u32p), _ptr(out["rayVisits"], _u32p), 0, 0)
    e = _FwdExperiment(int(minRays), int(maxRays if maxRays is not None else minRays), int(adaptiveSteps),
                       float(rseThreshold), int(seed) & 0xFFFFFFFF, int(batches), 1 if useReflections else 0,
                       int(reflectionMaxIterations), float(reflectionTolerance), int(surfaceReservoirSize),
                       int(divergenceStreak))
    rc = lib().oracle_forward_phi_ase(C.byref(m), C.byref(s), C.byref(e), int(threads or os.cpu_count() or 1),
                                      C.byref(r))
    if rc:
        raise ValueError(f"oracle_forward_phi_ase failed ({rc})")
    out["totalRays"] = int(r.totalRays)
    out["launches"] = int(r.launches)
    out["srmStatus"] = SRM_STATUS[r.srmStatus]
    out["srmPasses"] = int(r.srmPasses)
    out["srmRemainingFraction"] = float(r.srmRemainingFraction)
    return out


def tet_trace(mesh, spectrum, start_cell, origin, direction, *, wavelength=0, max_segments=64):
    """Single rays through a Tet4 mesh: segments, cells, lengths, lnGain, endPoint, status."""
    keep = _Keep()
    m = _tet_struct(mesh, keep)
    s = _spectrum_struct(spectrum, keep)
    sc = keep(np.ascontiguousarray(np.atleast_1d(np.asarray(start_cell, np.uint32))))
    o = keep(np.ascontiguousarray(np.asarray(origin, np.float64).reshape(-1, 3)))
    d = keep(np.ascontiguousarray(np.asarray(direction, np.float64).reshape(-1, 3)))
    n = sc.size
    if o.shape[0] != n or d.shape[0] != n:
        raise ValueError("start_cell, origin and direction must describe the same rays")
    out = {"segments": np.empty(n, np.uint32), "cells": np.zeros((n, max_segments), np.uint32),
           "lengths": np.zeros((n, max_segments)), "lnGain": np.empty(n), "endPoint": np.empty((n, 3)),
           "status": np.empty(n, np.int32)}
    rc = lib().oracle_tet_trace(C.byref(m), C.byref(s), int(wavelength), n, _ptr(sc, _u32p), _ptr(o, _f64p),
                                _ptr(d, _f64p), int(max_segments), _ptr(out["segments"], _u32p),
                                _ptr(out["cells"], _u32p), _ptr(out["lengths"], _f64p), _ptr(out["lnGain"], _f64p),
                                _ptr(out["endPoint"], _f64p), _ptr(out["status"], _i32p))
    if rc:
        raise ValueError(f"oracle_tet_trace failed ({rc})")
    return out
