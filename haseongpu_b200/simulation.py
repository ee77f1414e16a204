"""Host front end mirroring the reference's ``PhiASE`` call surface.

``PhiASE`` keeps the field names, ``run(gainMedium, crossSections)`` ->
``self`` and ``getResults()`` -> ``Result`` of pyInclude/simulation.py:110-489,
and ``Result`` the fields of pyInclude/structures.py:7-18.  Where the reference
hands the medium to the ``calcPhiASE`` executable through openPMD files
(pyInclude/openpmd/transport.py:1696-1717), this front end calls
libhase_b200.so directly through its C ABI (include/hase_b200.h).

Two propagation modes:

* ``"forward"`` (the default, as in the reference): the reference's current
  method on a Tet4 medium (``TetMesh``; a ``PrismMesh`` is split into its
  Tet4 twin), results per cell (include/hase_b200_forward.h).
* ``"backward"``: the importance-sampled prism method on a ``PrismMesh``,
  results per sample point (include/hase_b200.h).

The threshold is the relative standard error of each estimate, as the legacy
``mseThreshold`` and the reference's ``relativeStandardErrorThreshold``.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .mesh import PrismMesh
from .spectra import CrossSectionData


@dataclass
class Result:
    phiAse: np.ndarray = field(default_factory=lambda: np.empty(0, np.float32))
    standardError: np.ndarray = field(default_factory=lambda: np.empty(0))
    relativeStandardError: np.ndarray = field(default_factory=lambda: np.empty(0))
    totalRays: np.ndarray = field(default_factory=lambda: np.empty(0, np.uint32))
    dndtAse: np.ndarray = field(default_factory=lambda: np.empty(0))
    droppedRays: np.ndarray = field(default_factory=lambda: np.empty(0, np.uint32))
    srmStatus: str = "disabled"
    srmPasses: int = 0
    srmRemainingFraction: float = 0.0
    srmMaxIterations: int = 0
    srmDivergenceStreak: int = 0
    reflectingFaces: int = 0
    raysTraced: int = 0
    crossings: int = 0
    importanceMilliseconds: float = 0.0
    rayMilliseconds: float = 0.0
    totalMilliseconds: float = 0.0
    passes: int = 0
    unconvergedSamples: int = 0
    kernelLaunches: int = 0
    tallyMode: int = 0
    fallbackSamples: int = 0
    status: int = 0
    # backward solves: the legacy archives' ``mse``, the standard error of the
    # unnormalised estimator phi tau / N_tot (a length): RSE * phi * tau / N_tot
    legacyMse: np.ndarray = field(default_factory=lambda: np.empty(0))

    @property
    def mse(self) -> np.ndarray:
        """Legacy name of the per-sample relative standard error (the quantity
        every threshold applies to; ``legacyMse`` is the legacy archives' value)."""
        return self.relativeStandardError


# The reference's time integrators (pyInclude/openpmd/transport.py:1719-1727) and their
# hase_time_desc.integrator codes.
TIME_INTEGRATORS = {"frozen-phi-ase-runge-kutta-4": 0, "explicit-euler": 1, "heun": 2, "midpoint": 3,
                    "runge-kutta-4": 4, "implicit-euler": 5, "exponential-euler": 6}


def time_integrator(name) -> int:
    """The integrator code of a reference integrator name (or a code)."""
    if isinstance(name, str):
        if name not in TIME_INTEGRATORS:
            raise ValueError(f"unknown time integrator {name!r}; known: {', '.join(TIME_INTEGRATORS)}")
        return TIME_INTEGRATORS[name]
    code = int(name)
    if not 0 <= code < len(TIME_INTEGRATORS):
        raise ValueError(f"integrator code {code} outside 0 .. {len(TIME_INTEGRATORS) - 1}")
    return code


def solves_per_step(integrator, implicitIterations=0) -> int:
    """phi-ASE solves of one time step with phi-ASE on: the stages that re-solve it."""
    code = time_integrator(integrator)
    return {2: 2, 3: 2, 4: 4, 5: max(1, int(implicitIterations) or 8)}.get(code, 1)


class DeviceMesh:
    """A libhase_b200 context: the mesh tables resident on one device."""

    def __init__(self, mesh: PrismMesh, sigmaA, sigmaE, device: int = 0):
        self.mesh = mesh
        self._keep = []
        sa = self._hold(np.atleast_1d(np.asarray(sigmaA, np.float64)))
        se = self._hold(np.atleast_1d(np.asarray(sigmaE, np.float64)))
        if sa.size != se.size or sa.size == 0:
            raise ValueError("sigmaA and sigmaE must be non-empty and of equal length")
        desc = self._mesh_desc(mesh)
        spec = N.SpectrumDesc(sa.size, N.ptr(sa, N._f64p), N.ptr(se, N._f64p))
        handle = C.c_void_p()
        N.check(N.lib().hase_context_create(C.byref(desc), C.byref(spec), int(device), C.byref(handle)))
        self.handle = handle
        self.numberOfWavelengths = sa.size
        self.sigmaA, self.sigmaE = sa, se
        self.localTriangles = 0

    def set_local_proposal(self, triangles: int, farFraction: float = 0.0):
        """Local proposal (hase_context_set_local_proposal): per sample point its
        ``triangles`` nearest triangles x layers x slices as weighted candidates,
        a ``farFraction`` of the rays (0: 0.9) drawn from a beta V gain / d^2
        prior over the whole medium, every ray weighted by the mixture's
        probability; 0 restores the full proposal."""
        N.check(N.lib().hase_context_set_local_proposal(self.handle, int(triangles), float(farFraction)))
        self.localTriangles = min(int(triangles), self.mesh.numberOfTriangles)

    def set_grid_proposal(self, enable: bool = True):
        """Coarse-grid proposal (hase_context_set_grid_proposal): plain solves
        take their weights from the coarse gain grid instead of the importance
        walks; False restores the walks."""
        N.check(N.lib().hase_context_set_grid_proposal(self.handle, 1 if enable else 0))

    def grid_weights(self, firstSample, count, useReflections=False, monochromatic=False) -> np.ndarray:
        """The coarse-grid proposal's normalised weights (hase_grid_weights)."""
        slices = 5 if useReflections else 1
        w = np.empty((count, self.row_entries(slices)), np.float32)
        N.check(N.lib().hase_grid_weights(self.handle, int(firstSample), int(count), 1 if useReflections else 0,
                                          1 if monochromatic else 0, N.ptr(w, N._f32p)))
        return w

    def row_entries(self, slices: int) -> int:
        """Entries of a sample's weight row: every (slice, prism), or the local
        proposal's (slice, layer, candidate) entries."""
        if self.localTriangles:
            return slices * (self.mesh.numberOfLevels - 1) * self.localTriangles
        return slices * self.mesh.numberOfPrisms

    def _hold(self, a):
        a = np.ascontiguousarray(a)
        self._keep.append(a)
        return a

    def _mesh_desc(self, m: PrismMesh):
        def opt(a, t, dtype):
            return None if a is None else N.ptr(self._hold(np.asarray(a, dtype).ravel()), t)

        return N.MeshDesc(
            m.numberOfPoints, m.numberOfTriangles, m.numberOfLevels, N.ptr(self._hold(m.points), N._f64p),
            N.ptr(self._hold(m.triangles), N._u32p), m.thickness, N.ptr(self._hold(m.betaVolume), N._f64p),
            opt(m.betaCells, N._f64p, np.float64), opt(m.claddingCellTypes, N._u32p, np.uint32),
            int(m.claddingNumber), float(m.claddingAbsorption), float(m.nTot), float(m.crystalTFluo),
            opt(m.reflectivities, N._f64p, np.float64), opt(m.refractiveIndices, N._f64p, np.float64))

    def update_beta(self, betaVolume, betaCells=None):
        bv = np.ascontiguousarray(np.asarray(betaVolume, np.float64).ravel())
        if bv.size != self.mesh.numberOfPrisms:
            raise ValueError("betaVolume size mismatch")
        bc = None if betaCells is None else np.ascontiguousarray(np.asarray(betaCells, np.float64).ravel())
        if bc is not None and bc.size != self.mesh.numberOfSamples:
            raise ValueError("betaCells size mismatch")
        N.check(N.lib().hase_context_update_beta(self.handle, N.ptr(bv, N._f64p), N.ptr(bc, N._f64p)))

    def _descs(self, minRays, maxRays, mseThreshold, useReflections, monochromatic, nearFieldSampling, adaptiveSteps,
               repetitions, rngSeed, minSample, maxSample, raysPerThread, blockSize, workspaceBytes, rayKernelVariant,
               importanceLayers):
        S = self.mesh.numberOfSamples
        maxSample = S - 1 if maxSample is None else int(maxSample)
        n = maxSample - int(minSample) + 1
        if n <= 0:
            raise ValueError("empty sample range")
        out = Result(phiAse=np.empty(n, np.float32), standardError=np.empty(n), relativeStandardError=np.empty(n),
                     totalRays=np.empty(n, np.uint32), dndtAse=np.empty(n), droppedRays=np.empty(n, np.uint32))
        ex = N.ExperimentDesc(int(minRays), int(maxRays if maxRays is not None else minRays), float(mseThreshold),
                              1 if useReflections else 0, 1 if monochromatic else 0, 1 if nearFieldSampling else 0)
        cp = N.ComputeDesc(int(adaptiveSteps), int(repetitions), int(rngSeed) & 0xFFFFFFFF, int(minSample), maxSample,
                           int(raysPerThread), int(blockSize), int(workspaceBytes), int(rayKernelVariant),
                           int(importanceLayers))
        r = N.ResultDesc(N.ptr(out.phiAse, N._f32p), N.ptr(out.standardError, N._f64p),
                         N.ptr(out.relativeStandardError, N._f64p), N.ptr(out.totalRays, N._u32p),
                         N.ptr(out.dndtAse, N._f64p), N.ptr(out.droppedRays, N._u32p))
        return out, ex, cp, r, n

    @staticmethod
    def _fill(out, r, status):
        out.status = status
        out.raysTraced = int(r.raysTraced)
        out.crossings = int(r.crossings)
        out.importanceMilliseconds = float(r.importanceMilliseconds)
        out.rayMilliseconds = float(r.rayMilliseconds)
        out.totalMilliseconds = float(r.totalMilliseconds)
        out.passes = int(r.passes)
        out.unconvergedSamples = int(r.unconvergedSamples)
        out.kernelLaunches = int(r.kernelLaunches)
        return out

    def calc_phi_ase_learned(self, net, *, minRays, maxRays=None, mseThreshold=0.0, useReflections=False,
                             monochromatic=False, nearFieldSampling=True, adaptiveSteps=0, rngSeed=5489, minSample=0,
                             maxSample=None, mixture=0.0, fallbackVariance=0.0, workspaceBytes=0, rayKernelVariant=0,
                             raysPerThread=0) -> Result:
        """The solve with the learned proposal ``net`` (a ProposalNet on the same device)."""
        out, ex, cp, r, _ = self._descs(minRays, maxRays, mseThreshold, useReflections, monochromatic,
                                        nearFieldSampling, adaptiveSteps, 1, rngSeed, minSample, maxSample,
                                        raysPerThread, 0, workspaceBytes, rayKernelVariant, 0)
        ld = N.LearnedDesc(float(mixture), float(fallbackVariance), 0)
        status = N.check(N.lib().hase_calc_phi_ase_learned(self.handle, net.handle, C.byref(ex), C.byref(cp),
                                                           C.byref(ld), C.byref(r)), allow_warnings=True)
        self._fill(out, r, status)
        out.fallbackSamples = int(ld.fallbackSamples)
        return self._legacy_mse(out)

    def log_contributions(self, *, minRays, useReflections=False, monochromatic=False, nearFieldSampling=True,
                          rngSeed=5489, minSample=0, maxSample=None):
        """One pass of `minRays` rays per sample with the importance weights;
        returns (Result, contributions [samples][slices * P]) -- the summed ray
        contributions per (slice, prism), the proposal's training targets."""
        out, ex, cp, r, n = self._descs(minRays, minRays, 0.0, useReflections, monochromatic, nearFieldSampling, 0, 1,
                                        rngSeed, minSample, maxSample, 0, 0, 0, 0, 0)
        slices = 5 if useReflections else 1
        contrib = np.empty((n, self.row_entries(slices)), np.float32)
        status = N.check(N.lib().hase_log_contributions(self.handle, C.byref(ex), C.byref(cp),
                                                        N.ptr(contrib, N._f32p), C.byref(r)), allow_warnings=True)
        return self._fill(out, r, status), contrib

    @staticmethod
    def _time_descs(pump, time, width, keepPhi, P):
        pd = N.PumpDesc(float(pump["peakIntensity"]), float(pump["radius"]), float(pump["exponent"]),
                        float(pump.get("centerX", 0.0)), float(pump.get("centerY", 0.0)), float(pump["wavelength"]),
                        float(pump["sigmaA"]), float(pump["sigmaE"]), 1 if pump.get("retroreflect", True) else 0)
        steps = int(time["steps"])
        integrator = time_integrator(time.get("integrator", 0))
        iterations = int(time.get("implicitIterations", 0))
        td = N.TimeDesc(float(time["timeStep"]), steps, int(time.get("pumpSteps", steps)),
                        int(time.get("aseSteps", steps)), integrator, iterations)
        out = {"betaVolume": np.empty(P), "meanBeta": np.empty(steps + 1), "meanPhi": np.empty(steps),
               "pumpAbsorbed": np.empty(steps)}
        if keepPhi:
            out["phiHistory"] = np.empty((td.aseSteps * solves_per_step(integrator, iterations), width), np.float32)
        r = N.TimeResultDesc(N.ptr(out["betaVolume"], N._f64p), N.ptr(out["meanBeta"], N._f64p),
                             N.ptr(out["meanPhi"], N._f64p), N.ptr(out["pumpAbsorbed"], N._f64p),
                             N.ptr(out.get("phiHistory"), N._f32p))
        return pd, td, r, out

    @staticmethod
    def _time_out(out, r):
        out.update(aseMilliseconds=r.aseMilliseconds, pumpMilliseconds=r.pumpMilliseconds,
                   totalMilliseconds=r.totalMilliseconds, raysTraced=int(r.raysTraced),
                   fallbackSamples=int(r.fallbackSamples))
        return out

    def simulate(self, *, pump, time, net=None, fallbackVariance=0.0, minRays, maxRays=None, mseThreshold=0.0,
                 useReflections=False, monochromatic=False, nearFieldSampling=True, adaptiveSteps=0, rngSeed=5489,
                 keepPhi=False) -> dict:
        """Time-stepped rate equations (hase_simulate): `pump` and `time` are
        dicts with the fields of hase_pump_desc / hase_time_desc.  The
        context's beta is advanced in place."""
        _, ex, cp, _, _ = self._descs(minRays, maxRays, mseThreshold, useReflections, monochromatic, nearFieldSampling,
                                      adaptiveSteps, 1, rngSeed, 0, None, 0, 0, 0, 0, 0)
        pd, td, r, out = self._time_descs(pump, time, self.mesh.numberOfSamples, keepPhi, self.mesh.numberOfPrisms)
        out["status"] = N.check(N.lib().hase_simulate(self.handle, net.handle if net is not None else None,
                                                      float(fallbackVariance), C.byref(ex), C.byref(cp), C.byref(pd),
                                                      C.byref(td), C.byref(r)), allow_warnings=True)
        return self._time_out(out, r)

    def simulate_forward(self, twin, *, pump, time, forwardRayCount, maxRays=None, adaptiveSteps=0,
                         relativeStandardErrorThreshold=0.0, monochromatic=False, rngSeed=5489, batches=8,
                         useReflections=False, reflectionMaxIterations=40, reflectionTolerance=1.0e-4,
                         surfaceReservoirSize=32, keepPhi=False) -> dict:
        """Time-stepped rate equations with the ASE term from the forward
        method (hase_simulate_forward) on ``twin``, a TetDeviceMesh of
        ``TetMesh.fromPrismMesh(self.mesh)``.  ``phiHistory`` (keepPhi) is
        per prism.  The context's beta is advanced in place."""
        fw = N.ForwardDesc(int(forwardRayCount), int(maxRays if maxRays is not None else forwardRayCount),
                           int(adaptiveSteps), float(relativeStandardErrorThreshold), 1 if monochromatic else 0,
                           int(rngSeed) & 0xFFFFFFFF, int(batches), 0, 0, 1 if useReflections else 0,
                           int(reflectionMaxIterations), float(reflectionTolerance), int(surfaceReservoirSize), 0)
        P = self.mesh.numberOfPrisms
        pd, td, r, out = self._time_descs(pump, time, P, keepPhi, P)
        out["status"] = N.check(N.lib().hase_simulate_forward(self.handle, twin.handle, C.byref(fw), C.byref(pd),
                                                              C.byref(td), C.byref(r)), allow_warnings=True)
        return self._time_out(out, r)

    def proposal_features(self, firstSample, count, useReflections=False, monochromatic=False) -> np.ndarray:
        slices = 5 if useReflections else 1
        f = np.empty((int(count), self.row_entries(slices), N.PROPOSAL_FEATURES), np.float32)
        N.check(N.lib().hase_proposal_features(self.handle, int(firstSample), int(count), 1 if useReflections else 0,
                                               1 if monochromatic else 0, N.ptr(f, N._f32p)))
        return f

    def calc_phi_ase(self, *, minRays, maxRays=None, mseThreshold=0.0, useReflections=False, monochromatic=False,
                     nearFieldSampling=True, adaptiveSteps=0, repetitions=1, rngSeed=5489, minSample=0, maxSample=None, raysPerThread=0,
                     blockSize=0, workspaceBytes=0, rayKernelVariant=0, importanceLayers=0) -> Result:
        out, ex, cp, r, _ = self._descs(minRays, maxRays, mseThreshold, useReflections, monochromatic,
                                        nearFieldSampling, adaptiveSteps, repetitions, rngSeed, minSample, maxSample,
                                        raysPerThread, blockSize, workspaceBytes, rayKernelVariant, importanceLayers)
        status = N.check(N.lib().hase_calc_phi_ase(self.handle, C.byref(ex), C.byref(cp), C.byref(r)),
                         allow_warnings=True)
        out.status = status
        out.raysTraced = int(r.raysTraced)
        out.crossings = int(r.crossings)
        out.importanceMilliseconds = float(r.importanceMilliseconds)
        out.rayMilliseconds = float(r.rayMilliseconds)
        out.totalMilliseconds = float(r.totalMilliseconds)
        out.passes = int(r.passes)
        out.unconvergedSamples = int(r.unconvergedSamples)
        out.kernelLaunches = int(r.kernelLaunches)
        return self._legacy_mse(out)

    def _legacy_mse(self, out: Result) -> Result:
        out.legacyMse = out.relativeStandardError * out.phiAse.astype(np.float64) * (
            float(self.mesh.crystalTFluo) / float(self.mesh.nTot))
        return out

    def importance_weights(self, firstSample, count, useReflections=False) -> np.ndarray:
        slices = 5 if useReflections else 1
        w = np.empty((count, self.row_entries(slices)), np.float32)
        N.check(N.lib().hase_importance_weights(self.handle, int(firstSample), int(count), 1 if useReflections else 0,
                                                N.ptr(w, N._f32p)))
        return w

    def importance_crossings(self, firstSample, count, useReflections=False) -> int:
        """Crossings of the importance walks of the samples (hase_importance_crossings)."""
        n = np.zeros(1, np.uint64)
        N.check(N.lib().hase_importance_crossings(self.handle, int(firstSample), int(count),
                                                  1 if useReflections else 0, N.ptr(n, N._u64p)))
        return int(n[0])

    def learned_weights(self, net, firstSample, count, useReflections=False, monochromatic=False,
                        mixture=0.0) -> np.ndarray:
        """The learned proposal's normalised first-pass weights (hase_learned_weights)."""
        slices = 5 if useReflections else 1
        w = np.empty((count, self.row_entries(slices)), np.float32)
        N.check(N.lib().hase_learned_weights(self.handle, net.handle, int(firstSample), int(count),
                                             1 if useReflections else 0, 1 if monochromatic else 0, float(mixture),
                                             N.ptr(w, N._f32p)))
        return w

    def trace(self, start, tri, level, sample, slice_=None, wavelength=0):
        start = np.ascontiguousarray(np.asarray(start, np.float32).reshape(-1, 3))
        n = start.shape[0]
        arrs = [np.ascontiguousarray(np.asarray(a, np.uint32).reshape(n)) for a in
                (tri, level, sample, np.zeros(n) if slice_ is None else slice_)]
        ln = np.empty(n, np.float32)
        dist = np.empty(n, np.float32)
        dropped = np.empty(n, np.uint32)
        N.check(N.lib().hase_trace_rays(self.handle, n, N.ptr(start, N._f32p), *[N.ptr(a, N._u32p) for a in arrs],
                                        int(wavelength), N.ptr(ln, N._f32p), N.ptr(dist, N._f32p),
                                        N.ptr(dropped, N._u32p)))
        return ln, dist, dropped

    def close(self):
        if getattr(self, "handle", None):
            N.lib().hase_context_destroy(self.handle)
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


@dataclass
class PhiASE:
    """Configure and run the phi-ASE calculation for one gain-medium state."""

    config: object | None = None
    crossSections: CrossSectionData | None = None
    gainMedium: object | None = None       # TetMesh (forward) or PrismMesh
    propagationMode: str = "forward"
    minRays: int = 100000
    maxRays: int = 100000
    forwardRayCount: int | None = None
    relativeStandardErrorThreshold: float = 0.1
    repetitions: int = 4
    adaptiveSteps: int = 4
    useReflections: bool = False
    reflectionMaxIterations: int = 40
    reflectionTolerance: float = 1e-4
    surfaceReservoirSize: int = 32
    monochromatic: bool = False
    nearFieldSampling: bool = True
    backend: str | None = "cuda_sm100a"
    parallelMode: str = "single"
    numDevices: int = 1
    devices: list[int] = field(default_factory=list)
    minSampleRange: int | None = None
    maxSampleRange: int | None = None
    rngSeed: int | None = None
    writeVtk: bool = False

    _result: Result | None = field(default=None, init=False, repr=False)
    _context: object | None = field(default=None, init=False, repr=False)
    _tetTwin: tuple | None = field(default=None, init=False, repr=False)

    def __post_init__(self):
        if isinstance(self.config, dict):
            for key, value in self.config.items():
                if key == "mseThreshold":
                    raise ValueError("mseThreshold is named relativeStandardErrorThreshold")
                if not hasattr(self, key):
                    raise ValueError(f"unknown PhiASE setting '{key}'")
                setattr(self, key, value)
        if self.propagationMode not in ("forward", "backward"):
            raise ValueError("propagationMode must be 'forward' (Tet4 source rays) or 'backward' "
                             "(importance-sampled prism method)")
        if self.parallelMode != "single":
            raise ValueError("parallelMode must be 'single'; use one process per GPU for replicas")
        if self.backend not in (None, "cuda_sm100a"):
            raise ValueError(f"unknown backend '{self.backend}'; available: cuda_sm100a")
        if self.minRays <= 0 or self.maxRays < self.minRays and self.maxRays != 0:
            raise ValueError("need 0 < minRays <= maxRays")
        if self.relativeStandardErrorThreshold < 0:
            raise ValueError("relativeStandardErrorThreshold must be >= 0")

    def _device(self) -> int:
        return int(self.devices[0]) if self.devices else 0

    def run(self, gainMedium=None, crossSections: CrossSectionData | None = None) -> "PhiASE":
        medium = gainMedium if gainMedium is not None else self.gainMedium
        if medium is None:
            raise ValueError("PhiASE.run requires gainMedium")
        spectra = crossSections if crossSections is not None else self.crossSections
        if spectra is None:
            raise ValueError("PhiASE.run requires crossSections")
        sigmaA, sigmaE = spectra.resampled(self.monochromatic)
        if self.propagationMode == "forward":
            return self._run_forward(medium, sigmaA, sigmaE)
        if not isinstance(medium, PrismMesh):
            raise ValueError("propagationMode='backward' needs a PrismMesh gain medium")
        ctx = self._context
        if ctx is None or ctx.mesh is not medium or ctx.numberOfWavelengths != sigmaA.size:
            if ctx is not None:
                ctx.close()
            ctx = DeviceMesh(medium, sigmaA, sigmaE, device=self._device())
            self._context = ctx
        rays = self.forwardRayCount
        minRays = rays if rays else self.minRays
        maxRays = rays if rays else max(self.maxRays, self.minRays)
        self._result = ctx.calc_phi_ase(
            minRays=minRays, maxRays=maxRays, mseThreshold=self.relativeStandardErrorThreshold,
            useReflections=self.useReflections, monochromatic=self.monochromatic,
            nearFieldSampling=self.nearFieldSampling, adaptiveSteps=0 if rays else self.adaptiveSteps, repetitions=self.repetitions,
            rngSeed=5489 if self.rngSeed is None else self.rngSeed,
            minSample=self.minSampleRange or 0, maxSample=self.maxSampleRange)
        return self

    def _run_forward(self, medium, sigmaA, sigmaE) -> "PhiASE":
        from .forward import TetDeviceMesh
        from .tetmesh import TetMesh

        if isinstance(medium, PrismMesh):
            key = medium
            if self._tetTwin is None or self._tetTwin[0] is not medium:
                self._tetTwin = (medium, TetMesh.fromPrismMesh(medium))
            medium = self._tetTwin[1]
        elif not isinstance(medium, TetMesh):
            raise ValueError("propagationMode='forward' needs a TetMesh or PrismMesh gain medium")
        else:
            key = medium
        ctx = self._context
        if (not isinstance(ctx, TetDeviceMesh) or ctx.source is not key
                or ctx.numberOfWavelengths != sigmaA.size):
            if ctx is not None:
                ctx.close()
            ctx = TetDeviceMesh(medium, sigmaA, sigmaE, device=self._device())
            ctx.source = key
            self._context = ctx
        rays = self.forwardRayCount
        minRays = rays if rays else self.minRays
        maxRays = rays if rays else max(self.maxRays, self.minRays)
        self._result = ctx.calc_phi_ase(
            forwardRayCount=minRays, maxRays=maxRays, adaptiveSteps=0 if rays else self.adaptiveSteps,
            relativeStandardErrorThreshold=self.relativeStandardErrorThreshold, monochromatic=self.monochromatic,
            rngSeed=5489 if self.rngSeed is None else self.rngSeed, useReflections=self.useReflections,
            reflectionMaxIterations=self.reflectionMaxIterations, reflectionTolerance=self.reflectionTolerance,
            surfaceReservoirSize=self.surfaceReservoirSize)
        self._result.standardError = self._result.relativeStandardError * self._result.phiAse
        return self

    def getResults(self) -> Result:
        if self._result is None:
            raise RuntimeError("simulation has not been run yet")
        return self._result
