"""Drop-in for the reference's Python call surface.

The reference's ``PhiASE.run`` hands every solve to one function,
``transport.runPhiASE(phiAse, gainMedium, crossSections, **options)``
(pyInclude/simulation.py:452-483, pyInclude/openpmd/transport.py:1696-1716),
which writes the medium to an openPMD series and runs the ``calcPHiASE``
executable; its own tests replace exactly that function
(tests/python/phiAse/test_simulationWrapper.py:51-86).  ``runPhiASE`` here
has the same signature and returns a ``Result`` with the reference's field
names, solved by libhase_b200 on the GPU instead:

    import pyInclude.simulation as simulation
    from haseongpu_b200.reference_binding import runPhiASE
    simulation.transport.runPhiASE = runPhiASE

The reference's objects are read by their v2.2.0 attribute names, without
importing the reference:

* ``GainMedium`` (pyInclude/geometry/core.py:1080): ``topology`` is a
  ``MeshTopology`` (``points`` [Np, 2], ``trianglePointIndices`` [T, 3],
  ``levels``, ``thickness``; a prism mesh) or a ``VolumeTopology``
  (pyInclude/geometry/volume.py:231: ``points`` [V, 3], ``cellPointIndices``
  [C, 4], ``faceBoundaries`` [C, 4]; a Tet4 mesh with its surface optics);
  the physical properties come from ``get(name).value`` (``betaVolume`` in
  Fortran order: prism t + l T, as this package's layout).
* ``SpectralDecomposition``: ``wavelengths*`` / ``crossSection*`` arrays and
  ``resolution`` (the names of this package's ``CrossSectionData``).
* ``PhiASE``: the solver fields of pyInclude/simulation.py:130-176 this build
  implements (propagation mode, ray counts, threshold, adaptive steps,
  reflections, monochromatic, seed, sample range); the transport-only fields
  (openPMD backend, workspace, watchdog, MPI layout) have no meaning here.
"""

from __future__ import annotations

import numpy as np

from .mesh import PrismMesh
from .simulation import PhiASE as _PhiASE
from .simulation import Result
from .spectra import CrossSectionData
from .tetmesh import TetMesh

# PhiASE fields copied onto this package's PhiASE (same names and meaning).
SOLVER_FIELDS = ("propagationMode", "minRays", "maxRays", "forwardRayCount", "relativeStandardErrorThreshold",
                 "repetitions", "adaptiveSteps", "useReflections", "reflectionMaxIterations", "reflectionTolerance",
                 "surfaceReservoirSize", "monochromatic", "rngSeed", "minSampleRange", "maxSampleRange")

_PROPERTIES = ("betaVolume", "claddingCellTypes", "claddingNumber", "claddingAbsorption", "nTot", "crystalTFluo")


def _property(medium, name, default=None):
    try:
        value = medium.get(name).value
    except (KeyError, ValueError, AttributeError):
        return default
    return default if value is None else value


def point_beta(triangles, numberOfPoints, numberOfLevels, betaVolume):
    """beta at every sample point (point p at level k): the mean beta of the
    prisms that have the point as a vertex (layers k - 1 and k) -- the input
    of dndtAse for a medium that carries beta per prism only (v2.2.0 has no
    ``betaCells``)."""
    T = triangles.shape[0]
    L = numberOfLevels - 1
    beta = np.asarray(betaVolume, np.float64).reshape(L, T)
    total = np.zeros((numberOfLevels, numberOfPoints))
    count = np.zeros((numberOfLevels, numberOfPoints))
    for l in range(L):
        for corner in range(3):
            for k in (l, l + 1):
                np.add.at(total[k], triangles[:, corner], beta[l])
                np.add.at(count[k], triangles[:, corner], 1.0)
    return (total / np.maximum(count, 1.0)).ravel()


def medium_from_reference(gainMedium):
    """The reference's GainMedium as this package's PrismMesh (MeshTopology)
    or TetMesh (VolumeTopology)."""
    topology = gainMedium.topology
    p = {name: _property(gainMedium, name) for name in _PROPERTIES}
    if p["betaVolume"] is None or p["nTot"] is None or p["crystalTFluo"] is None:
        raise ValueError("the gain medium needs betaVolume, nTot and crystalTFluo")
    common = dict(nTot=float(p["nTot"]), crystalTFluo=float(p["crystalTFluo"]),
                  claddingNumber=int(p["claddingNumber"] if p["claddingNumber"] is not None else 1),
                  claddingAbsorption=float(p["claddingAbsorption"] or 0.0))
    clad = p["claddingCellTypes"]
    if hasattr(topology, "trianglePointIndices"):  # MeshTopology: an extruded prism mesh
        if topology.levels is None or topology.thickness is None:
            raise ValueError("the gain medium's MeshTopology needs levels and thickness")
        points = np.asarray(topology.points, np.float64)
        triangles = np.asarray(topology.trianglePointIndices, np.uint32)
        levels = int(topology.levels)
        beta = np.asarray(p["betaVolume"], np.float64).ravel()
        return PrismMesh(points=points, triangles=triangles, numberOfLevels=levels,
                         thickness=float(topology.thickness), betaVolume=beta,
                         betaCells=point_beta(triangles, points.shape[0], levels, beta),
                         claddingCellTypes=None if clad is None else np.asarray(clad, np.uint32).ravel(), **common)
    if hasattr(topology, "cellPointIndices"):  # VolumeTopology: Tet4 cells
        optics = {}
        faces = getattr(topology, "faceBoundaries", None)
        if faces is not None and np.any(np.asarray(faces) > 0) and getattr(gainMedium, "_surfaceOptics", None):
            reflectivity, inside, outside = gainMedium._surfaceOpticsArrays()
            optics = dict(cellFaceBoundaries=np.asarray(faces, np.int32), surfaceReflectivities=reflectivity,
                          surfaceRefractiveIndexInside=inside, surfaceRefractiveIndexOutside=outside)
        return TetMesh(points=np.asarray(topology.points, np.float64),
                       cells=np.asarray(topology.cellPointIndices, np.uint32),
                       betaVolume=np.asarray(p["betaVolume"], np.float64).ravel(),
                       claddingCellTypes=None if clad is None else np.asarray(clad, np.uint32).ravel(),
                       **common, **optics)
    raise TypeError("the gain medium's topology is neither a MeshTopology nor a VolumeTopology")


def spectra_from_reference(crossSections) -> CrossSectionData:
    """The reference's SpectralDecomposition (same attribute names)."""
    return CrossSectionData(crossSections.wavelengthsAbsorption, crossSections.crossSectionAbsorption,
                            crossSections.wavelengthsEmission, crossSections.crossSectionEmission,
                            int(getattr(crossSections, "resolution", 1) or 1))


def solver_from_reference(phiAse) -> _PhiASE:
    """This package's PhiASE configured from the reference's PhiASE fields."""
    settings = {name: getattr(phiAse, name) for name in SOLVER_FIELDS if getattr(phiAse, name, None) is not None}
    return _PhiASE(config=settings)


def runPhiASE(phiAse, gainMedium, crossSections, *, transport=None, command_prefix=None, workspace_dir=None,
              watchdog_interval=None, openpmdSession=None) -> Result:
    """The reference's ``transport.runPhiASE``, solved by libhase_b200.  The
    transport options are accepted for the call's signature and unused."""
    del transport, command_prefix, workspace_dir, watchdog_interval, openpmdSession
    solver = solver_from_reference(phiAse)
    return solver.run(gainMedium=medium_from_reference(gainMedium),
                      crossSections=spectra_from_reference(crossSections)).getResults()


# The reference's name of a CUDA GPU backend (AlpakaBackends, as its tests select it).
BACKEND = "Nvidia_Gpu_CudaRt"


def backends() -> list[str]:
    """``AlpakaBackends.all()`` of the reference's launcher: this library's GPU backend."""
    return [BACKEND]


def ensure_backend_available(backend=None, executable=None):
    """``transport._ensure_backend_available``: no openPMD series is written, so every
    transport selection is accepted."""
    del executable
    return backend


def patch_targets(simulation_module):
    """The (object, attribute, replacement) triples that route the reference's
    ``PhiASE.run`` (module ``pyInclude.simulation``) to this library: the
    backend query and the transport check of its launcher
    (pyInclude/simulation.py:61-107) and ``transport.runPhiASE``."""
    return [(simulation_module.AlpakaBackends, "all", staticmethod(backends)),
            (simulation_module.transport, "_ensure_backend_available", ensure_backend_available),
            (simulation_module.transport, "runPhiASE", runPhiASE)]


def install(simulation_module) -> None:
    """Route the reference's Python call surface to libhase_b200 for the rest
    of the process: ``install(pyInclude.simulation)``."""
    for obj, name, value in patch_targets(simulation_module):
        setattr(obj, name, value)
