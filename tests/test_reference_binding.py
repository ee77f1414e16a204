"""The reference's Python call surface routed to libhase_b200
(haseongpu_b200.reference_binding).

* CPU: with the reference's Python front end importable from the directory
  named by the environment variable HASEONGPU_REFERENCE (a HASEonGPU source
  tree; skipped when unset), its own ``PhiASE.run(...).getResults()`` -- the
  call its tests mock at ``transport.runPhiASE``
  (tests/python/phiAse/test_simulationWrapper.py:51-86) -- goes through the
  binding into the library: its GainMedium (MeshTopology or Tet4
  VolumeTopology) and SpectralDecomposition arrive unchanged, and without a
  GPU the library's own context creation answers HASE_NO_DEVICE.
* GPU: the same binding on stand-ins with the reference's attribute names
  returns the result of a direct solve of the same medium, bit for bit.
"""

from __future__ import annotations

import importlib
import os
import sys
from types import SimpleNamespace

import numpy as np
import pytest

REFERENCE = os.environ.get("HASEONGPU_REFERENCE")


def _reference():
    if not REFERENCE:
        pytest.skip("HASEONGPU_REFERENCE (a HASEonGPU source tree) is not set")
    if REFERENCE not in sys.path:
        sys.path.insert(0, REFERENCE)
    try:
        return importlib.import_module("pyInclude"), importlib.import_module("pyInclude.simulation")
    except Exception as exc:  # the reference's front end or its dependencies missing
        pytest.skip(f"the reference's Python front end does not import: {exc}")


def _gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def _prism_medium(ref):
    topo = ref.MeshTopology.fromGrid(ref.Grid(xExtent=1, yExtent=1, zExtent=0.5, tileSizeX=0.25, tileSizeY=0.25,
                                              tileSizeZ=0.1))
    T, L = topo.numberOfTriangles, topo.levels - 1
    beta = np.random.default_rng(4).uniform(0.05, 0.3, (T, L))
    return ref.GainMedium(topology=topo).withPhysicalProperties(
        betaVolume=beta, claddingCellTypes=np.zeros(T, np.uint32), nTot=2.76e20, crystalTFluo=9.5e-4,
        claddingNumber=1, claddingAbsorption=0.0), beta


def test_reference_phiase_run_reaches_the_library(monkeypatch):
    ref, simulation = _reference()
    from haseongpu_b200 import PrismMesh, _native
    from haseongpu_b200 import reference_binding as rb

    medium, beta = _prism_medium(ref)
    spectra = ref.SpectralDecomposition.monochromatic(wavelength=940e-9, crossSectionAbsorption=0.01e-20,
                                                      crossSectionEmission=0.02e-20)
    seen = {}

    def spy(phiAse, gainMedium, crossSections, **kw):
        seen.update(phiAse=phiAse, medium=rb.medium_from_reference(gainMedium),
                    spectra=rb.spectra_from_reference(crossSections), kw=kw)
        return rb.runPhiASE(phiAse, gainMedium, crossSections, **kw)

    for obj, name, value in rb.patch_targets(simulation):
        monkeypatch.setattr(obj, name, value)
    monkeypatch.setattr(simulation.transport, "runPhiASE", spy)
    phi = ref.PhiASE(propagationMode="backward", minRays=2000, maxRays=2000, monochromatic=True, rngSeed=7,
                     relativeStandardErrorThreshold=0.1, adaptiveSteps=1, useReflections=False)
    if _gpu():
        res = phi.run(gainMedium=medium, crossSections=spectra).getResults()
        assert res.phiAse.shape == (medium.topology.numberOfPoints * medium.topology.levels,)
        assert np.all(res.totalRays == 2000) and np.all(res.phiAse > 0)
    else:
        with pytest.raises(_native.HaseError) as err:
            phi.run(gainMedium=medium, crossSections=spectra)
        assert err.value.status == _native.HASE_NO_DEVICE  # hase_context_create ran and found no GPU
    # the reference's objects arrived unchanged
    m = seen["medium"]
    assert isinstance(m, PrismMesh) and seen["phiAse"] is phi
    np.testing.assert_array_equal(m.points, medium.topology.points)
    np.testing.assert_array_equal(m.triangles, medium.topology.trianglePointIndices)
    assert m.numberOfLevels == medium.topology.levels and m.thickness == medium.topology.thickness
    np.testing.assert_array_equal(m.betaVolume, beta.ravel(order="F"))  # prism t + l T
    assert m.nTot == 2.76e20 and m.crystalTFluo == 9.5e-4 and m.claddingNumber == 1
    np.testing.assert_array_equal(seen["spectra"].crossSectionAbsorption, [0.01e-20])
    np.testing.assert_array_equal(seen["spectra"].crossSectionEmission, [0.02e-20])
    solver = rb.solver_from_reference(phi)
    assert (solver.propagationMode, solver.minRays, solver.rngSeed, solver.monochromatic) == ("backward", 2000, 7,
                                                                                              True)


def test_reference_tet4_medium_reaches_the_forward_method(monkeypatch):
    ref, simulation = _reference()
    from haseongpu_b200 import TetMesh, _native
    from haseongpu_b200 import reference_binding as rb

    medium, _ = _prism_medium(ref)
    prism = rb.medium_from_reference(medium)
    tet = TetMesh.fromPrismMesh(prism)
    vol = importlib.import_module("pyInclude.geometry.volume")
    topo = vol.VolumeTopology.fromTetrahedra(tet.points, tet.cells.astype(np.int64))
    gm = ref.GainMedium(topology=topo).withPhysicalProperties(
        betaVolume=tet.betaVolume, nTot=2.76e20, crystalTFluo=9.5e-4, claddingNumber=1, claddingAbsorption=0.0)
    converted = rb.medium_from_reference(gm)
    assert isinstance(converted, TetMesh)
    np.testing.assert_array_equal(converted.cells, tet.cells)
    np.testing.assert_array_equal(converted.betaVolume, tet.betaVolume)
    for obj, name, value in rb.patch_targets(simulation):
        monkeypatch.setattr(obj, name, value)
    spectra = ref.SpectralDecomposition.monochromatic(wavelength=940e-9, crossSectionAbsorption=0.01e-20,
                                                      crossSectionEmission=0.02e-20)
    phi = ref.PhiASE(minRays=20000, maxRays=20000, monochromatic=True, rngSeed=3, adaptiveSteps=1)  # forward mode
    if _gpu():
        res = phi.run(gainMedium=gm, crossSections=spectra).getResults()
        assert res.phiAse.shape == (tet.numberOfCells,) and np.all(np.isfinite(res.phiAse))
    else:
        with pytest.raises(_native.HaseError) as err:
            phi.run(gainMedium=gm, crossSections=spectra)
        assert err.value.status == _native.HASE_NO_DEVICE


class _Property:
    def __init__(self, value):
        self.value = value


class _StandInMedium:
    """An object with the reference GainMedium's attribute names (topology,
    get(name).value), as the binding reads it."""

    def __init__(self, topology, **physical):
        self.topology = topology
        self.physical = physical

    def get(self, name):
        if name not in self.physical:
            raise KeyError(name)
        return _Property(self.physical[name])


@pytest.mark.gpu
def test_binding_equals_a_direct_solve():
    from haseongpu_b200 import DeviceMesh
    from haseongpu_b200 import reference_binding as rb
    from haseongpu_b200.configs import disc_small

    w = disc_small()
    mesh = w.mesh
    topo = SimpleNamespace(points=mesh.points, trianglePointIndices=mesh.triangles, levels=mesh.numberOfLevels,
                           thickness=mesh.thickness)
    medium = _StandInMedium(topo, betaVolume=mesh.betaVolume, nTot=mesh.nTot, crystalTFluo=mesh.crystalTFluo,
                            claddingNumber=1, claddingAbsorption=0.0)
    sa, se = w.spectra.resampled(True)
    spectra = SimpleNamespace(wavelengthsAbsorption=[1030e-9], crossSectionAbsorption=sa[:1],
                              wavelengthsEmission=[1030e-9], crossSectionEmission=se[:1], resolution=1)
    phi = SimpleNamespace(propagationMode="backward", minRays=20000, maxRays=20000, relativeStandardErrorThreshold=0.0,
                          adaptiveSteps=1, useReflections=False, monochromatic=True, rngSeed=11, minSampleRange=100,
                          maxSampleRange=227)
    res = rb.runPhiASE(phi, medium, spectra, transport="adios2", workspace_dir="unused")
    converted = rb.medium_from_reference(medium)
    with DeviceMesh(converted, sa[:1], se[:1]) as ctx:
        ref = ctx.calc_phi_ase(minRays=20000, maxRays=20000, adaptiveSteps=1, monochromatic=True, rngSeed=11,
                               minSample=100, maxSample=227)
    np.testing.assert_array_equal(res.phiAse, ref.phiAse)
    np.testing.assert_array_equal(res.relativeStandardError, ref.relativeStandardError)
    np.testing.assert_array_equal(res.totalRays, ref.totalRays)
    np.testing.assert_allclose(res.standardError, ref.relativeStandardError * ref.phiAse, rtol=1e-6)
    np.testing.assert_array_equal(res.dndtAse, ref.dndtAse)
