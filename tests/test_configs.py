"""The seeded workload generators match the configurations they stand for."""

from __future__ import annotations

import numpy as np
import pytest


def test_media64_follows_config_3():
    from haseongpu_b200.configs import media64

    w = media64()
    assert len(w.media) == 64 and (w.minRays, w.maxRays, w.threshold) == (10_000, 10_000_000, 0.001)
    T = np.array([m.mesh.numberOfTriangles for m in w.media])
    L = np.array([m.mesh.numberOfLevels for m in w.media])
    R = np.array([np.sqrt((m.mesh.points ** 2).sum(1)).max() for m in w.media])
    H = np.array([m.mesh.thickness * (m.mesh.numberOfLevels - 1) for m in w.media])
    nl = np.array([m.wavelengths for m in w.media])
    assert 150 <= T.min() and T.max() <= 22_000 and np.median(T) < 5_000   # log-uniform 200 .. 20,000
    assert L.min() >= 5 and L.max() <= 40
    assert R.min() >= 0.5 - 1e-9 and R.max() <= 3.0 + 1e-9
    assert H.min() >= 0.3 - 1e-9 and H.max() <= 2.0 + 1e-9
    assert nl.min() >= 1 and nl.max() <= 8 and len(set(nl)) > 4
    for m in w.media[:8]:
        assert m.spectra.resampled(False)[0].size == m.wavelengths
        assert np.all(m.mesh.betaVolume > 0) and m.mesh.betaVolume.max() < 1
    # deterministic
    again = media64()
    assert all(np.array_equal(a.mesh.betaVolume, b.mesh.betaVolume) for a, b in zip(w.media, again.media))


def test_media_training_is_disjoint_and_small():
    from haseongpu_b200.configs import media64, media_training

    tr = media_training()
    assert len(tr) == 24 and max(m.mesh.numberOfTriangles for m in tr) <= 3000
    ev = {m.mesh.numberOfPrisms for m in media64().media}
    assert sum(m.mesh.numberOfPrisms in ev for m in tr) < 4  # other seed: no copies of the evaluation media


def test_pulse_follows_config_5():
    from haseongpu_b200.configs import pulse
    from haseongpu_b200.tetmesh import TetMesh

    w = pulse()
    m = w.mesh
    assert 18_000 <= m.numberOfTriangles <= 22_000 and m.numberOfLevels == 30
    assert w.spectra.resampled(False)[0].size == 8
    assert np.allclose(m.reflectivities, [0.3, 0.9])
    assert np.all(m.betaVolume == 0)
    t = w.time
    assert t["steps"] == 50 and t["pumpSteps"] == 50 and abs(t["timeStep"] * t["steps"] - 1e-3) < 1e-12
    tet = TetMesh.fromPrismMesh(m)
    assert tet.numberOfCells == 3 * m.numberOfPrisms
    assert (tet.cellFaceBoundaries > 0).sum() == 2 * m.numberOfTriangles


def test_tet_surface_fields_validate():
    from haseongpu_b200.tetmesh import TetMesh

    pts = np.array([(0.0, 0, 0), (1.0, 0, 0), (0.0, 1, 0), (0.0, 0, 1)])
    with pytest.raises(ValueError):
        TetMesh(pts, np.array([(0, 1, 2, 3)]), [0.1], 1e20, 1e-3, cellFaceBoundaries=np.zeros((2, 4)))
    with pytest.raises(ValueError):
        TetMesh(pts, np.array([(0, 1, 2, 3)]), [0.1], 1e20, 1e-3, reflectivities=np.zeros((3, 2)))
    m = TetMesh(pts, np.array([(0, 1, 2, 3)]), [0.1], 1e20, 1e-3).withReflectingBoundary(0.4, 1.5, 1.0)
    assert m.boundaryFaces().all() and np.all(m.cellFaceBoundaries == 1)
    assert m.numberOfSurfaces == 2 and m.surfaceReflectivities[1] == 0.4
    refl, nin, nout = m.surfaceArrays()
    assert nin[1] == 1.5 and nout[1] == 1.0
