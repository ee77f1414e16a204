"""GPU parity of the forward method's surface-reservoir reflections
(include/hase_b200_forward.h, useReflections) against the oracle
(oracle/hase_oracle_forward.cpp) and known answers.

The device and the oracle draw the same Philox streams, so the source pass
deposits the same rays at the same faces.  The device sorts each face's
slots by ray index (the oracle applies deposits in ray order), so below the
slot limit both reservoirs hold the same records in the same order and the
reflected passes walk the same rays: the whole chain replays to rounding
(per-cell phi as float, pass counts and status exactly).
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NTOT, TAU, SA, SE = 1e20, 1e-3, 1e-21, 2e-20


def _ball(gain, divisions=4):
    from haseongpu_b200.tetmesh import TetMesh, beta_from_gain

    return TetMesh.ball(1.0, divisions, beta_from_gain(gain, NTOT, SA, SE), NTOT, TAU)


def _ctx(mesh):
    from haseongpu_b200 import TetDeviceMesh, build

    build.build_library()
    return TetDeviceMesh(mesh, [SA], [SE], device=0)


def test_zero_reflectivity_equals_the_plain_solve():
    mesh = _ball(0.5).withReflectingBoundary(0.0)
    with _ctx(mesh) as ctx:
        plain = ctx.calc_phi_ase(forwardRayCount=200_000, rngSeed=4)
        r = ctx.calc_phi_ase(forwardRayCount=200_000, rngSeed=4, useReflections=True)
    assert plain.srmStatus == "disabled" and r.srmStatus == "converged" and r.srmPasses == 0
    assert r.reflectingFaces == int(mesh.boundaryFaces().sum())
    np.testing.assert_allclose(r.phiAse, plain.phiAse, rtol=1e-6)
    np.testing.assert_array_equal(r.totalRays, plain.totalRays)


@pytest.mark.parametrize("R,passes", [(0.5, 14), (0.3, 8)])
def test_transparent_medium_loses_exactly_r_per_pass(R, passes):
    with _ctx(_ball(0.0).withReflectingBoundary(R)) as ctx:
        r = ctx.calc_phi_ase(forwardRayCount=100_000, rngSeed=2, useReflections=True, reflectionMaxIterations=100)
    assert r.srmStatus == "converged" and r.srmPasses == passes
    np.testing.assert_allclose(r.srmRemainingFraction, R ** passes, rtol=1e-9)


@pytest.mark.parametrize("gain,R,status", [(0.3, 0.3, "converged"), (1.0, 0.9, "diverged")])
def test_chain_replays_the_oracle(oracle, gain, R, status):
    mesh = _ball(gain).withReflectingBoundary(R)
    kw = dict(minRays=40_000, seed=9)
    ref = oracle.forward_phi_ase(mesh, ([SA], [SE]), useReflections=True, surfaceReservoirSize=256, **kw)
    with _ctx(mesh) as ctx:
        dev = ctx.calc_phi_ase(forwardRayCount=40_000, rngSeed=9, useReflections=True, surfaceReservoirSize=256)
    assert dev.srmStatus == ref["srmStatus"] == status
    assert dev.srmPasses == ref["srmPasses"]
    np.testing.assert_allclose(dev.srmRemainingFraction, ref["srmRemainingFraction"], rtol=1e-9)
    np.testing.assert_array_equal(dev.totalRays, ref["rayVisits"])
    np.testing.assert_allclose(dev.phiAse, ref["phiAse"], rtol=1e-5)
    np.testing.assert_allclose(dev.relativeStandardError, ref["relativeStandardError"], rtol=1e-4)


def test_reflections_add_flux_and_full_reservoirs_stay_unbiased(oracle):
    mesh = _ball(0.3).withReflectingBoundary(0.3)
    with _ctx(mesh) as ctx:
        plain = ctx.calc_phi_ase(forwardRayCount=400_000, rngSeed=1)
        big = ctx.calc_phi_ase(forwardRayCount=400_000, rngSeed=1, useReflections=True, surfaceReservoirSize=512)
        small = ctx.calc_phi_ase(forwardRayCount=400_000, rngSeed=7, useReflections=True, surfaceReservoirSize=4)
    ratio = big.phiAse / plain.phiAse
    assert np.all(ratio > 1.0) and 1.5 < ratio.mean() < 4.0
    assert big.srmStatus == small.srmStatus == "converged"
    # 4 slots per face overflow and replace; the medium-wide flux stays within a few percent
    vol = mesh.cellVolumes()
    assert (small.phiAse * vol).sum() == pytest.approx((big.phiAse * vol).sum(), rel=0.05)


def test_total_internal_reflection_and_pass_limit():
    mesh = _ball(0.3)
    with _ctx(mesh.withReflectingBoundary(0.0, nInside=1.8, nOutside=1.0)) as ctx:
        plain = ctx.calc_phi_ase(forwardRayCount=100_000, rngSeed=3)
        tir = ctx.calc_phi_ase(forwardRayCount=100_000, rngSeed=3, useReflections=True)
        capped = ctx.calc_phi_ase(forwardRayCount=100_000, rngSeed=3, useReflections=True, reflectionMaxIterations=2)
    assert tir.srmPasses >= 1 and (tir.phiAse / plain.phiAse).mean() > 1.2
    assert capped.srmStatus == "max_iterations" and capped.srmPasses == 2 and capped.srmMaxIterations == 2


def test_phiase_forward_with_prism_reflectivities():
    from haseongpu_b200 import PhiASE
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    kw = dict(propagationMode="forward", forwardRayCount=400_000, monochromatic=True, rngSeed=5)
    plain = PhiASE(**kw).run(w.mesh, w.spectra).getResults()
    refl = PhiASE(useReflections=True, **kw).run(w.mesh, w.spectra).getResults()
    assert plain.srmStatus == "disabled" and refl.srmStatus in ("converged", "stable")
    assert refl.reflectingFaces == 2 * w.mesh.numberOfTriangles
    assert refl.phiAse.sum() > plain.phiAse.sum()


def test_reflections_on_a_mesh_without_reflecting_surfaces():
    mesh = _ball(0.3)
    with _ctx(mesh) as ctx:
        plain = ctx.calc_phi_ase(forwardRayCount=100_000, rngSeed=6)
        r = ctx.calc_phi_ase(forwardRayCount=100_000, rngSeed=6, useReflections=True)
    assert r.reflectingFaces == 0 and r.srmStatus == "converged" and r.srmPasses == 0
    np.testing.assert_array_equal(r.phiAse, plain.phiAse)
