"""The surface-reservoir reflection passes of the forward method in the oracle
(include/core/forwardSrm.hpp:100-365, include/kernels/forward/accumulation.hpp:455-833,
include/kernels/reflection.hpp:21-47).

- A reflecting surface of reflectivity 0 deposits nothing: the chain ends as
  converged without a pass and phi equals the solve without reflections.
- Known answer: in a transparent medium (g = 0) every reflected ray reaches
  another reflecting face with its weight unchanged, so the reflected weight
  falls by exactly R per pass; the chain ends as converged at the first pass
  p with R^p < tolerance, with remaining fraction R^p.
- Below the lasing threshold the chain converges and adds to phi; above it
  (round-trip gain x R > 1) it ends as diverged; a pass limit ends it as
  max_iterations.
- Total internal reflection alone (reflectivity 0, n_in > n_out) reflects.
- The Tet4 twin of a prism mesh carries the prism's top/bottom reflectivities.
"""

from __future__ import annotations

import numpy as np
import pytest

from haseongpu_b200.tetmesh import TetMesh, beta_from_gain

NTOT, TAU, SA, SE = 1e20, 1e-3, 1e-21, 2e-20
SPEC = (np.array([SA]), np.array([SE]))
KW = dict(minRays=8000, seed=3, batches=8, threads=1)


def _ball(gain, divisions=4):
    return TetMesh.ball(1.0, divisions, beta_from_gain(gain, NTOT, SA, SE), NTOT, TAU)


def test_zero_reflectivity_changes_nothing(oracle):
    ball = _ball(0.5)
    plain = oracle.forward_phi_ase(ball, SPEC, **KW)
    r = oracle.forward_phi_ase(ball.withReflectingBoundary(0.0), SPEC, useReflections=True, **KW)
    assert plain["srmStatus"] == "disabled"
    assert r["srmStatus"] == "converged" and r["srmPasses"] == 0
    np.testing.assert_array_equal(r["phiAse"], plain["phiAse"])
    np.testing.assert_array_equal(r["rayVisits"], plain["rayVisits"])


@pytest.mark.parametrize("R,passes", [(0.5, 14), (0.3, 8), (0.9, 88)])
def test_transparent_medium_loses_exactly_r_per_pass(oracle, R, passes):
    ball = _ball(0.0)
    r = oracle.forward_phi_ase(ball.withReflectingBoundary(R), SPEC, useReflections=True, reflectionMaxIterations=100,
                               **KW)
    assert r["srmStatus"] == "converged"
    assert r["srmPasses"] == passes
    np.testing.assert_allclose(r["srmRemainingFraction"], R ** passes, rtol=1e-9)


def test_reflections_below_threshold_converge_and_add_flux(oracle):
    ball = _ball(0.3)
    plain = oracle.forward_phi_ase(ball, SPEC, **KW)
    r = oracle.forward_phi_ase(ball.withReflectingBoundary(0.3), SPEC, useReflections=True, **KW)
    assert r["srmStatus"] == "converged" and 1 <= r["srmPasses"] < 40
    assert r["srmRemainingFraction"] < 1e-4
    ratio = r["phiAse"] / plain["phiAse"]
    assert np.all(ratio > 1.0) and 1.5 < ratio.mean() < 4.0
    # reflected rays tally too: more visits than the source rays alone
    assert r["rayVisits"].sum() > plain["rayVisits"].sum()


def test_lasing_diverges_and_pass_limit_stops(oracle):
    ball = _ball(1.0)
    r = oracle.forward_phi_ase(ball.withReflectingBoundary(0.9), SPEC, useReflections=True, **KW)
    assert r["srmStatus"] == "diverged" and r["srmPasses"] == 3 and r["srmRemainingFraction"] > 1.0
    r = oracle.forward_phi_ase(_ball(0.3).withReflectingBoundary(0.3), SPEC, useReflections=True,
                               reflectionMaxIterations=2, **KW)
    assert r["srmStatus"] == "max_iterations" and r["srmPasses"] == 2


def test_total_internal_reflection_alone_reflects(oracle):
    ball = _ball(0.3)
    plain = oracle.forward_phi_ase(ball, SPEC, **KW)
    r = oracle.forward_phi_ase(ball.withReflectingBoundary(0.0, nInside=1.8, nOutside=1.0), SPEC,
                               useReflections=True, **KW)
    assert r["srmPasses"] >= 1
    assert (r["phiAse"] / plain["phiAse"]).mean() > 1.2


def test_tet4_twin_carries_prism_reflectivities():
    from haseongpu_b200.configs import disc_poly

    prism = disc_poly().mesh
    tet = TetMesh.fromPrismMesh(prism)
    T = prism.numberOfTriangles
    ids = tet.cellFaceBoundaries
    assert ids is not None and (ids > 0).sum() == 2 * T
    bnd = tet.boundaryFaces()
    assert np.all(bnd[ids > 0])  # only boundary faces carry a surface
    z = tet.points[:, 2]
    for c, f in zip(*np.nonzero(ids > 0)):
        face = np.delete(tet.cells[c], f)
        sid = ids[c, f]
        top = sid % 2 == 0
        assert np.allclose(z[face], z.max() if top else 0.0)
        t = (sid - 1) // 2
        assert tet.surfaceReflectivities[sid] == prism.reflectivities[t, 1 if top else 0]
        n = prism.refractiveIndices
        assert tet.surfaceRefractiveIndexInside[sid] == (n[2] if top else n[0])
        assert tet.surfaceRefractiveIndexOutside[sid] == (n[3] if top else n[1])
