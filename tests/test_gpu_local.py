"""The local proposal (hase_context_set_local_proposal): per sample point its
K nearest triangles x layers x slices weighted (importance walks or the
learned network), a fixed share of the rays drawn from a beta V / d^2 prior
over the whole medium, each ray weighted by the mixture's probability.

- Unbiased: per-sample estimates agree with the full importance-sampled
  solve within the combined Monte Carlo error (polychromatic, reflections).
- Known answer: the analytic flux of a uniform medium.
- All triangles as candidates (no far rays) and a very small candidate set
  (most of the flux from far rays) both stay unbiased.
- The candidate rows: weights of the candidates equal the full solve's
  weights of the same (slice, prism) entries.
- The learned proposal on candidate entries is unbiased too.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import analytic_phi

pytestmark = pytest.mark.gpu


def _z(a, b):
    sig = np.hypot(a.relativeStandardError * a.phiAse, b.relativeStandardError * b.phiAse)
    return (a.phiAse.astype(np.float64) - b.phiAse) / sig


@pytest.fixture(scope="module")
def poly():
    from haseongpu_b200 import DeviceMesh, build
    from haseongpu_b200.configs import disc_poly

    build.build_library()
    w = disc_poly()
    sa, se = w.spectra.resampled()
    ctx = DeviceMesh(w.mesh, sa, se, device=0)
    yield w, ctx
    ctx.close()


@pytest.mark.parametrize("K", [64, 12])
def test_local_proposal_is_unbiased(poly, K):
    w, ctx = poly
    kw = dict(minRays=400_000, useReflections=True, minSample=3000, maxSample=3063)
    full = ctx.calc_phi_ase(rngSeed=3, **kw)
    ctx.set_local_proposal(K)
    try:
        local = ctx.calc_phi_ase(rngSeed=4, **kw)
    finally:
        ctx.set_local_proposal(0)
    assert local.droppedRays.sum() == 0 and local.totalRays[0] == 400_000
    z = _z(local, full)
    assert np.max(np.abs(z)) < 4.5, np.max(np.abs(z))
    assert abs(z.mean()) < 4.0 / np.sqrt(z.size), z.mean()
    # the same medium-wide flux
    assert abs(local.phiAse.astype(np.float64).sum() / full.phiAse.sum() - 1.0) < 3e-3


def test_local_candidates_carry_the_full_weights(poly):
    """A candidate entry (j, l, k) has the full solve's weight of (slice j,
    prism cand[k] + l T), up to the common normalisation (both rows are
    divided by their maxima, and the nearest prisms hold the maximum)."""
    w, ctx = poly
    mesh = w.mesh
    s = 2222
    full = ctx.importance_weights(s, 1, True)[0]
    ctx.set_local_proposal(32)
    try:
        local = ctx.importance_weights(s, 1, True)[0]
    finally:
        ctx.set_local_proposal(0)
    T, L, P = mesh.numberOfTriangles, mesh.numberOfLevels - 1, mesh.numberOfPrisms
    pt = s % mesh.numberOfPoints
    # the library's candidate order: FP32 centroids and points, FP64 squared distances, ties by index
    v = mesh.points[mesh.triangles]
    cen = ((v[:, 0] + v[:, 1] + v[:, 2]) / 3.0).astype(np.float32).astype(np.float64)
    d = cen - mesh.points[pt].astype(np.float32).astype(np.float64)
    d2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]
    cand = np.lexsort((np.arange(T), d2))[:32]
    j, l, k = np.meshgrid(np.arange(5), np.arange(L), np.arange(32), indexing="ij")
    expect = full[j * P + l * T + cand[k]].ravel()
    got = local.reshape(-1)
    scale = got.max() / expect.max()
    np.testing.assert_allclose(got, expect * scale, rtol=1e-5, atol=1e-7 * got.max())


@pytest.mark.parametrize("K", [1014, 24])
def test_local_proposal_analytic_uniform_medium(K):
    from haseongpu_b200 import DeviceMesh
    from haseongpu_b200.configs import disc_small

    base = disc_small().mesh
    beta, nTot, tau, sa, se = 0.2, 1.38e20, 9.41e-4, 1.1e-21, 2.2e-20
    mesh = base.withBeta(np.full(base.numberOfPrisms, beta))
    g = nTot * (beta * (se + sa) - sa)
    Np = mesh.numberOfPoints
    rr = np.linalg.norm(mesh.points, axis=1)
    samples = [5 * Np, int(np.argmax(rr)) + 4 * Np, int(np.argsort(rr)[40]) + 9 * Np]
    with DeviceMesh(mesh, [sa], [se]) as ctx:
        ctx.set_local_proposal(K)
        for s in samples:
            r = ctx.calc_phi_ase(minRays=4_000_000, minSample=s, maxSample=s, rngSeed=99)
            expect = analytic_phi(mesh, mesh.samplePoints()[s], beta, g, nTot, tau, 1024, 1024)
            rel = r.phiAse[0] / expect - 1.0
            assert abs(rel) < max(4 * r.relativeStandardError[0], 3e-4), (K, s, rel, r.relativeStandardError[0])
            assert r.droppedRays[0] == 0


def test_local_learned_proposal_is_unbiased(poly):
    from haseongpu_b200.proposal import ProposalNet

    w, ctx = poly
    kw = dict(minRays=400_000, useReflections=True, minSample=5100, maxSample=5131)
    full = ctx.calc_phi_ase(rngSeed=7, **kw)
    ctx.set_local_proposal(48)
    try:
        with ProposalNet(seed=11) as net:  # untrained: the estimator must stay unbiased regardless
            learned = ctx.calc_phi_ase_learned(net, rngSeed=8, **kw)
            W = ctx.learned_weights(net, 5100, 2, True)
    finally:
        ctx.set_local_proposal(0)
    assert W.shape == (2, 5 * (w.mesh.numberOfLevels - 1) * 48)
    z = _z(learned, full)
    assert np.max(np.abs(z)) < 4.5 and abs(z.mean()) < 4.0 / np.sqrt(z.size), (np.max(np.abs(z)), z.mean())


def test_local_proposal_logs_candidate_contributions(poly):
    """Logged contributions: every ray (near or far) whose prism is one of the
    point's candidates adds to its entry, so the row's sum over the rays is
    the candidates' part of the estimate, between 0 and phi."""
    w, ctx = poly
    ctx.set_local_proposal(64)
    try:
        res, contrib = ctx.log_contributions(minRays=200_000, useReflections=True, minSample=4000, maxSample=4003,
                                             rngSeed=5)
    finally:
        ctx.set_local_proposal(0)
    assert contrib.shape == (4, 5 * (w.mesh.numberOfLevels - 1) * 64)
    near = contrib.astype(np.float64).sum(axis=1) / res.totalRays
    assert np.all(near > 0) and np.all(near < res.phiAse)


def test_local_mode_is_rejected_by_batches(poly):
    from haseongpu_b200 import MediaBatch, _native as N

    _, ctx = poly
    ctx.set_local_proposal(16)
    try:
        with MediaBatch(0) as b, pytest.raises(N.HaseError):
            b.solve([(ctx, 0, 3)], minRays=100)
    finally:
        ctx.set_local_proposal(0)


def test_warm_started_series_runs_and_matches_the_plain_series():
    """The warm-started learned series (learned.warm_started_series) on a
    small pump series with the local proposal: every step fine-tunes the
    network and solves all samples with it; beta follows the plain local
    series within the Monte Carlo noise of phi-ASE, and the pump-only part
    (mean beta after the first step, before any phi-ASE) is identical."""
    from haseongpu_b200 import DeviceMesh
    from haseongpu_b200.configs import disc_small
    from haseongpu_b200.learned import warm_started_series
    from haseongpu_b200.proposal import ProposalNet

    w = disc_small()
    sa, se = w.spectra.resampled(True)
    mesh = w.mesh.withBeta(np.zeros(w.mesh.numberOfPrisms))
    pump = dict(peakIntensity=16e3, radius=0.6, exponent=40.0, wavelength=940e-9, sigmaA=0.8e-20, sigmaE=0.16e-20)
    tm = dict(timeStep=50e-6, steps=4)
    with DeviceMesh(mesh, sa, se) as ctx:
        ctx.set_local_proposal(12)
        plain = ctx.simulate(pump=pump, time=tm, minRays=4000, rngSeed=3)
    with DeviceMesh(mesh, sa, se) as ctx, ProposalNet(seed=2) as net:
        ctx.set_local_proposal(12)
        ws = warm_started_series(ctx, net, pump, tm, rays=4000, useReflections=False, monochromatic=True,
                                 log_samples=16, log_rays=4000, train_steps=5, rngSeed=3)
    assert len(ws["meanBeta"]) == 5 and len(ws["loss"]) == 3 and ws["raysTraced"] > 0
    assert np.all(np.isfinite(ws["loss"]))
    assert ws["meanBeta"][1] == pytest.approx(plain["meanBeta"][1], rel=1e-9)
    np.testing.assert_allclose(ws["meanBeta"], plain["meanBeta"], rtol=2e-3)
