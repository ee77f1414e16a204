"""The learned proposal inside the phi-ASE solve (include/hase_b200_proposal.h).

- Features of (sample, slice, prism) pairs match their definition (CPU).
- The logged contributions sum to the estimate: sum_jp c_jp / N = phi.
- The estimator stays unbiased under any proposal network (untrained and
  trained against the importance weights, within the combined errors).
- A network trained on 32 seeded pump fields lowers the per-ray variance on
  unseen fields: against the importance weights with near-field start points,
  and by more than an order of magnitude against the reference's plain
  importance sampling with uniform start points.
- Fallback: a sample whose per-ray variance exceeds the limit restarts with
  the importance weights.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from haseongpu_b200 import DeviceMesh, build
    from haseongpu_b200.configs import disc_small

    build.build_library()
    w = disc_small()
    sa, se = w.spectra.resampled(True)
    ctx = DeviceMesh(w.mesh, sa, se, device=0)
    yield w.mesh, sa, se, ctx
    ctx.close()


@pytest.fixture(scope="module")
def trained(small):
    from haseongpu_b200 import learned as LP

    mesh, _, _, ctx = small
    data = LP.training_set(ctx, LP.pump_fields(mesh, 32, LP.TRAIN_SEED))
    net, hist = LP.train_proposal(data, steps=3000)
    ctx.update_beta(mesh.betaVolume)
    yield net, hist
    net.close()


def test_features_match_definition(small):
    mesh, sa, se, ctx = small
    first, count = 123, 3
    f = ctx.proposal_features(first, count, monochromatic=True)
    assert f.shape == (count, mesh.numberOfPrisms, 12) and np.all(np.isfinite(f))
    T, Np = mesh.numberOfTriangles, mesh.numberOfPoints
    cen = mesh.points[mesh.triangles].mean(axis=1)
    R = np.sqrt((mesh.points ** 2).sum(1)).max()
    H = mesh.thickness * (mesh.numberOfLevels - 1)
    for i in range(count):
        s = first + i
        S = np.array([*mesh.points[s % Np], (s // Np) * mesh.thickness])
        p = np.arange(mesh.numberOfPrisms)
        c = np.column_stack([cen[p % T], (p // T + 0.5) * mesh.thickness])
        d = np.linalg.norm(c - S, axis=1)
        np.testing.assert_allclose(f[i, :, 0:3], np.broadcast_to(S / [R, R, H], (p.size, 3)), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(f[i, :, 3:6], (c - S) / [R, R, H], rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(f[i, :, 6], np.log(d / R), rtol=1e-4, atol=1e-5)
        np.testing.assert_allclose(f[i, :, 7], mesh.betaVolume.astype(np.float32), rtol=1e-6)
        np.testing.assert_allclose(f[i, :, 10], 0.0)
        np.testing.assert_allclose(f[i, :, 11], np.log(se[0] / sa[0]), rtol=1e-4)


def test_logged_contributions_sum_to_the_estimate(small):
    mesh, _, _, ctx = small
    res, con = ctx.log_contributions(minRays=20000, monochromatic=True, minSample=40, maxSample=71, rngSeed=3)
    est = con.astype(np.float64).sum(axis=1) / res.totalRays
    np.testing.assert_allclose(est, res.phiAse, rtol=2e-4)
    ref = ctx.calc_phi_ase(minRays=20000, monochromatic=True, minSample=40, maxSample=71, rngSeed=3)
    np.testing.assert_array_equal(ref.phiAse, res.phiAse)  # logging does not change the rays


def _z(a, b):
    return (a.phiAse - b.phiAse) / np.sqrt((a.standardError) ** 2 + (b.standardError) ** 2)


def test_learned_estimates_are_unbiased(small, trained):
    from haseongpu_b200.proposal import ProposalNet

    mesh, _, _, ctx = small
    net, _ = trained
    kw = dict(minRays=50000, monochromatic=True, minSample=2000, maxSample=2511, rngSeed=8)
    plain = ctx.calc_phi_ase(**kw)
    with ProposalNet(seed=5) as untrained:
        for n in (untrained, net):
            r = ctx.calc_phi_ase_learned(n, **kw)
            z = _z(r, plain)
            assert abs(z.mean()) < 4.0 / np.sqrt(z.size), z.mean()
            assert np.mean(np.abs(z) < 4.0) > 0.99
            assert r.fallbackSamples == 0 and np.all(r.totalRays == 50000)


def test_trained_network_lowers_the_variance_on_unseen_fields(small, trained):
    from haseongpu_b200 import learned as LP

    mesh, _, _, ctx = small
    net, hist = trained
    assert hist[-200:].mean() < hist[:50].mean()
    for k, beta in enumerate(LP.pump_fields(mesh, 2, LP.EVAL_SEED)):
        ctx.update_beta(beta)
        kw = dict(minRays=20000, monochromatic=True, minSample=0, maxSample=mesh.numberOfSamples - 1, rngSeed=50 + k)
        legacy = LP.per_ray_variance(ctx.calc_phi_ase(nearFieldSampling=False, **kw))
        near = LP.per_ray_variance(ctx.calc_phi_ase(**kw))
        lv = LP.per_ray_variance(ctx.calc_phi_ase_learned(net, **kw))
        assert np.median(lv) < 0.75 * np.median(near), (np.median(lv), np.median(near))
        assert np.median(lv) < 0.1 * np.median(legacy)
        assert lv.max() < 0.01 * legacy.max()
    ctx.update_beta(mesh.betaVolume)


def test_fallback_restarts_samples_with_the_importance_weights(small, trained):
    mesh, _, _, ctx = small
    net, _ = trained
    kw = dict(minRays=20000, maxRays=80000, adaptiveSteps=2, mseThreshold=1e-9, monochromatic=True, minSample=100,
              maxSample=163, rngSeed=4)
    plain = ctx.calc_phi_ase(**kw)
    r = ctx.calc_phi_ase_learned(net, fallbackVariance=1e-12, **kw)
    assert r.fallbackSamples == 64
    assert np.all(r.totalRays == 80000 - 20000)  # restarted after the first pass
    z = _z(r, plain)
    assert np.mean(np.abs(z) < 4.0) > 0.95
    none = ctx.calc_phi_ase_learned(net, fallbackVariance=1e9, **kw)
    assert none.fallbackSamples == 0 and np.all(none.totalRays == 80000)
