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


def _feature_grid(mesh, A, B, cells_along=48):
    """The coarse gain grid the features sample, restated in float32: the
    mean g = A beta - B of the prisms whose centre lies in each cell
    (ascending triangle order), empty cells filled sweep by sweep from their
    filled 4-neighbours (+x, -x, +y, -y)."""
    f32 = np.float32
    pts = mesh.points.astype(f32)
    x0, y0 = pts[:, 0].min(), pts[:, 1].min()
    x1, y1 = pts[:, 0].max(), pts[:, 1].max()
    cell = f32(max(x1 - x0, y1 - y0) / f32(cells_along) * f32(1.0001))
    gx, gy = int(np.ceil((x1 - x0) / cell)) + 1, int(np.ceil((y1 - y0) / cell)) + 1
    cen = pts[mesh.triangles].astype(np.float64).mean(axis=1).astype(f32)
    ix = np.minimum(gx - 1, ((cen[:, 0] - x0) / cell).astype(np.int64))
    iy = np.minimum(gy - 1, ((cen[:, 1] - y0) / cell).astype(np.int64))
    T, L = mesh.numberOfTriangles, mesh.numberOfLevels - 1
    beta = mesh.betaVolume.astype(f32).reshape(L, T)
    grid = np.zeros((L, gy, gx), f32)
    filled = np.zeros((gy, gx), bool)
    for l in range(L):
        total = np.zeros((gy, gx), f32)
        count = np.zeros((gy, gx), np.int64)
        for t in range(T):
            total[iy[t], ix[t]] = f32(total[iy[t], ix[t]] + f32(A * float(beta[l, t]) - B))
            count[iy[t], ix[t]] += 1
        grid[l] = np.where(count > 0, total / np.maximum(count, 1).astype(f32), f32(0))
        filled = count > 0
    for _ in range(gx + gy):
        now = []
        for y in range(gy):
            for x in range(gx):
                if filled[y, x]:
                    continue
                nbs = [(y, x + 1), (y, x - 1), (y + 1, x), (y - 1, x)]
                nbs = [(a, b) for a, b in nbs if 0 <= a < gy and 0 <= b < gx and filled[a, b]]
                if nbs:
                    now.append((y, x, nbs))
        if not now:
            break
        for l in range(L):
            vals = []
            for y, x, nbs in now:
                acc = f32(0)
                for a, b in nbs:
                    acc = f32(acc + grid[l, a, b])
                vals.append(f32(acc / f32(len(nbs))))
            for (y, x, _), v in zip(now, vals):
                grid[l, y, x] = v
        for y, x, _ in now:
            filled[y, x] = True
    return grid, x0, y0, cell


def test_feature_grid_matches_its_definition(small):
    """Feature 8 (the straight-line ln gain estimated on the coarse grid at 8
    points of the segment) on a non-uniform beta field, against the grid
    restated on the CPU: the device builds the grid from the resident beta."""
    from haseongpu_b200 import learned as LP

    mesh, sa, se, ctx = small
    beta = LP.pump_fields(mesh, 1, 99)[0]
    ctx.update_beta(beta)
    try:
        first, count = 321, 2
        f = ctx.proposal_features(first, count, monochromatic=True)
    finally:
        ctx.update_beta(mesh.betaVolume)
    A, B = mesh.nTot * (se[0] + sa[0]), mesh.nTot * sa[0]
    grid, x0, y0, cell = _feature_grid(mesh.withBeta(beta), A, B)
    T, Np, L, h = mesh.numberOfTriangles, mesh.numberOfPoints, mesh.numberOfLevels - 1, mesh.thickness
    cen = mesh.points[mesh.triangles].mean(axis=1)
    p = np.arange(mesh.numberOfPrisms)
    for i in range(count):
        s = first + i
        S = np.array([*mesh.points[s % Np], (s // Np) * h])
        c = np.column_stack([cen[p % T], (p // T + 0.5) * h])
        lng = np.zeros(p.size)
        for k in range(8):
            a = (k + 0.5) / 8
            x, y, z = (S + a * (c - S)).T
            ly = np.clip((z / h).astype(np.int64), 0, L - 1)
            gxi = np.clip(((x - x0) / cell).astype(np.int64), 0, grid.shape[2] - 1)
            gyi = np.clip(((y - y0) / cell).astype(np.int64), 0, grid.shape[1] - 1)
            lng += grid[ly, gyi, gxi]
        lng = lng / 8 * np.linalg.norm(c - S, axis=1)
        rel = np.abs(f[i, :, 8] - lng) / np.maximum(np.abs(lng), 1e-3)
        assert np.quantile(rel, 0.999) < 1e-4, np.quantile(rel, 0.999)  # a point on a cell edge may round over


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
