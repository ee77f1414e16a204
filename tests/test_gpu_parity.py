"""GPU parity: libhase_b200 (through its C ABI) against the FP64 oracle.

Levels (tolerances are the ones stated for this path):
* Philox4x32-10 on the device: bit-exact with the oracle and the Random123 known answers.
* Deterministic kernels: ln(gain) along fixed rays within 1e-5 (i.e. gain
  within 1e-5 relative) and normalised importance weights within 1e-5
  relative for at least 99.9 % of rays; the FP32 geometry moves the crossing
  point of a ray that grazes an edge (|n.u| << 1) by ~1e-7/|n.u| cm, so the
  few remaining rays are held to 5e-4.
* Integer ray->prism map: bit-exact with the oracle given identical weights.
* Full estimator replayed with the device's own weights: the oracle walks the
  same rays in FP64, so per-sample phi agrees to 1e-4 relative.
* Statistical: against the legacy golden buffers and the analytic known answer
  within the Monte Carlo error.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, analytic_phi, legacy_mesh, legacy_spectrum

pytestmark = pytest.mark.gpu


def _ctx(mesh, sa, se):
    from haseongpu_b200 import DeviceMesh

    return DeviceMesh(mesh, sa, se)


def _random_rays(mesh, n, rng, slices=1):
    T, L, Np = mesh.numberOfTriangles, mesh.numberOfLevels, mesh.numberOfPoints
    tri = rng.integers(0, T, n)
    level = rng.integers(0, L - 1, n)
    u = rng.uniform(size=(n, 2))
    flip = u.sum(axis=1) > 1
    u[flip] = 1 - u[flip]
    p = mesh.points[mesh.triangles[tri]]
    xy = p[:, 0] + u[:, :1] * (p[:, 1] - p[:, 0]) + u[:, 1:] * (p[:, 2] - p[:, 0])
    z = (level + rng.uniform(0.01, 0.99, n)) * mesh.thickness
    start = np.column_stack([xy, z]).astype(np.float32).astype(np.float64)  # exactly representable in FP32
    sample = rng.integers(0, Np * L, n)
    slice_ = rng.integers(0, slices, n)
    return start, tri, level, sample, slice_


def test_device_philox_matches_oracle(native, oracle):
    rng = np.random.default_rng(3)
    ctr = rng.integers(0, 2**32, size=(4096, 4), dtype=np.uint64).astype(np.uint32)
    key = (0xA4093822, 0x299F31D0)
    dev = native.philox(ctr, key)
    for i in range(0, 4096, 97):
        assert tuple(dev[i]) == tuple(oracle.philox(ctr[i], key))
    kat = native.philox([[0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344]], key)
    assert tuple(kat[0]) == (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


@pytest.mark.parametrize("name", ["cylindrical", "true_cladding"])
def test_trace_matches_oracle(oracle, name):
    mesh = legacy_mesh(name, claddingAbsorption=5.5 if name == "true_cladding" else None)
    sa, se = legacy_spectrum(name)
    rng = np.random.default_rng(11)
    start, tri, level, sample, sl = _random_rays(mesh, 20000, rng)
    with _ctx(mesh, sa, se) as ctx:
        ln_d, dist_d, drop_d = ctx.trace(start, tri, level, sample, sl)
    ln_o, dist_o, drop_o = oracle.trace(mesh, (sa, se), start, tri, level, sample, sl)
    assert drop_o.sum() == 0 and drop_d.sum() == 0
    np.testing.assert_allclose(dist_d, dist_o, rtol=2e-6)
    err = np.abs(ln_d.astype(np.float64) - ln_o)
    assert np.quantile(err, 0.999) < 1e-5 and err.max() < 5e-4, (err.max(), np.quantile(err, 0.999))


def test_trace_with_reflections_matches_oracle(oracle):
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    mesh = w.mesh
    sa, se = w.spectra.resampled()
    rng = np.random.default_rng(5)
    start, tri, level, sample, sl = _random_rays(mesh, 20000, rng, slices=5)
    with _ctx(mesh, sa, se) as ctx:
        ln_d, _, drop_d = ctx.trace(start, tri, level, sample, sl, wavelength=7)
    ln_o, _, drop_o = oracle.trace(mesh, (sa, se), start, tri, level, sample, sl, wavelength=7)
    assert drop_o.sum() == 0 and drop_d.sum() == 0
    err = np.abs(ln_d.astype(np.float64) - ln_o)
    assert np.quantile(err, 0.999) < 1e-5 and err.max() < 5e-4, (err.max(), np.quantile(err, 0.999))


@pytest.mark.parametrize("workload", ["disc_small", "disc_poly"])
def test_importance_kernels_give_identical_estimates(workload):
    """The line-team kernel (importanceLayers 0) and the layer-group kernel
    (2, 4, 8 layers per thread) run the same per-line arithmetic: identical
    weights, hence identical ray maps and bit-identical estimates; and the
    crossing count of the walks is positive and reproducible."""
    from haseongpu_b200 import configs

    w = configs.WORKLOADS[workload]()
    sa, se = w.spectra.resampled(w.monochromatic)
    kw = dict(minRays=3000, useReflections=w.useReflections, monochromatic=w.monochromatic, rngSeed=5,
              minSample=100, maxSample=131)
    with _ctx(w.mesh, sa, se) as ctx:
        runs = [ctx.calc_phi_ase(importanceLayers=g, **kw) for g in (0, 2, 4, 8)]
        n1 = ctx.importance_crossings(100, 32, w.useReflections)
        n2 = ctx.importance_crossings(100, 32, w.useReflections)
    for r in runs[1:]:
        np.testing.assert_array_equal(r.phiAse, runs[0].phiAse)
        np.testing.assert_array_equal(r.relativeStandardError, runs[0].relativeStandardError)
    lines = 32 * (5 if w.useReflections else 1) * w.mesh.numberOfPrisms
    assert n1 == n2 and n1 > lines


@pytest.mark.parametrize("reflections", [False, True])
def test_importance_weights_match_oracle(oracle, reflections):
    from haseongpu_b200.configs import disc_poly, disc_small

    w = disc_poly() if reflections else disc_small()
    mesh = w.mesh
    sa, se = w.spectra.resampled(w.monochromatic)
    samples = [0, 17, mesh.numberOfPoints * 3 + 5, mesh.numberOfSamples - 1]
    with _ctx(mesh, sa, se) as ctx:
        for s in samples:
            dev = ctx.importance_weights(s, 1, reflections)[0].astype(np.float64)
            ref = oracle.importance(mesh, (sa, se), s, 5 if reflections else 1)
            ref = ref / ref.max()
            big = ref > 1e-6
            rel = np.abs(dev[big] / ref[big] - 1.0)
            assert np.quantile(rel, 0.999) < 1e-5 and rel.max() < 5e-4, (np.quantile(rel, 0.999), rel.max())
            np.testing.assert_array_equal(dev == 0, ref == 0)


def test_ray_map_bit_exact(native, oracle):
    rng = np.random.default_rng(9)
    rows = []
    for n in (1, 7, 1000, 9126, 40000):
        w = rng.uniform(0, 1, n).astype(np.float32) ** 4
        w[rng.uniform(size=n) < 0.3] = 0.0
        rows.append(w)
    for w in rows:
        for rays in (1, 999, 100000, 10_000_000):
            phase = int(rng.integers(0, 2**32))
            Q, q, off = native.ray_map(w[None, :], rays, [phase])
            Qo, qo, offo = oracle.ray_map(w, rays, phase)
            assert int(Q[0]) == Qo
            np.testing.assert_array_equal(q[0], qo)
            np.testing.assert_array_equal(off[0], offo)


def test_device_weights_map_bit_exact(oracle):
    """The map kernel on the importance kernel's own weights equals the oracle's map."""
    from haseongpu_b200.configs import disc_small

    w = disc_small()
    with _ctx(w.mesh, *w.spectra.resampled(True)) as ctx:
        W = ctx.importance_weights(100, 3)
    from haseongpu_b200 import _native

    Q, q, off = _native.ray_map(W, 123457, [1, 2, 3])
    for i in range(3):
        Qo, qo, offo = oracle.ray_map(W[i], 123457, i + 1)
        assert int(Q[i]) == Qo
        np.testing.assert_array_equal(off[i], offo)


@pytest.mark.parametrize("workload", ["disc_small", "disc_poly"])
def test_estimator_replay_matches_oracle(oracle, workload):
    from haseongpu_b200 import configs

    w = configs.WORKLOADS[workload]()
    mesh = w.mesh
    sa, se = w.spectra.resampled(w.monochromatic)
    first, count = 37, 24
    with _ctx(mesh, sa, se) as ctx:
        W = ctx.importance_weights(first, count, w.useReflections)
        dev = ctx.calc_phi_ase(minRays=20000, useReflections=w.useReflections, monochromatic=w.monochromatic,
                               rngSeed=1234, minSample=first, maxSample=first + count - 1)
    ref = oracle.phi_ase(mesh, (sa, se), minRays=20000, useReflections=w.useReflections, seed=1234,
                         minSample=first, maxSample=first + count - 1, weights=W)
    np.testing.assert_array_equal(dev.totalRays, ref["totalRays"])
    assert dev.droppedRays.sum() == 0 and ref["droppedRays"].sum() == 0
    np.testing.assert_allclose(dev.phiAse, ref["phiAse"], rtol=1e-4)
    np.testing.assert_allclose(dev.relativeStandardError, ref["mse"], rtol=1e-3, atol=1e-7)


@pytest.mark.parametrize("workload", ["disc_small", "disc_poly"])
def test_adaptive_multipass_replay_matches_oracle(oracle, workload):
    """Kernel (d): the multi-pass adaptive solve (geometric ray targets, only
    the samples above the threshold topped up on each pass) replayed by the
    oracle with the device's weights.  The threshold is set inside the
    first-pass error distribution so that samples stop on different passes.
    The device and the oracle compare slightly different FP32/FP64 errors
    with the threshold, so the oracle is run at threshold * (1 -+ 2e-3):
    every device sample must stop exactly where one of the two stops (and
    almost all where both do), with phi within 1e-4 of that oracle run."""
    from haseongpu_b200 import configs

    w = configs.WORKLOADS[workload]()
    mesh = w.mesh
    sa, se = w.spectra.resampled(w.monochromatic)
    first, count = 150, 96
    # six geometric passes 4096 -> 32768 rays (the error falls by 2^(1/4) per
    # pass), the threshold where the median sample stops on the fourth
    kw = dict(minRays=4096, maxRays=32768, adaptiveSteps=6, useReflections=w.useReflections)
    growth = (32768 / 4096) ** (1.0 / 6)  # the schedule's own arithmetic (include/core/types.hpp:333-354)
    targets = [min(32768, max(4096, int(np.ceil(4096 * growth ** k)))) if k < 6 else 32768 for k in range(7)]
    rng = dict(minSample=first, maxSample=first + count - 1)
    with _ctx(mesh, sa, se) as ctx:
        W = ctx.importance_weights(first, count, w.useReflections)
        one = ctx.calc_phi_ase(minRays=4096, useReflections=w.useReflections, monochromatic=w.monochromatic,
                               rngSeed=77, **rng)
        thr = float(np.median(one.relativeStandardError)) * np.sqrt(4096 / targets[3])
        dev = ctx.calc_phi_ase(mseThreshold=thr, monochromatic=w.monochromatic, rngSeed=77, **kw, **rng)
    lo, hi = (oracle.phi_ase(mesh, (sa, se), mseThreshold=thr * f, seed=77, weights=W, **kw, **rng)
              for f in (1.0 - 2e-3, 1.0 + 2e-3))
    assert len(np.unique(dev.totalRays)) >= 3, np.unique(dev.totalRays)  # several passes end somewhere
    assert set(np.unique(dev.totalRays)) <= set(targets)
    same_lo, same_hi = dev.totalRays == lo["totalRays"], dev.totalRays == hi["totalRays"]
    assert np.all(same_lo | same_hi), np.flatnonzero(~(same_lo | same_hi))
    assert np.mean(same_lo & same_hi) >= 0.9  # the rest sit within 0.2 % of the threshold on some pass
    ref = np.where(same_lo, lo["phiAse"], hi["phiAse"])
    np.testing.assert_allclose(dev.phiAse, ref, rtol=1e-4)
    ref_rse = np.where(same_lo, lo["mse"], hi["mse"])
    np.testing.assert_allclose(dev.relativeStandardError, ref_rse, rtol=1e-3, atol=1e-7)
    assert dev.raysTraced == int(dev.totalRays.astype(np.int64).sum())
    assert dev.unconvergedSamples == int(np.sum(dev.relativeStandardError > thr))


@pytest.mark.parametrize("name", ["cuboid", "cylindrical"])
def test_gpu_matches_legacy_serial_reference(name):
    """Per-sample agreement with the legacy serial buffers (1e6 rays/sample,
    uniform start points): ratios within 0.3 % (mean) / 0.5 % (median) for
    both samplers, dndt exact, and the near-field estimator's volume integral
    within 0.3 %."""
    d = np.load(GOLDEN / f"legacy_{name}.npz")
    mesh = legacy_mesh(name)
    sa, se = legacy_spectrum(name)
    with _ctx(mesh, sa, se) as ctx:
        plain = ctx.calc_phi_ase(minRays=200000, rngSeed=5489, nearFieldSampling=False)
        near = ctx.calc_phi_ase(minRays=200000, rngSeed=5489)
    legacy = d["phiASE"]
    for r in (plain, near):
        assert r.droppedRays.sum() <= 1e-7 * r.raysTraced
        ratio = r.phiAse / legacy
        assert abs(ratio.mean() - 1.0) < 0.003, ratio.mean()
        assert abs(np.median(ratio) - 1.0) < 0.005, np.median(ratio)
        np.testing.assert_allclose(r.dndtAse,
                                   (d["betaCells"] * (se[0] + sa[0]) - sa[0]) * r.phiAse.astype(np.float64), rtol=1e-12)
    assert abs(near.phiAse.astype(np.float64).sum() / legacy.sum() - 1.0) < 0.003
    assert np.median(near.relativeStandardError) < 0.5 * np.median(plain.relativeStandardError)


@pytest.mark.parametrize("name", ["cuboid", "cylindrical"])
def test_gpu_within_3_sigma_of_the_oracle(oracle, name):
    """The statistical level at its stated tolerance: per-sample phi of the
    device (near-field start points, bounded weights, seed 11) against the
    FP64 oracle's independent estimate (seed 12), every sample of the legacy
    meshes, within 3 sigma of the combined Monte Carlo standard error
    sigma = sqrt(sigma_gpu^2 + sigma_oracle^2).  The i.i.d. error formula
    overstates the error of the systematic (stratified) ray->prism split, so
    z is narrower than N(0, 1): at most 0.5 % of samples beyond 3 sigma
    (0.27 % for N(0, 1)), a centred mean and a spread below 1.05."""
    mesh = legacy_mesh(name)
    sa, se = legacy_spectrum(name)
    with _ctx(mesh, sa, se) as ctx:
        dev = ctx.calc_phi_ase(minRays=20000, rngSeed=11)
    ref = oracle.phi_ase(mesh, (sa, se), minRays=20000, seed=12)
    sig = np.hypot(dev.relativeStandardError * dev.phiAse, ref["mse"] * ref["phiAse"])
    z = (dev.phiAse - ref["phiAse"]) / sig
    assert np.mean(np.abs(z) < 3.0) >= 0.995, np.mean(np.abs(z) < 3.0)
    assert abs(z.mean()) < 4.0 / np.sqrt(z.size), z.mean()
    assert z.std() < 1.05, z.std()


@pytest.mark.parametrize("name", ["cuboid", "cylindrical"])
def test_legacy_buffers_scatter_like_the_uniform_estimator(name):
    """Why the legacy buffers are not held to 3 sigma per sample: with uniform
    start points the 1/d^2 weight of the prisms touching a sample has an
    infinite variance (P(X > x) ~ x^-3/2), so a 1e6-ray estimate is skewed
    below its mean and its sample error is not a standard deviation.  Against
    the bounded near-field estimate at 4e6 rays (relative error ~5e-4), the
    standardised deviations z = (estimate - near) / sigma_1e6 of the legacy
    buffers and of this build's own uniform-start estimator at the same 1e6
    rays are both skewed the same way (median below -0.3), and the legacy
    buffers scatter at most 1.8x wider (their proposal has no prism volume
    and splits rays by floor plus random leftovers)."""
    d = np.load(GOLDEN / f"legacy_{name}.npz")
    mesh = legacy_mesh(name)
    sa, se = legacy_spectrum(name)
    with _ctx(mesh, sa, se) as ctx:
        near = ctx.calc_phi_ase(minRays=4_000_000, rngSeed=21)
        plain = ctx.calc_phi_ase(minRays=1_000_000, rngSeed=22, nearFieldSampling=False)
    assert np.median(near.relativeStandardError) < 1.5e-3
    sig = plain.relativeStandardError * plain.phiAse
    z_legacy = (d["phiASE"] - near.phiAse) / sig
    z_ours = (plain.phiAse - near.phiAse) / sig
    assert np.median(z_ours) < -0.3 and np.median(z_legacy) < -0.3, (np.median(z_ours), np.median(z_legacy))
    spread = lambda z: np.subtract(*np.percentile(z, [80, 20]))  # noqa: E731
    assert 1.0 <= spread(z_legacy) / spread(z_ours) <= 1.8, spread(z_legacy) / spread(z_ours)
    assert abs(np.mean(d["phiASE"] / near.phiAse) - 1.0) < 0.003


def test_gpu_matches_legacy_true_cladding_run():
    d = np.load(GOLDEN / "legacy_true_cladding.npz")
    sp = ([float(d["sigmaA"])], [float(d["sigmaE"])])
    means = []
    for k, absorption in enumerate(d["claddingAbsorptions"]):
        mesh = legacy_mesh("true_cladding", claddingAbsorption=float(absorption))
        with _ctx(mesh, *sp) as ctx:
            r = ctx.calc_phi_ase(minRays=2000, rngSeed=5489)
        ratio = r.phiAse / d["phiASE"][k]
        assert abs(ratio.mean() - 1.0) < 0.03 and abs(np.median(ratio) - 1.0) < 0.02
        np.testing.assert_array_equal(r.totalRays, d["totalRays"][k])
        means.append(r.phiAse.mean())
    assert means[0] > means[1] > means[2]


@pytest.mark.parametrize("near", [True, False])
def test_gpu_analytic_uniform_medium(near):
    from haseongpu_b200.configs import disc_small

    base = disc_small().mesh
    beta, nTot, tau, sa, se = 0.2, 1.38e20, 9.41e-4, 1.1e-21, 2.2e-20
    mesh = base.withBeta(np.full(base.numberOfPrisms, beta))
    g = nTot * (beta * (se + sa) - sa)
    Np = mesh.numberOfPoints
    rr = np.linalg.norm(mesh.points, axis=1)
    outer, inner = int(np.argmax(rr)), int(np.argsort(rr)[40])
    samples = [0, 5 * Np, outer + 4 * Np, inner + 9 * Np, outer]
    with _ctx(mesh, [sa], [se]) as ctx:
        for s in samples:
            r = ctx.calc_phi_ase(minRays=4_000_000, minSample=s, maxSample=s, rngSeed=99, nearFieldSampling=near)
            expect = analytic_phi(mesh, mesh.samplePoints()[s], beta, g, nTot, tau, 1024, 1024)
            rel = r.phiAse[0] / expect - 1.0
            tol = max(4 * r.relativeStandardError[0], 3e-4 if near else 1e-3)
            assert abs(rel) < tol, (s, rel, r.relativeStandardError[0])


def test_gpu_adaptive_relaunch_only_active_samples():
    mesh = legacy_mesh("cylindrical")
    sa, se = legacy_spectrum("cylindrical")
    with _ctx(mesh, sa, se) as ctx:
        r = ctx.calc_phi_ase(minRays=1000, maxRays=64000, adaptiveSteps=3, mseThreshold=0.02, maxSample=399)
    assert set(np.unique(r.totalRays)) <= {1000, 4000, 16000, 64000}
    assert np.all((r.relativeStandardError <= 0.02) | (r.totalRays == 64000))
    assert len(np.unique(r.totalRays)) > 1  # some samples stopped early, others were relaunched
    assert r.raysTraced == int(r.totalRays.astype(np.int64).sum())
    assert r.unconvergedSamples == int(np.sum(r.relativeStandardError > 0.02))


def test_gpu_reproducible_and_seed_dependent():
    mesh = legacy_mesh("cuboid")
    sa, se = legacy_spectrum("cuboid")
    with _ctx(mesh, sa, se) as ctx:
        a = ctx.calc_phi_ase(minRays=5000, rngSeed=1, maxSample=299)
        b = ctx.calc_phi_ase(minRays=5000, rngSeed=1, maxSample=299)
        c = ctx.calc_phi_ase(minRays=5000, rngSeed=2, maxSample=299)
    np.testing.assert_array_equal(a.phiAse, b.phiAse)
    assert np.any(a.phiAse != c.phiAse)


def test_phiase_front_end_runs_and_validates():
    from haseongpu_b200 import CrossSectionData, PhiASE

    mesh = legacy_mesh("cylindrical")
    sa, se = legacy_spectrum("cylindrical")
    spectra = CrossSectionData.monochromatic(wavelength=905e-9, crossSectionAbsorption=sa[0],
                                             crossSectionEmission=se[0])
    p = PhiASE(propagationMode="backward", minRays=4000, maxRays=4000, adaptiveSteps=1,
               relativeStandardErrorThreshold=0.1,
               monochromatic=True, rngSeed=7, minSampleRange=10, maxSampleRange=59)
    res = p.run(gainMedium=mesh, crossSections=spectra).getResults()
    assert res.phiAse.shape == (50,) and np.all(res.phiAse > 0)
    assert np.all(res.totalRays == 4000)
    np.testing.assert_allclose(res.standardError, res.relativeStandardError * res.phiAse, rtol=1e-6)
    mesh2 = mesh.withBeta(mesh.betaVolume * 0.5)
    res2 = p.run(gainMedium=mesh2, crossSections=spectra).getResults()
    assert res2.phiAse.mean() < res.phiAse.mean()


def test_update_beta_matches_fresh_context():
    mesh = legacy_mesh("cuboid")
    sa, se = legacy_spectrum("cuboid")
    beta2 = np.clip(mesh.betaVolume * 1.7, 0, 1)
    with _ctx(mesh, sa, se) as ctx:
        ctx.update_beta(beta2)
        a = ctx.calc_phi_ase(minRays=3000, maxSample=199, rngSeed=3)
    with _ctx(mesh.withBeta(beta2), sa, se) as ctx:
        b = ctx.calc_phi_ase(minRays=3000, maxSample=199, rngSeed=3)
    np.testing.assert_array_equal(a.phiAse, b.phiAse)


def test_invalid_arguments_raise():
    from haseongpu_b200._native import HaseError

    mesh = legacy_mesh("cuboid")
    sa, se = legacy_spectrum("cuboid")
    with _ctx(mesh, sa, se) as ctx:
        with pytest.raises(HaseError):
            ctx.calc_phi_ase(minRays=0)
        with pytest.raises(HaseError):
            ctx.calc_phi_ase(minRays=10, minSample=5, maxSample=mesh.numberOfSamples)
        with pytest.raises(HaseError):
            ctx.update_beta(np.full(mesh.numberOfPrisms, np.nan))


def test_every_ray_kernel_variant_gives_the_same_estimate():
    """The autotuner's launch shapes change scheduling only: identical results."""
    from haseongpu_b200.autotune import RAYS_PER_LANE, variant_names

    mesh = legacy_mesh("cylindrical")
    sa, se = legacy_spectrum("cylindrical")
    with _ctx(mesh, sa, se) as ctx:
        ref = ctx.calc_phi_ase(minRays=20000, rngSeed=4, maxSample=63)
        for v in range(len(variant_names())):
            for rpt in (RAYS_PER_LANE[0], RAYS_PER_LANE[-1]):
                r = ctx.calc_phi_ase(minRays=20000, rngSeed=4, maxSample=63, rayKernelVariant=v, raysPerThread=rpt)
                np.testing.assert_allclose(r.phiAse, ref.phiAse, rtol=1e-6)
                np.testing.assert_array_equal(r.totalRays, ref.totalRays)


@pytest.mark.parametrize("case", ["true_cladding", "disc_poly_reflections"])
def test_monochromatic_walk_matches_the_general_walk(case):
    """A monochromatic solve walks a table of each prism's gain coefficient g
    (built once per solve); the same medium given its wavelength pair twice
    takes the general walk, which reads beta and evaluates g at every crossing,
    and draws the same rays.  Both must agree bit for bit, cladding prisms and
    reflections included."""
    from haseongpu_b200 import configs

    if case == "true_cladding":
        mesh = legacy_mesh("true_cladding", claddingAbsorption=5.5)
        sa, se = legacy_spectrum("true_cladding")
        kw = dict(minRays=20000, rngSeed=5, maxSample=255)
    else:
        w = configs.disc_poly()
        mesh = w.mesh
        sa, se = (list(map(float, v[:1])) for v in w.spectra.resampled(True))
        kw = dict(minRays=20000, rngSeed=5, minSample=1000, maxSample=1127, useReflections=True)
    with _ctx(mesh, sa, se) as one, _ctx(mesh, sa * 2, se * 2) as two:
        a = one.calc_phi_ase(monochromatic=True, **kw)
        b = two.calc_phi_ase(monochromatic=False, **kw)
    assert a.crossings > 0
    np.testing.assert_array_equal(a.phiAse, b.phiAse)
    np.testing.assert_array_equal(a.relativeStandardError, b.relativeStandardError)
    np.testing.assert_array_equal(a.totalRays, b.totalRays)
    assert a.crossings == b.crossings


def test_gpu_polychromatic_seeds_agree_within_reported_error():
    """Two seeds of a polychromatic solve with reflections (disc_poly, 16
    wavelengths) agree within their reported errors: every ray averages its
    gain over the spectrum, so the rays are independent and the reported
    relative error holds."""
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    sa, se = w.spectra.resampled()
    kw = dict(minRays=400_000, useReflections=True, minSample=3000, maxSample=3127)
    with _ctx(w.mesh, sa, se) as ctx:
        a = ctx.calc_phi_ase(rngSeed=3, **kw)
        b = ctx.calc_phi_ase(rngSeed=5, **kw)
    sig = np.hypot(a.relativeStandardError * a.phiAse, b.relativeStandardError * b.phiAse)
    z = (a.phiAse.astype(np.float64) - b.phiAse) / sig
    assert z.std() < 1.3 and np.abs(z).max() < 4.5, (z.std(), np.abs(z).max())


def test_gpu_spectral_mean_equals_the_mean_of_monochromatic_solves():
    """A polychromatic solve averages every ray's gain over the spectrum (the
    walk's path integrals give each wavelength's exponent); its estimate is
    the mean of the monochromatic solves of the 16 wavelengths, within the
    combined Monte Carlo error (disc_poly, reflections, independent seeds)."""
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    sa, se = w.spectra.resampled()
    kw = dict(minRays=200_000, useReflections=True, minSample=3000, maxSample=3031)
    with _ctx(w.mesh, sa, se) as ctx:
        poly = ctx.calc_phi_ase(rngSeed=3, **kw)
    phis, var = [], []
    for lam in range(len(sa)):
        with _ctx(w.mesh, [float(sa[lam])], [float(se[lam])]) as one:
            r = one.calc_phi_ase(rngSeed=10 + lam, **kw)
        phis.append(r.phiAse.astype(np.float64))
        var.append((r.relativeStandardError * r.phiAse.astype(np.float64)) ** 2)
    mean = np.mean(phis, axis=0)
    sigma = np.hypot(poly.relativeStandardError * poly.phiAse, np.sqrt(np.sum(var, axis=0)) / len(sa))
    z = (poly.phiAse.astype(np.float64) - mean) / sigma
    assert np.abs(z).max() < 4.5 and abs(z.mean()) < 4.0 / np.sqrt(z.size), (np.abs(z).max(), z.mean())
