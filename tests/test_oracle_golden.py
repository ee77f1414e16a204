"""CPU tests: the FP64 oracle against the reference's golden data.

Pins (reference paths):
* Philox4x32-10 known answers (Random123 kat_vectors, the generator the
  reference uses through alpaka: include/kernels/forward/accumulation.hpp:389).
* Per-triangle tables against pyInclude/geometry/core.py:_derived_topology.
* phi-ASE against the legacy serial buffers tests/data/compareSerial/phiase_reference.npz
  (1e6 rays/sample) and the legacy backward-method run
  tests/data/laserPumpCladding/true_cladding_no_reflection_phiase_reference.
* dndt = (beta (sigmaE + sigmaA) - sigmaA) phi, exact on every stored value.
* The analytic known answer for uniform beta and gain
  (tests/python/phiAse/test_analyticalSphere.py:19-31, generalised).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, analytic_phi, legacy_mesh, legacy_spectrum

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expected", KAT)
def test_philox_known_answers(oracle, ctr, key, expected):
    assert tuple(oracle.philox(ctr, key)) == expected


@pytest.mark.parametrize("name", ["cuboid", "cylindrical", "true_cladding", "delaunay"])
def test_tables_match_reference_builder(oracle, name):
    ref = np.load(GOLDEN / "mesh_tables.npz")
    pts, tri = ref[f"{name}_points2d"], ref[f"{name}_triangles"]
    T = tri.shape[0]
    ours = oracle.build_tables(pts, tri)
    fo = lambda key: ref[f"{name}_{key}"].reshape(3, T).T  # reference stores F-order [e*T + t]
    np.testing.assert_array_equal(ours["neighbors"], fo("triangleNeighbors"))
    np.testing.assert_array_equal(ours["forbiddenEdge"], fo("forbiddenEdge"))
    p = pts[tri]
    orient = np.sign((p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 1, 1] - p[:, 0, 1]) * (p[:, 2, 0] - p[:, 0, 0]))
    # the reference keeps the right-hand normal of each edge; ours points outward
    np.testing.assert_allclose(ours["normalX"], orient[:, None] * fo("triangleNormalsX"), atol=1e-12)
    np.testing.assert_allclose(ours["normalY"], orient[:, None] * fo("triangleNormalsY"), atol=1e-12)
    np.testing.assert_allclose(ours["centerX"], ref[f"{name}_triangleCenterX"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(ours["centerY"], ref[f"{name}_triangleCenterY"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(ours["area"].astype(np.float32), ref[f"{name}_triangleSurfaces"], rtol=1e-6)
    # edge line passes through the reference's normal point
    npnt = fo("triangleNormalPoint")
    np.testing.assert_allclose(ours["edgeC"], ours["normalX"] * pts[npnt, 0] + ours["normalY"] * pts[npnt, 1],
                               atol=1e-12)


@pytest.mark.parametrize("name", ["cuboid", "cylindrical"])
def test_dndt_formula_is_exact_on_legacy_buffers(name):
    d = np.load(GOLDEN / f"legacy_{name}.npz")
    pred = (d["betaCells"] * (d["sigmaE"] + d["sigmaA"]) - d["sigmaA"]) * d["phiASE"]
    np.testing.assert_array_equal(pred, d["dndtAse"])


@pytest.mark.parametrize("name", ["cuboid", "cylindrical"])
def test_oracle_matches_legacy_serial_reference(oracle, name):
    d = np.load(GOLDEN / f"legacy_{name}.npz")
    mesh = legacy_mesh(name)
    samples = np.arange(0, d["phiASE"].size, 61)
    phi = np.empty(samples.size)
    rse = np.empty(samples.size)
    for i, s in enumerate(samples):
        r = oracle.phi_ase(mesh, legacy_spectrum(name), minRays=20000, minSample=int(s), maxSample=int(s))
        phi[i], rse[i] = r["phiAse"][0], r["mse"][0]
        assert r["droppedRays"][0] == 0
    ratio = phi / d["phiASE"][samples]
    # The legacy buffers hold 1e6 rays/sample: their own error is ~0.1 %.
    assert abs(ratio.mean() - 1.0) < 0.01, ratio.mean()
    assert abs(np.median(ratio) - 1.0) < 0.01, np.median(ratio)
    z = (phi - d["phiASE"][samples]) / (rse * phi)
    assert np.mean(np.abs(z) < 3.0) > 0.85  # heavy-tailed 1/d^2 weights: the RSE itself is noisy


def test_oracle_matches_legacy_true_cladding_run(oracle):
    d = np.load(GOLDEN / "legacy_true_cladding.npz")
    sp = ([float(d["sigmaA"])], [float(d["sigmaE"])])
    means = []
    for k, absorption in enumerate(d["claddingAbsorptions"]):
        mesh = legacy_mesh("true_cladding", claddingAbsorption=float(absorption))
        r = oracle.phi_ase(mesh, sp, minRays=2000, minSample=0, maxSample=4209, seed=5489)
        assert r["droppedRays"].sum() == 0
        ratio = r["phiAse"] / d["phiASE"][k]
        # Both are 2,000-ray estimates; the legacy one drops prisms whose
        # floor(N w/W) is 0 and re-spreads the remainder uniformly.
        assert abs(ratio.mean() - 1.0) < 0.03
        assert abs(np.median(ratio) - 1.0) < 0.02
        means.append(r["phiAse"].mean())
        np.testing.assert_array_equal(r["totalRays"], d["totalRays"][k])
    assert means[0] > means[1] > means[2]  # cladding absorption lowers the flux


def test_legacy_mse_is_the_scaled_standard_error(oracle):
    """The legacy archive's ``mse`` is the standard error of the unnormalised
    estimator, phi tau / N_tot (a length), not a relative error:
    mse = RSE * phi * tau / N_tot.  Per sample both RSEs are noisy 2,000-ray
    estimates of a heavy-tailed weight, so the mapping is pinned on the
    distribution: every decile of the archive's mse * (N_tot/tau) / phi lies
    within 1.0-1.3x of the same decile of the oracle's RSE with uniform start
    points (the legacy estimator; its cruder floor-plus-leftover ray split
    accounts for the excess), while the archive's mse itself is ~20x below
    that RSE.  Every threshold of this build is applied to the RSE, the
    reference's current relativeStandardErrorThreshold."""
    d = np.load(GOLDEN / "legacy_true_cladding.npz")
    sp = ([float(d["sigmaA"])], [float(d["sigmaE"])])
    mesh = legacy_mesh("true_cladding", claddingAbsorption=float(d["claddingAbsorptions"][0]))
    r = oracle.phi_ase(mesh, sp, minRays=2000, seed=5489, nearField=False)
    scale = float(d["nTot"]) / float(d["crystalTFluo"])
    deciles = [10, 25, 50, 75, 90]
    for k in range(3):
        rse_legacy = d["mse"][k] * scale / d["phiASE"][k]
        ratio = np.percentile(rse_legacy, deciles) / np.percentile(r["mse"], deciles)
        assert np.all((ratio > 1.0) & (ratio < 1.3)), ratio
    assert np.median(r["mse"]) / np.median(d["mse"][0]) > 10.0


@pytest.mark.parametrize("near", [True, False])
@pytest.mark.parametrize("where", ["centre_bottom", "centre_mid", "edge_mid", "interior_top"])
def test_oracle_analytic_uniform_medium(oracle, where, near):
    from haseongpu_b200.configs import disc_small

    base = disc_small().mesh
    beta, nTot, tau, sa, se = 0.2, 1.38e20, 9.41e-4, 1.1e-21, 2.2e-20
    mesh = base.withBeta(np.full(base.numberOfPrisms, beta))
    g = nTot * (beta * (se + sa) - sa)
    Np = mesh.numberOfPoints
    outer = int(np.argmax(np.linalg.norm(mesh.points, axis=1)))
    inner = int(np.argsort(np.linalg.norm(mesh.points, axis=1))[40])
    sample = {"centre_bottom": 0, "centre_mid": 5 * Np, "edge_mid": outer + 4 * Np, "interior_top": inner + 9 * Np}[where]
    xyz = mesh.samplePoints()[sample]
    expect = analytic_phi(mesh, xyz, beta, g, nTot, tau)
    r = oracle.phi_ase(mesh, ([sa], [se]), minRays=200000, minSample=sample, maxSample=sample, nearField=near)
    assert r["droppedRays"][0] == 0
    rel = r["phiAse"][0] / expect - 1.0
    assert abs(rel) < max(4.0 * r["mse"][0], 1e-3 if near else 2e-3), (rel, r["mse"][0])


def test_ray_map_systematic_sampling(oracle):
    rng = np.random.default_rng(7)
    w = rng.uniform(0, 1, 500).astype(np.float32)
    w[rng.uniform(size=500) < 0.2] = 0.0
    for rays, phase in [(1, 0), (1000, 123456789), (777, 0xFFFFFFFF), (100000, 42)]:
        Q, q, off = oracle.ray_map(w, rays, phase)
        assert Q == int(q.astype(np.uint64).sum())
        assert off[0] == 0 and off[-1] == rays and np.all(np.diff(off.astype(np.int64)) >= 0)
        n = np.diff(off.astype(np.int64))
        expect = rays * q.astype(np.float64) / Q
        assert np.all(n >= np.floor(expect) - 1e-9) and np.all(n <= np.ceil(expect) + 1e-9)
        assert np.all(n[w == 0] == 0)
        assert np.all(q[w > 0] >= 1)
    Q, q, off = oracle.ray_map(np.zeros(10, np.float32), 100, 0)
    assert Q == 0 and np.all(off == 0)


def test_oracle_adaptive_schedule(oracle):
    mesh = legacy_mesh("cylindrical")
    r = oracle.phi_ase(mesh, legacy_spectrum("cylindrical"), minRays=1000, maxRays=64000, adaptiveSteps=3,
                       mseThreshold=0.02, minSample=0, maxSample=60)
    targets = {1000, 4000, 16000, 64000}
    assert set(np.unique(r["totalRays"])) <= targets
    converged = r["mse"] <= 0.02
    assert np.all(converged | (r["totalRays"] == 64000))
    assert np.all(r["totalRays"][r["totalRays"] > 1000] > 1000)
