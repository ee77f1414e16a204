"""GPU parity of the forward Tet4 path (include/hase_b200_forward.h) against
the FP64 forward oracle and the reference's known answers.

Tolerances: the device and the oracle build identical tables on the host and
draw identical Philox4x32-10 streams, so both walk the same rays; they differ
only by FMA contraction and the last bit of log / sincos / expm1, i.e. ~1e-15
relative per ray.  Per-cell phi is rounded to float at the end (as the
reference's Result.phiAse), so replayed cells agree to a few float ulps; a ray
that passes within ~1e-15 of a cell edge may take the other (equally valid)
side on one of the two, so a handful of cells may differ by one ray's share.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN, legacy_mesh

pytestmark = pytest.mark.gpu


def _fixture(name="true_cladding", absorption=None):
    from haseongpu_b200 import TetMesh

    return TetMesh.fromFixture(GOLDEN / f"tet4_{name}.npz", claddingAbsorption=absorption)


def _spectrum():
    d = np.load(GOLDEN / "tet4_true_cladding.npz")
    return [float(d["sigmaA"])], [float(d["sigmaE"])]


def _ctx(mesh, sa, se):
    from haseongpu_b200 import TetDeviceMesh, build

    build.build_library()
    return TetDeviceMesh(mesh, sa, se, device=0)


def _random_rays(mesh, n, seed):
    rng = np.random.default_rng(seed)
    cells = rng.integers(0, mesh.numberOfCells, n).astype(np.uint32)
    P = mesh.points[mesh.cells[cells].astype(np.int64)]
    origin = np.einsum("nk,nkd->nd", rng.dirichlet(np.ones(4), n), P)
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    return cells, origin, u


@pytest.mark.parametrize("name", ["true_cladding", "cylindrical"])
def test_device_tables_equal_oracle_tables(oracle, name):
    mesh = _fixture(name)
    ref = oracle.tet_tables(mesh)
    with _ctx(mesh, *_spectrum()) as ctx:
        dev = ctx.tables()
    np.testing.assert_array_equal(dev["neighbors"], ref["neighbors"])
    np.testing.assert_array_equal(dev["neighborFace"], ref["neighborFace"])
    # the device keeps three planes per cell and rebuilds the fourth as
    # 1 - (sum of the others): equal to rounding
    scale = np.abs(ref["gradients"]).max()
    np.testing.assert_allclose(dev["planes"][:, :, :3], ref["gradients"], rtol=1e-12, atol=1e-12 * scale)
    np.testing.assert_array_equal(dev["volumes"], ref["volumes"])


def test_trace_matches_oracle_paths(oracle):
    mesh = _fixture(absorption=5.5)
    sa, se = _spectrum()
    cells, origin, u = _random_rays(mesh, 4096, 11)
    ref = oracle.tet_trace(mesh, (sa, se), cells, origin, u, max_segments=128)
    with _ctx(mesh, sa, se) as ctx:
        dev = ctx.trace(cells, origin, u, max_segments=128)
    np.testing.assert_array_equal(dev["status"], ref["status"])
    assert np.all(dev["status"] == 0)
    same = np.all(dev["cells"] == ref["cells"], axis=1) & (dev["segments"] == ref["segments"])
    assert same.mean() >= 0.999, f"{(~same).sum()} of 4096 paths differ"
    np.testing.assert_allclose(dev["lnGain"][same], ref["lnGain"][same], rtol=1e-11, atol=1e-12)
    np.testing.assert_allclose(dev["endPoint"][same], ref["endPoint"][same], rtol=0, atol=1e-12)
    np.testing.assert_allclose(dev["lengths"][same], ref["lengths"][same], rtol=0, atol=1e-12)


def test_trace_reference_edge_cases():
    """tests/forwardRayTraversal.cpp:156-256 on the device: the 30-tet vertex
    fan and perpendicular incidence."""
    from haseongpu_b200 import TetMesh

    pts = [(0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, -1.0)]
    pts += [(np.cos(2 * np.pi * k / 15), np.sin(2 * np.pi * k / 15), 0.0) for k in range(15)]
    cells = [(0, 1, 3 + k, 3 + (k + 1) % 15) for k in range(15)]
    cells += [(0, 2, 3 + (k + 1) % 15, 3 + k) for k in range(15)]
    fan = TetMesh(np.array(pts), np.array(cells), np.full(30, 0.1), 1e20, 1e-3)
    o = fan.points[1] * 0.2 + fan.points[3] * 0.1 + fan.points[4] * 0.3
    with _ctx(fan, [1e-21], [2e-20]) as ctx:
        r = ctx.trace([0], o, -o / np.linalg.norm(o))
    n = int(r["segments"][0])
    assert r["status"][0] == 0 and r["cells"][0, 0] == 0
    assert r["cells"][0, n - 1] == 23 and r["lengths"][0, n - 1] > 0.0
    assert r["lengths"][0, 0] == pytest.approx(np.linalg.norm(o), rel=1e-12)

    pts2 = np.array([(-1.0, 0, 0), (0.0, 0, 0), (0.0, 1, 0), (0.0, 0, 1), (1.0, 0, 0)])
    two = TetMesh(pts2, np.array([(0, 1, 2, 3), (4, 1, 3, 2)]), np.full(2, 0.1), 1e20, 1e-3)
    with _ctx(two, [1e-21], [2e-20]) as ctx:
        r = ctx.trace([0], [-0.4, 0.2, 0.2], [1.0, 0.0, 0.0])
    assert r["status"][0] == 0 and r["segments"][0] == 2
    np.testing.assert_array_equal(r["cells"][0, :2], [0, 1])
    np.testing.assert_allclose(r["lengths"][0, :2], [0.4, 0.6], rtol=1e-14)


def _replay_compare(dev, ref, *, quantile_tol=1e-5):
    rel = np.abs(dev.phiAse.astype(np.float64) / ref["phiAse"] - 1.0)
    assert np.quantile(rel, 0.999) < quantile_tol, np.sort(rel)[-10:]
    assert rel.max() < 2e-2, np.sort(rel)[-10:]
    differ = dev.totalRays != ref["rayVisits"]
    assert differ.mean() < 2e-3
    np.testing.assert_array_equal(dev.droppedRays, ref["droppedRays"])


@pytest.mark.parametrize("absorption", [0.0, 5.5, 55.0])
def test_calc_replays_the_oracle(oracle, absorption):
    mesh = _fixture(absorption=absorption)
    sa, se = _spectrum()
    ref = oracle.forward_phi_ase(mesh, (sa, se), minRays=400_000, seed=21)
    with _ctx(mesh, sa, se) as ctx:
        dev = ctx.calc_phi_ase(forwardRayCount=400_000, rngSeed=21)
    _replay_compare(dev, ref)
    np.testing.assert_allclose(dev.relativeStandardError, ref["relativeStandardError"], rtol=1e-3)
    np.testing.assert_allclose(dev.dndtAse, ref["dndtAse"], rtol=1e-5, atol=0)
    assert dev.raysTraced == 400_000 and dev.passes == 1
    assert dev.crossings == int(dev.totalRays.sum())


@pytest.mark.parametrize("mode", ["global", "shared"])
def test_tally_modes_agree(mode):
    mesh = _fixture(absorption=5.5)
    sa, se = _spectrum()
    with _ctx(mesh, sa, se) as ctx:
        a = ctx.calc_phi_ase(forwardRayCount=200_000, rngSeed=5, tallyMode=mode)
        b = ctx.calc_phi_ase(forwardRayCount=200_000, rngSeed=5, tallyMode="global")
    assert a.tallyMode == (2 if mode == "shared" else 1)
    np.testing.assert_allclose(a.phiAse, b.phiAse, rtol=1e-6)
    np.testing.assert_array_equal(a.totalRays, b.totalRays)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_reference_tet4_integrals(k):
    """Volume integrals of the reference's current Tet4 run (true-cladding README)."""
    d = np.load(GOLDEN / "tet4_true_cladding.npz")
    mesh = _fixture(absorption=float(d["claddingAbsorptions"][k]))
    with _ctx(mesh, *_spectrum()) as ctx:
        r = ctx.calc_phi_ase(forwardRayCount=4_000_000, rngSeed=99)
    V = mesh.cellVolumes()
    clad = mesh.claddingMask()
    pv = r.phiAse.astype(np.float64) * V
    ref = d["currentIntegrals"][k]
    assert pv.sum() == pytest.approx(ref[0], rel=3e-3)
    assert pv[~clad].sum() == pytest.approx(ref[1], rel=3e-3)
    assert pv[clad].sum() == pytest.approx(ref[2], rel=1e-2)
    assert int(r.droppedRays.sum()) == 0


@pytest.mark.parametrize("radius,gain", [(1.0, 2.0), (0.25, 16.0), (4.0, 1.2)])
def test_analytic_sphere_centre(radius, gain):
    """tests/python/phiAse/test_analyticalSphere.py: rtol 0.05 at the centre."""
    from haseongpu_b200 import TetMesh
    from haseongpu_b200.tetmesh import analytic_sphere_centre, beta_from_gain

    nTot, sa, se, tau = 1.38e20, 0.11e-20, 2.1e-20, 9.41e-4
    beta = beta_from_gain(gain, nTot, sa, se)
    mesh = TetMesh.ball(radius, 20, beta, nTot, tau)
    with _ctx(mesh, [sa], [se]) as ctx:
        r = ctx.calc_phi_ase(forwardRayCount=2_000_000, rngSeed=1234)
    centre = mesh.numberOfPoints // 2
    near = np.any(mesh.cells == centre, axis=1)
    V = mesh.cellVolumes()
    numerical = np.sum(r.phiAse[near] * V[near]) / V[near].sum()
    assert r.totalRays[near].min() > 0
    assert numerical == pytest.approx(analytic_sphere_centre(gain, radius, beta, nTot, tau), rel=0.05)


def test_adaptive_launches_match_oracle(oracle):
    mesh = _fixture(absorption=5.5)
    sa, se = _spectrum()
    kw = dict(minRays=20_000, maxRays=320_000, adaptiveSteps=4, rseThreshold=1e-9, seed=3)
    ref = oracle.forward_phi_ase(mesh, (sa, se), **kw)
    with _ctx(mesh, sa, se) as ctx:
        dev = ctx.calc_phi_ase(forwardRayCount=20_000, maxRays=320_000, adaptiveSteps=4,
                               relativeStandardErrorThreshold=1e-9, rngSeed=3)
        easy = ctx.calc_phi_ase(forwardRayCount=20_000, maxRays=320_000, adaptiveSteps=4,
                                relativeStandardErrorThreshold=10.0, rngSeed=3)
    assert dev.passes == ref["launches"] == 5 and dev.raysTraced == 320_000
    _replay_compare(dev, ref)
    assert dev.unconvergedSamples == mesh.numberOfCells
    assert easy.passes == 1 and easy.raysTraced == 20_000 and easy.unconvergedSamples == 0


def test_polychromatic_replay(oracle):
    mesh = _fixture(absorption=5.5)
    sa, se = [5e-21, 3e-21, 1e-21], [1e-20, 2e-20, 5e-21]
    ref = oracle.forward_phi_ase(mesh, (sa, se), minRays=300_000, seed=8)
    with _ctx(mesh, sa, se) as ctx:
        dev = ctx.calc_phi_ase(forwardRayCount=300_000, rngSeed=8)
        mono = ctx.calc_phi_ase(forwardRayCount=300_000, rngSeed=8, monochromatic=True)
    _replay_compare(dev, ref)
    mref = oracle.forward_phi_ase(mesh, (sa[:1], se[:1]), minRays=300_000, seed=8)
    _replay_compare(mono, mref)


def test_update_beta_matches_fresh_context():
    mesh = _fixture(absorption=5.5)
    sa, se = _spectrum()
    beta2 = np.clip(mesh.betaVolume * 1.5, 0, 1)
    with _ctx(mesh, sa, se) as ctx:
        ctx.update_beta(beta2)
        a = ctx.calc_phi_ase(forwardRayCount=200_000, rngSeed=4)
    with _ctx(mesh.withBeta(beta2), sa, se) as ctx:
        b = ctx.calc_phi_ase(forwardRayCount=200_000, rngSeed=4)
    np.testing.assert_allclose(a.phiAse, b.phiAse, rtol=1e-6)


def test_phiase_forward_front_end_on_prism_twin(oracle):
    """PhiASE(propagationMode='forward') on a PrismMesh runs its Tet4 twin."""
    from haseongpu_b200 import CrossSectionData, PhiASE, TetMesh

    prism = legacy_mesh("cylindrical")
    d = np.load(GOLDEN / "legacy_cylindrical.npz")
    spectra = CrossSectionData.monochromatic(wavelength=905e-9, crossSectionAbsorption=float(d["sigmaA"]),
                                             crossSectionEmission=float(d["sigmaE"]))
    p = PhiASE(forwardRayCount=300_000, monochromatic=True, rngSeed=17)
    res = p.run(gainMedium=prism, crossSections=spectra).getResults()
    tet = TetMesh.fromPrismMesh(prism)
    assert res.phiAse.shape == (tet.numberOfCells,)
    ref = oracle.forward_phi_ase(tet, ([float(d["sigmaA"])], [float(d["sigmaE"])]), minRays=300_000, seed=17)
    _replay_compare(res, ref)
    np.testing.assert_allclose(res.standardError, res.relativeStandardError * res.phiAse, rtol=1e-6)
