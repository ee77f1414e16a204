"""CPU pins of the forward Tet4 oracle (the checker of the forward GPU path).

- Tet4 topology against the reference's own builder
  (pyInclude/geometry/volume.py:_deriveTet4Topology, golden tet4_tables.npz).
- Traversal edge cases of the reference's tests/forwardRayTraversal.cpp:156-256
  (a ray through a vertex shared by 30 tets; perpendicular incidence).
- Volume integrals of the reference's current Tet4 run on the true-cladding
  disc (tests/data/laserPumpCladding/true_cladding_no_reflection_phiase_reference/README.md).
- The analytic sphere centre of tests/python/phiAse/test_analyticalSphere.py.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN
from haseongpu_b200.tetmesh import TetMesh, analytic_sphere_centre, beta_from_gain


def _fixture_mesh(name="true_cladding", absorption=None):
    return TetMesh.fromFixture(GOLDEN / f"tet4_{name}.npz", claddingAbsorption=absorption)


def _fan_mesh():
    pts = [(0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, 0.0, -1.0)]
    pts += [(np.cos(2 * np.pi * k / 15), np.sin(2 * np.pi * k / 15), 0.0) for k in range(15)]
    cells = [(0, 1, 3 + k, 3 + (k + 1) % 15) for k in range(15)]
    cells += [(0, 2, 3 + (k + 1) % 15, 3 + k) for k in range(15)]
    return TetMesh(np.array(pts), np.array(cells), np.full(30, 0.1), 1e20, 1e-3)


@pytest.mark.parametrize("name", ["true_cladding", "cylindrical"])
def test_tet_tables_match_reference_builder(oracle, name):
    mesh = _fixture_mesh(name)
    ours = oracle.tet_tables(mesh)
    ref = np.load(GOLDEN / "tet4_tables.npz")
    fv = ref["faceVertices"]
    # reference local face j holds vertices fv[j]; ours: face f is opposite vertex f
    opposite = np.array([({0, 1, 2, 3} - set(map(int, row))).pop() for row in fv])
    nbr_ref = ref[f"{name}_neighborCells"]
    nface_ref = ref[f"{name}_neighborLocalFaces"]
    exp_nbr = np.empty_like(nbr_ref)
    exp_face = np.empty_like(nface_ref)
    exp_nbr[:, opposite] = nbr_ref
    exp_face[:, opposite] = np.where(nface_ref >= 0, opposite[np.maximum(nface_ref, 0)], -1)
    np.testing.assert_array_equal(ours["neighbors"], exp_nbr)
    np.testing.assert_array_equal(ours["neighborFace"], exp_face)
    np.testing.assert_allclose(ours["volumes"], ref[f"{name}_cellVolumes"], rtol=1e-6)
    # barycentric gradients: lambda_f(v_k) = delta_fk
    P = mesh.points[mesh.cells.astype(np.int64)]
    lam = 1.0 * (np.arange(4)[:, None] == 0) + np.einsum("cfd,ckd->cfk", ours["gradients"], P - P[:, :1])
    np.testing.assert_allclose(lam, np.broadcast_to(np.eye(4), lam.shape), atol=1e-9)


def test_true_cladding_volumes_match_readme(oracle):
    """648 cladding cells of 3.615535851812808 cm^3 in 19.566038838161607 cm^3 (README.md:17-24)."""
    mesh = _fixture_mesh()
    V = oracle.tet_tables(mesh)["volumes"]
    clad = mesh.claddingMask()
    assert int(clad.sum()) == 648
    assert V.sum() == pytest.approx(19.566038838161607, rel=1e-12)
    assert V[clad].sum() == pytest.approx(3.615535851812808, rel=1e-12)


def test_traversal_through_vertex_shared_by_30_tets(oracle):
    """tests/forwardRayTraversal.cpp:156-215: the ray aimed at the shared vertex
    continues into cell 23 on the far side with positive length."""
    mesh = _fan_mesh()
    pts = mesh.points
    origin = pts[1] * 0.2 + pts[3] * 0.1 + pts[4] * 0.3
    u = -origin / np.linalg.norm(origin)
    r = oracle.tet_trace(mesh, ([1e-21], [2e-20]), [0], origin, u)
    n = int(r["segments"][0])
    cells, lengths = r["cells"][0, :n], r["lengths"][0, :n]
    assert r["status"][0] == 0
    assert cells[0] == 0
    assert lengths[0] == pytest.approx(np.linalg.norm(origin), rel=1e-12)
    assert cells[-1] == 23 and lengths[-1] > 0.0
    assert np.all(lengths[1:-1] < 1e-14)  # zero-length steps around the vertex only
    assert lengths.sum() == pytest.approx(np.linalg.norm(origin) + np.linalg.norm(r["endPoint"][0]), rel=1e-12)


def test_traversal_perpendicular_incidence(oracle):
    """tests/forwardRayTraversal.cpp:217-256: two tets sharing the x = 0 plane."""
    pts = np.array([(-1.0, 0, 0), (0.0, 0, 0), (0.0, 1, 0), (0.0, 0, 1), (1.0, 0, 0)])
    mesh = TetMesh(pts, np.array([(0, 1, 2, 3), (4, 1, 3, 2)]), np.full(2, 0.1), 1e20, 1e-3)
    tab = oracle.tet_tables(mesh)
    assert tab["neighbors"][0, 0] == 1 and tab["neighborFace"][0, 0] == 0
    r = oracle.tet_trace(mesh, ([1e-21], [2e-20]), [0], [-0.4, 0.2, 0.2], [1.0, 0.0, 0.0])
    assert r["status"][0] == 0 and r["segments"][0] == 2
    np.testing.assert_array_equal(r["cells"][0, :2], [0, 1])
    np.testing.assert_allclose(r["lengths"][0, :2], [0.4, 0.6], rtol=1e-14)
    np.testing.assert_allclose(r["endPoint"][0], [0.6, 0.2, 0.2], rtol=1e-14)


def test_trace_ln_gain_is_g_times_chord(oracle):
    """Uniform beta: ln gain = g * (chord length inside the mesh)."""
    mesh = _fixture_mesh(absorption=0.0)
    mesh = mesh.withBeta(np.full(mesh.numberOfCells, 0.3))
    mesh.claddingCellTypes = None
    sa, se = 5e-21, 1e-20
    rng = np.random.default_rng(4)
    cells = rng.integers(0, mesh.numberOfCells, 64).astype(np.uint32)
    P = mesh.points[mesh.cells[cells].astype(np.int64)]
    w = rng.dirichlet(np.ones(4), 64)
    origin = np.einsum("nk,nkd->nd", w, P)
    u = rng.normal(size=(64, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    r = oracle.tet_trace(mesh, ([sa], [se]), cells, origin, u, max_segments=256)
    assert np.all(r["status"] == 0)
    g = mesh.nTot * (0.3 * (sa + se) - sa)
    chord = np.einsum("nd,nd->n", r["endPoint"] - origin, u)
    np.testing.assert_allclose(r["lnGain"], g * chord, rtol=1e-10)
    np.testing.assert_allclose(r["lengths"].sum(axis=1), chord, rtol=1e-10)


@pytest.mark.parametrize("k", [0, 1, 2])
def test_forward_oracle_matches_reference_tet4_integrals(oracle, k):
    """Volume integrals sum(phi V) of the reference's current Tet4 run (README
    'current Tet4' table), total / gain / cladding, for absorption 0, 5.5, 55."""
    d = np.load(GOLDEN / "tet4_true_cladding.npz")
    mesh = _fixture_mesh(absorption=float(d["claddingAbsorptions"][k]))
    r = oracle.forward_phi_ase(mesh, ([float(d["sigmaA"])], [float(d["sigmaE"])]), minRays=1_000_000, seed=7)
    V = mesh.cellVolumes()
    clad = mesh.claddingMask()
    pv = r["phiAse"] * V
    total, gain, cl = pv.sum(), pv[~clad].sum(), pv[clad].sum()
    ref = d["currentIntegrals"][k]
    assert total == pytest.approx(ref[0], rel=5e-3)
    assert gain == pytest.approx(ref[1], rel=5e-3)
    assert cl == pytest.approx(ref[2], rel=1.5e-2)
    assert r["droppedRays"].sum() == 0
    assert r["totalRays"] == 1_000_000 and r["launches"] == 1
    assert np.all(r["rayVisits"] > 0)
    # dndt = (beta (sE + sA) - sA) phi (include/core/forwardPhiAseUtilities.hpp:16-25)
    sa, se = float(d["sigmaA"]), float(d["sigmaE"])
    np.testing.assert_allclose(r["dndtAse"], (mesh.betaVolume * (se + sa) - sa) * r["phiAse"], rtol=1e-15)


@pytest.mark.parametrize("radius,gain", [(1.0, 2.0), (0.25, 16.0), (4.0, 1.2)])
def test_forward_oracle_analytic_sphere_centre(oracle, radius, gain):
    nTot, sa, se, tau = 1.38e20, 0.11e-20, 2.1e-20, 9.41e-4
    beta = beta_from_gain(gain, nTot, sa, se)
    mesh = TetMesh.ball(radius, 20, beta, nTot, tau)
    r = oracle.forward_phi_ase(mesh, ([sa], [se]), minRays=1_000_000, seed=1234)
    centre = mesh.numberOfPoints // 2
    assert np.allclose(mesh.points[centre], 0.0)
    near = np.any(mesh.cells == centre, axis=1)
    V = mesh.cellVolumes()
    numerical = np.sum(r["phiAse"][near] * V[near]) / V[near].sum()
    expected = analytic_sphere_centre(gain, radius, beta, nTot, tau)
    assert numerical == pytest.approx(expected, rel=0.05)


def test_forward_oracle_is_deterministic_and_thread_independent(oracle):
    mesh = _fixture_mesh(absorption=5.5)
    spec = ([5e-21], [1e-20])
    a = oracle.forward_phi_ase(mesh, spec, minRays=100_000, seed=3, threads=1)
    b = oracle.forward_phi_ase(mesh, spec, minRays=100_000, seed=3, threads=4)
    c = oracle.forward_phi_ase(mesh, spec, minRays=100_000, seed=4, threads=4)
    np.testing.assert_allclose(a["phiAse"], b["phiAse"], rtol=1e-6)  # FP64 sum order, then float phi
    np.testing.assert_array_equal(a["rayVisits"], b["rayVisits"])
    assert not np.array_equal(a["phiAse"], c["phiAse"])


def test_forward_oracle_adaptive_launches(oracle):
    """include/core/forwardPhiAseEvaluator.hpp:114-178: rays of a launch add to
    the previous ones; stop when every cell meets the threshold or at maxRays."""
    mesh = _fixture_mesh(absorption=5.5)
    spec = ([5e-21], [1e-20])
    r = oracle.forward_phi_ase(mesh, spec, minRays=20_000, maxRays=320_000, adaptiveSteps=4, rseThreshold=1e-9,
                               seed=3)
    assert r["launches"] == 5 and r["totalRays"] == 320_000
    one = oracle.forward_phi_ase(mesh, spec, minRays=320_000, seed=3)
    assert np.median(r["relativeStandardError"]) == pytest.approx(np.median(one["relativeStandardError"]), rel=0.1)
    easy = oracle.forward_phi_ase(mesh, spec, minRays=20_000, maxRays=320_000, adaptiveSteps=4, rseThreshold=10.0,
                                  seed=3)
    assert easy["launches"] == 1 and easy["totalRays"] == 20_000


def test_forward_oracle_polychromatic_stratified_wavelengths(oracle):
    """Two identical spectral pairs give the monochromatic answer (stratified
    wavelength bins, include/kernels/forward/volumeSampling.hpp:19-32)."""
    mesh = _fixture_mesh(absorption=5.5)
    one = oracle.forward_phi_ase(mesh, ([5e-21], [1e-20]), minRays=200_000, seed=9)
    two = oracle.forward_phi_ase(mesh, ([5e-21, 5e-21], [1e-20, 1e-20]), minRays=200_000, seed=9)
    np.testing.assert_array_equal(one["phiAse"], two["phiAse"])


def test_prism_to_tet4_split_is_conforming(oracle):
    """Tet4 twin of a prism mesh: every inner face is shared by exactly two
    cells; boundary faces are the top and bottom triangles plus two per side
    quad; volumes add up to the prism volumes."""
    from conftest import legacy_mesh

    prism = legacy_mesh("cylindrical")
    tet = TetMesh.fromPrismMesh(prism)
    tab = oracle.tet_tables(tet)  # raises if a face is shared by more than two cells
    T, L = prism.numberOfTriangles, prism.numberOfLevels
    edges = np.sort(np.concatenate([prism.triangles[:, [0, 1]], prism.triangles[:, [1, 2]],
                                    prism.triangles[:, [2, 0]]]), axis=1)
    _, counts = np.unique(edges, axis=0, return_counts=True)
    boundary_edges = int((counts == 1).sum())
    assert int((tab["neighbors"] < 0).sum()) == 2 * T + 2 * boundary_edges * (L - 1)
    np.testing.assert_allclose(tab["volumes"].reshape(-1, 3).sum(axis=1), prism.prismVolumes(), rtol=1e-10)
