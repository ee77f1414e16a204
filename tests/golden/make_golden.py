#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden from the HASEonGPU reference tree.

This script is run once, in a container where the reference checkout is mounted
at ``/root/reference`` (override with ``--reference``).  It never runs on the
GPU machine; the tests only read the ``.npz`` files it writes.

What it extracts (all citations are paths inside the reference project):

* ``legacy_cuboid.npz`` / ``legacy_cylindrical.npz`` -- the legacy prism
  (wedge) geometry of ``example/data/cuboid.vtk`` / ``cylindrical.vtk``
  (Tet4 files, regrouped into wedges with the reference's own
  ``utils/convert_vtk_topology.py:_wedge_from_tetrahedra``), their
  ``betaVolume`` / ``betaCells`` / material attributes, the first
  (sigma_a, sigma_e) pair of ``example/input/sigma_{a,e}.txt`` and the legacy
  serial phi-ASE / dndt-ASE point buffers of
  ``tests/data/compareSerial/phiase_reference.npz`` (1e6 rays per sample,
  monochromatic, no reflections; ``tests/data/compareSerial/README.md``).
* ``legacy_true_cladding.npz`` -- the 421-point x 10-level disc with a cladding
  ring, and the legacy backward-method phi-ASE / MSE / totalRays at 2,000 rays
  per sample for cladding absorption 0, 5.5 and 55 cm^-1
  (``tests/data/laserPumpCladding/true_cladding_no_reflection_phiase_reference``).
  N_tot and the fluorescence lifetime are not stored in that archive; the
  medium it was generated from (``example/laserPumpCladdingApi.py:240-241``)
  uses N_tot = 2 * 1.388e20 cm^-3 and tau = 9.41e-4 s.
* ``tet4_true_cladding.npz`` -- the Tet4 twin of that disc
  (``example/data/ptTet4.vtk``, three tetrahedra per wedge) with the cladding
  tags and beta of the true-cladding run, and the reference's own forward
  Tet4 volume integrals (total / gain / cladding for absorption 0, 5.5,
  55 cm^-1) parsed from the table in that fixture's README.md.
* ``tet4_cylindrical.npz`` -- ``example/data/cylindrical.vtk`` as Tet4 cells
  with its per-cell betaVolume and material attributes.
* ``tet4_tables.npz`` -- the reference's own Tet4 topology
  (``pyInclude/geometry/volume.py:_deriveTet4Topology``: neighbour cells,
  neighbour local faces and cell volumes, with its local-face table
  ``TET4_FACE_VERTICES``) for the two Tet4 fixtures above.
* ``mesh_tables.npz`` -- the reference's own per-triangle tables
  (``pyInclude/geometry/core.py:_derived_topology``: centres, surfaces, edge
  normals, normal points, neighbours, forbidden edges) for the three meshes
  above plus the reference Bowyer-Watson triangulation
  (``pyInclude/geometry/core.py:_delaunay``) of a small seeded point set.
"""

from __future__ import annotations

import argparse
import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _load_module(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def _wedges_from_vtk(ref: Path, vtk_name: str):
    vtk = _load_module(ref / "pyInclude" / "geometry" / "vtk.py", "_ref_vtk")
    conv = _load_module(ref / "utils" / "convert_vtk_topology.py", "_ref_conv")
    points, cells, cell_types, point_data, cell_data, fields = vtk._parseVtk(ref / "example" / "data" / vtk_name)
    tets = np.asarray(cells, dtype=np.uint32)
    assert tets.shape[1] == 4 and tets.shape[0] % 3 == 0
    wedges = np.asarray([conv._wedge_from_tetrahedra(points, g) for g in tets.reshape(-1, 3, 4)], dtype=np.uint32)
    return np.asarray(points, np.float64), wedges, point_data, cell_data, fields


def _prism_layout(points3, wedges, n_points, n_levels, thickness):
    """Map wedges to (triangle, level) with prism index = triangle + level * T."""
    base = wedges[:, :3]
    level_of = np.rint(points3[base[:, 0], 2] / thickness).astype(np.int64)
    n_wedges = wedges.shape[0]
    n_tri = n_wedges // (n_levels - 1)
    assert n_tri * (n_levels - 1) == n_wedges
    tri = (base % n_points).astype(np.uint32)
    triangles = tri[level_of == 0]
    assert triangles.shape[0] == n_tri
    key = {tuple(sorted(t)): i for i, t in enumerate(triangles.tolist())}
    prism_index = np.empty(n_wedges, np.int64)
    for w in range(n_wedges):
        t = key[tuple(sorted(tri[w].tolist()))]
        prism_index[w] = t + level_of[w] * n_tri
    assert np.array_equal(np.sort(prism_index), np.arange(n_wedges))
    return triangles, prism_index


def _legacy_compare_serial(ref: Path, name: str, out: Path):
    points3, wedges, point_data, cell_data, fields = _wedges_from_vtk(ref, f"{name}.vtk")
    n_points = int(np.asarray(fields["structuredNumberOfPoints"]).ravel()[0])
    n_levels = int(np.asarray(fields["structuredNumberOfLevels"]).ravel()[0])
    thickness = float(np.asarray(fields["structuredThickness"]).ravel()[0])
    triangles, prism_index = _prism_layout(points3, wedges, n_points, n_levels, thickness)
    n_tri = triangles.shape[0]

    def per_wedge(values):
        grouped = np.asarray(values).reshape(-1, 3, *np.asarray(values).shape[1:])
        assert np.all(grouped == grouped[:, :1]), "tet children of a wedge disagree"
        return grouped[:, 0]

    beta_w = per_wedge(cell_data["betaVolume"]).astype(np.float64)
    beta_volume = np.empty_like(beta_w)
    beta_volume[prism_index] = beta_w
    clad_w = per_wedge(fields["claddingCellTypes"]).astype(np.uint32)
    clad_p = np.empty_like(clad_w)
    clad_p[prism_index] = clad_w
    clad_tri = clad_p[:n_tri]
    assert np.all(clad_p.reshape(n_levels - 1, n_tri) == clad_tri[None, :])

    sigma_a = np.loadtxt(ref / "example" / "input" / "sigma_a.txt")
    sigma_e = np.loadtxt(ref / "example" / "input" / "sigma_e.txt")
    legacy = np.load(ref / "tests" / "data" / "compareSerial" / "phiase_reference.npz")
    np.savez_compressed(
        out,
        points2d=points3[:n_points, :2].copy(),
        triangles=triangles,
        numberOfLevels=np.uint32(n_levels),
        thickness=np.float64(thickness),
        betaVolume=beta_volume,
        betaCells=np.asarray(point_data["betaCells"], np.float64),
        claddingCellTypes=clad_tri,
        claddingNumber=np.uint32(np.asarray(fields["claddingNumber"]).ravel()[0]),
        claddingAbsorption=np.float64(np.asarray(fields["claddingAbsorption"]).ravel()[0]),
        nTot=np.float64(np.asarray(fields["nTot"]).ravel()[0]),
        crystalTFluo=np.float64(np.asarray(fields["crystalTFluo"]).ravel()[0]),
        refractiveIndices=np.asarray(fields["refractiveIndices"], np.float64),
        sigmaA=np.float64(sigma_a.ravel()[0]),
        sigmaE=np.float64(sigma_e.ravel()[0]),
        phiASE=legacy[f"{name}_phiASE"],
        dndtAse=legacy[f"{name}_dndtAse"],
        raysPerSample=np.uint32(1_000_000),
        provenance=np.asarray(json.dumps({
            "geometry": f"example/data/{name}.vtk",
            "legacyResult": "tests/data/compareSerial/phiase_reference.npz",
            "generator": "BaseVersionSerial, mt19937 seed 5489, 1e6 rays/sample, first spectral pair",
        })),
    )
    return points3[:n_points, :2].copy(), triangles


def _legacy_true_cladding(ref: Path, out: Path):
    path = ref / "tests" / "data" / "laserPumpCladding" / "true_cladding_no_reflection_phiase_reference" / "phiase_reference.npz"
    d = np.load(path)
    meta = json.loads(str(d["metadata"]))
    geo = meta["geometry"]
    n_points = geo["numberOfBasePoints"]
    n_tri = geo["numberOfBaseTriangles"]
    n_levels = geo["numberOfLevels"]
    points3 = d["points"]
    cells = d["cells"]
    triangles = cells[:n_tri, :3].astype(np.uint32)
    for level in range(n_levels - 1):
        assert np.array_equal(cells[level * n_tri:(level + 1) * n_tri, :3], triangles + level * n_points)
    thickness = float(points3[n_points, 2] - points3[0, 2])
    mat = meta["material"]
    np.savez_compressed(
        out,
        points2d=points3[:n_points, :2].copy(),
        triangles=triangles,
        numberOfLevels=np.uint32(n_levels),
        thickness=np.float64(thickness),
        betaVolume=d["wedgeBetaVolume"].astype(np.float64),
        betaCells=np.full(n_points * n_levels, mat["betaCells"], np.float64),
        claddingCellTypes=d["baseCladdingCellTypes"].astype(np.uint32),
        claddingNumber=np.uint32(mat["claddingNumber"]),
        claddingAbsorptions=np.asarray(mat["claddingAbsorptions"], np.float64),
        nTot=np.float64(2 * 1.388e20),
        crystalTFluo=np.float64(9.41e-4),
        sigmaA=np.float64(mat["crossSectionAbsorption"]),
        sigmaE=np.float64(mat["crossSectionEmission"]),
        phiASE=d["phiASE"],
        mse=d["mse"],
        totalRays=d["totalRays"],
        raysPerSample=np.uint32(meta["parameters"]["raysPerSample"]),
        provenance=np.asarray(json.dumps({
            "legacyResult": str(path.relative_to(ref)),
            "nTotAndTau": "example/laserPumpCladdingApi.py:240-241",
            "diagnostics": meta["diagnostics"],
        })),
    )
    return points3[:n_points, :2].copy(), triangles


def _readme_integrals(readme: Path):
    """Rows '| absorption | partition | legacy | current Tet4 | bias |' of the README table."""
    import re

    rows = []
    for line in readme.read_text(encoding="utf-8").splitlines():
        m = re.match(r"\|\s*([0-9.]+)\s*\|\s*(total|gain|cladding)\s*\|\s*([0-9.eE+-]+)\s*\|\s*([0-9.eE+-]+)\s*\|", line)
        if m:
            rows.append((float(m.group(1)), m.group(2), float(m.group(3)), float(m.group(4))))
    return rows


def _tet4_true_cladding(ref: Path, out: Path):
    vtk = _load_module(ref / "pyInclude" / "geometry" / "vtk.py", "_ref_vtk")
    points, cells, cell_types, point_data, cell_data, fields = vtk._parseVtk(ref / "example" / "data" / "ptTet4.vtk")
    tets = np.asarray(cells, dtype=np.uint32)
    base = ref / "tests" / "data" / "laserPumpCladding" / "true_cladding_no_reflection_phiase_reference"
    d = np.load(base / "phiase_reference.npz")
    meta = json.loads(str(d["metadata"]))
    wedge_types = d["wedgeCladdingCellTypes"].astype(np.uint32)
    tet_types = np.repeat(wedge_types, 3)
    assert tets.shape == (3 * wedge_types.size, 4)
    for wedge, children in zip(d["cells"], tets.reshape(-1, 3, 4)):
        assert np.array_equal(np.unique(children), np.sort(wedge))
    mat = meta["material"]
    beta = np.where(tet_types == mat["claddingNumber"], 0.0, mat["gainBetaVolume"])
    rows = _readme_integrals(base / "README.md")
    absorptions = np.asarray(mat["claddingAbsorptions"], np.float64)
    parts = ("total", "gain", "cladding")
    current = np.zeros((absorptions.size, 3))
    legacy = np.zeros((absorptions.size, 3))
    for a, part, leg, cur in rows:
        i = int(np.argmin(np.abs(absorptions - a)))
        current[i, parts.index(part)] = cur
        legacy[i, parts.index(part)] = leg
    assert np.all(current > 0)
    np.savez_compressed(
        out, points=np.asarray(points, np.float64), cells=tets, betaVolume=beta, claddingCellTypes=tet_types,
        claddingNumber=np.uint32(mat["claddingNumber"]), claddingAbsorptions=absorptions,
        nTot=np.float64(2 * 1.388e20), crystalTFluo=np.float64(9.41e-4),
        sigmaA=np.float64(mat["crossSectionAbsorption"]), sigmaE=np.float64(mat["crossSectionEmission"]),
        currentIntegrals=current, legacyIntegrals=legacy, partitions=np.asarray(parts),
        provenance=np.asarray(json.dumps({
            "geometry": "example/data/ptTet4.vtk",
            "integrals": str((base / "README.md").relative_to(ref)),
            "note": "current Tet4 = the reference's forward estimator, no reflections, monochromatic",
        })))


def _tet4_from_vtk(ref: Path, name: str, out: Path):
    vtk = _load_module(ref / "pyInclude" / "geometry" / "vtk.py", "_ref_vtk")
    points, cells, cell_types, point_data, cell_data, fields = vtk._parseVtk(ref / "example" / "data" / f"{name}.vtk")
    sigma_a = np.loadtxt(ref / "example" / "input" / "sigma_a.txt")
    sigma_e = np.loadtxt(ref / "example" / "input" / "sigma_e.txt")
    np.savez_compressed(
        out, points=np.asarray(points, np.float64), cells=np.asarray(cells, np.uint32),
        betaVolume=np.asarray(cell_data["betaVolume"], np.float64),
        claddingCellTypes=np.asarray(fields["claddingCellTypes"], np.uint32),
        claddingNumber=np.uint32(np.asarray(fields["claddingNumber"]).ravel()[0]),
        claddingAbsorption=np.float64(np.asarray(fields["claddingAbsorption"]).ravel()[0]),
        nTot=np.float64(np.asarray(fields["nTot"]).ravel()[0]),
        crystalTFluo=np.float64(np.asarray(fields["crystalTFluo"]).ravel()[0]),
        sigmaA=np.float64(sigma_a.ravel()[0]), sigmaE=np.float64(sigma_e.ravel()[0]),
        provenance=np.asarray(json.dumps({"geometry": f"example/data/{name}.vtk"})))


def _tet4_tables(ref: Path, fixtures, out: Path):
    sys.path.insert(0, str(ref))
    from pyInclude.geometry import volume  # noqa: PLC0415  (reference frontend, importable here)

    payload = {"faceVertices": np.asarray(volume.TET4_FACE_VERTICES, np.int32)}
    for name, path in fixtures.items():
        d = np.load(path)
        topo = volume._deriveTet4Topology(np.asarray(d["points"], np.float64), np.asarray(d["cells"], np.int64), None)
        payload[f"{name}_neighborCells"] = np.asarray(topo["neighborCells"], np.int32)
        payload[f"{name}_neighborLocalFaces"] = np.asarray(topo["neighborLocalFaces"], np.int32)
        payload[f"{name}_cellVolumes"] = np.asarray(topo["cellVolumes"], np.float32)
    np.savez_compressed(out, **payload)


def _mesh_tables(ref: Path, meshes, out: Path):
    sys.path.insert(0, str(ref))
    from pyInclude.geometry import core  # noqa: PLC0415  (reference frontend, importable here)

    payload = {}
    for name, (pts, tris) in meshes.items():
        tables = core._derived_topology(np.ascontiguousarray(pts), np.ascontiguousarray(tris))
        payload[f"{name}_points2d"] = pts
        payload[f"{name}_triangles"] = tris
        for key, value in tables.items():
            payload[f"{name}_{key}"] = np.asarray(value)
    rng = np.random.default_rng(20261203)
    small = rng.uniform(-1.0, 1.0, size=(40, 2))
    small_pts, small_tris = core._delaunay(small)
    payload["delaunay_points2d"] = small_pts
    payload["delaunay_triangles"] = small_tris
    tables = core._derived_topology(np.ascontiguousarray(small_pts), np.ascontiguousarray(small_tris))
    for key, value in tables.items():
        payload[f"delaunay_{key}"] = np.asarray(value)
    np.savez_compressed(out, **payload)


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", type=Path, default=Path("/root/reference"))
    args = parser.parse_args(argv)
    ref = args.reference
    meshes = {}
    for name in ("cuboid", "cylindrical"):
        meshes[name] = _legacy_compare_serial(ref, name, HERE / f"legacy_{name}.npz")
    meshes["true_cladding"] = _legacy_true_cladding(ref, HERE / "legacy_true_cladding.npz")
    _tet4_true_cladding(ref, HERE / "tet4_true_cladding.npz")
    _tet4_from_vtk(ref, "cylindrical", HERE / "tet4_cylindrical.npz")
    _tet4_tables(ref, {"true_cladding": HERE / "tet4_true_cladding.npz",
                       "cylindrical": HERE / "tet4_cylindrical.npz"}, HERE / "tet4_tables.npz")
    _mesh_tables(ref, meshes, HERE / "mesh_tables.npz")
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
