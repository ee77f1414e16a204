"""CPU tests of the prism walk records (hase_mesh_tables, built on the host).

The walks rely on two properties of these records instead of testing for
them per crossing:

* the two triangles of an edge store exactly negated normals, so the entry
  edge's dd is exactly minus the dd > 0 it was chosen with and fails the
  dd > 0 test;
* in the walks' copy a mesh-boundary edge has NaN normals, so it fails the
  same test.

Both are checked here on the legacy fixtures and on the seeded workload
meshes, with and without consistently oriented triangles, together with
the neighbour codes (the neighbour of an edge's neighbour is the edge)."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import legacy_mesh


def _records(native, mesh):
    from haseongpu_b200 import _native as N

    pts = np.ascontiguousarray(mesh.points, np.float64)
    tri = np.ascontiguousarray(mesh.triangles, np.uint32)
    T = tri.shape[0]
    desc = N.MeshDesc(mesh.numberOfPoints, T, mesh.numberOfLevels, N.ptr(pts, N._f64p), N.ptr(tri, N._u32p),
                      mesh.thickness, None, None, None, 0, 0.0, 1.0, 1.0, None, None)
    rec = np.zeros((T, 12), np.float32)
    walk = np.zeros((T, 12), np.float32)
    native.check(native.lib().hase_mesh_tables(C.byref(desc), rec.ctypes.data_as(C.POINTER(C.c_float)),
                                               walk.ctypes.data_as(C.POINTER(C.c_float))))
    return rec, walk


def _meshes():
    from haseongpu_b200.configs import disc_poly, disc_small

    out = [("cuboid", legacy_mesh("cuboid")), ("cylindrical", legacy_mesh("cylindrical")),
           ("disc_small", disc_small().mesh), ("disc_poly", disc_poly().mesh)]
    # the cylinder with every other triangle's vertex order reversed
    m = legacy_mesh("cylindrical")
    flipped = m.triangles.copy()
    flipped[::2] = flipped[::2, ::-1]
    m.triangles = flipped
    out.append(("cylindrical, mixed orientation", m))
    return out


NX, NY, C0, NB = (0, 3, 6), (1, 4, 7), (2, 5, 8), (9, 10, 11)


@pytest.mark.parametrize("name,mesh", _meshes(), ids=lambda v: v if isinstance(v, str) else "")
def test_shared_edges_store_exactly_negated_normals(native, name, mesh):
    rec, walk = _records(native, mesh)
    T = rec.shape[0]
    nb = rec[:, 9:12].copy().view(np.int32)
    shared = boundary = 0
    for t in range(T):
        for e in range(3):
            code = int(nb[t, e])
            if code < 0:
                boundary += 1
                assert np.isnan(walk[t, NX[e]]) and np.isnan(walk[t, NY[e]]), (t, e)
                assert walk[t, C0[e]] == rec[t, C0[e]]
                continue
            u, f = code >> 2, code & 3
            assert int(nb[u, f]) == (t << 2 | e), (t, e)
            # exact negation, bit for bit
            assert rec[u, NX[f]] == -rec[t, NX[e]] and rec[u, NY[f]] == -rec[t, NY[e]], (t, e, u, f)
            assert walk[t, NX[e]] == rec[t, NX[e]] and walk[t, NY[e]] == rec[t, NY[e]]
            shared += 1
    assert shared > 0 and boundary > 0
    # the copy differs from the records only in the boundary normals (columns
    # 9..11 are the neighbour codes, -1 reads as a NaN float there)
    assert np.array_equal(walk[:, 9:].view(np.int32), rec[:, 9:].view(np.int32))
    geo_w, geo_r = walk[:, :9], rec[:, :9]
    same = ~np.isnan(geo_w)
    assert np.array_equal(geo_w[same], geo_r[same])
    assert np.isnan(geo_w).sum() == 2 * boundary and not np.isnan(geo_r).any()


def test_entry_edge_fails_the_exit_test(native):
    """dd = -(n . u) of the edge a walk entered through is exactly minus the
    dd > 0 of the same edge in the triangle it left, for FP32 directions."""
    mesh = legacy_mesh("cylindrical")
    rec, _ = _records(native, mesh)
    nb = rec[:, 9:12].copy().view(np.int32)
    rng = np.random.default_rng(3)
    f32 = np.float32
    checked = 0
    for _ in range(2000):
        t, e = int(rng.integers(rec.shape[0])), int(rng.integers(3))
        code = int(nb[t, e])
        if code < 0:
            continue
        u, f = code >> 2, code & 3
        a = rng.uniform(0, 2 * np.pi)
        ux, uy = f32(np.cos(a)), f32(np.sin(a))
        dd_out = -np.float32(np.float32(rec[t, NX[e]] * ux) + np.float32(rec[t, NY[e]] * uy))
        dd_in = -np.float32(np.float32(rec[u, NX[f]] * ux) + np.float32(rec[u, NY[f]] * uy))
        assert dd_in == -dd_out
        if dd_out > 0:
            assert not dd_in > 0
        checked += 1
    assert checked > 1000


def test_mesh_tables_rejects_missing_arrays(native):
    from haseongpu_b200 import _native as N

    desc = N.MeshDesc()
    assert native.lib().hase_mesh_tables(C.byref(desc), None, None) == native.HASE_INVALID_ARGUMENT
