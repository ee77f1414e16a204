"""CPU tests of the boundary and the host logic (no compute call needs a GPU).

* libhase_b200.so builds for sm_100a, loads, and exports every symbol
  include/hase_b200.h declares; the ctypes structures match the header.
* Without a device the entry points fail loudly with HASE_NO_DEVICE (no CPU fallback).
* Spectral resampling keeps the properties the reference tests for
  hase::utils::interpolateLinear (tests/interpolation.cpp): exact on linear
  data, no overshoot between samples.
* PhiASE argument validation mirrors pyInclude/simulation.py (ValueError).
"""

from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

from conftest import REPO


def _header_text():
    return "\n".join(p.read_text() for p in sorted((REPO / "include").glob("*.h")))


def _header_functions():
    text = _header_text()
    return sorted(set(re.findall(r"^(?:const char\*|int|hase_status)\s+(hase_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol(native):
    declared = _header_functions()
    assert declared == sorted(native.EXPORTED_SYMBOLS)
    lib = native.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert lib.hase_abi_version() == 2
    assert lib.hase_status_string(7) == b"no CUDA device"


def test_structures_match_header(native):
    text = _header_text()
    for cname, pyt in [("hase_mesh_desc", native.MeshDesc), ("hase_spectrum_desc", native.SpectrumDesc),
                       ("hase_experiment_desc", native.ExperimentDesc), ("hase_compute_desc", native.ComputeDesc),
                       ("hase_result", native.ResultDesc), ("hase_tet_mesh_desc", native.TetMeshDesc),
                       ("hase_forward_desc", native.ForwardDesc), ("hase_forward_result", native.ForwardResultDesc),
                       ("hase_pump_desc", native.PumpDesc), ("hase_time_desc", native.TimeDesc),
                       ("hase_time_result", native.TimeResultDesc), ("hase_proposal_batch", native.ProposalBatch),
                       ("hase_proposal_train_desc", native.ProposalTrainDesc), ("hase_learned_desc", native.LearnedDesc),
                       ("hase_batch_instance", native.BatchInstance), ("hase_batch_stats", native.BatchStats)]:
        body = re.search(r"typedef struct \{([^{}]*)\}\s*" + cname + ";", text).group(1)
        fields = re.findall(r"\b(\w+);", re.sub(r"/\*.*?\*/", "", body, flags=re.S))
        assert fields == [f for f, _ in pyt._fields_], cname


def test_library_is_sm100a_code(native):
    out = native.LIB_PATH.read_bytes()
    assert b"sm_100a" in out


def _has_device(native):
    n = C.c_int(0)
    try:
        cudart = C.CDLL("libcudart.so")
    except OSError:
        return False
    return cudart.cudaGetDeviceCount(C.byref(n)) == 0 and n.value > 0


def test_no_device_fails_loudly(native):
    if _has_device(native):
        pytest.skip("a CUDA device is present")
    with pytest.raises(native.HaseError) as err:
        native.philox([[0, 0, 0, 0]], [0, 0])
    assert err.value.status == native.HASE_NO_DEVICE
    from haseongpu_b200 import DeviceMesh
    from conftest import legacy_mesh, legacy_spectrum

    with pytest.raises(native.HaseError) as err:
        DeviceMesh(legacy_mesh("cuboid"), *legacy_spectrum("cuboid"))
    assert err.value.status == native.HASE_NO_DEVICE
    from haseongpu_b200 import TetDeviceMesh, TetMesh

    with pytest.raises(native.HaseError) as err:
        TetDeviceMesh(TetMesh.fromPrismMesh(legacy_mesh("cuboid")), *legacy_spectrum("cuboid"))
    assert err.value.status == native.HASE_NO_DEVICE
    from haseongpu_b200 import MediaBatch

    with pytest.raises(native.HaseError) as err:
        MediaBatch(0)
    assert err.value.status == native.HASE_NO_DEVICE


def test_tet_context_rejects_bad_meshes_before_touching_a_device(native):
    """Argument checks run before the device query (HASE_INVALID_ARGUMENT, not a fallback)."""
    from haseongpu_b200 import TetDeviceMesh, TetMesh

    pts = np.array([(0.0, 0, 0), (1.0, 0, 0), (0.0, 1, 0), (0.0, 0, 1)])
    flat = TetMesh(pts, np.array([(0, 1, 2, 3)]), [0.1], 1e20, 1e-3)
    flat.nTot = -1.0
    with pytest.raises(native.HaseError) as err:
        TetDeviceMesh(flat, [1e-21], [2e-20])
    assert err.value.status == native.HASE_INVALID_ARGUMENT
    bad = TetMesh(pts, np.array([(0, 1, 2, 3)]), [0.1], 1e20, 1e-3)
    bad.points = np.ascontiguousarray(np.where(np.isfinite(bad.points), bad.points, 0.0))
    bad.points[0, 0] = np.nan
    with pytest.raises(native.HaseError) as err:
        TetDeviceMesh(bad, [1e-21], [2e-20])
    assert err.value.status == native.HASE_INVALID_ARGUMENT


def test_interpolate_linear_exact_on_linear_data():
    from haseongpu_b200 import interpolate_linear

    rng = np.random.default_rng(0)
    m, b = rng.uniform(-1000, 1000, 2)
    for n in (100, 1000):
        x = np.sort(rng.uniform(-1000, 1000, n))
        y = m * x + b
        for ni in (n, 10 * n, 100 * n):
            yi = interpolate_linear(y, x, ni)
            xi = x[0] + np.arange(ni) * (x[-1] - x[0]) / (ni - 1)
            assert yi.size == ni
            assert np.max(np.abs(yi - (m * xi + b))) < 1e-8


def test_interpolate_linear_no_overshoot():
    from haseongpu_b200 import interpolate_linear

    rng = np.random.default_rng(0xBADC0DE)
    x = np.sort(rng.uniform(-1000, 1000, 1000))
    y = rng.uniform(-1000, 1000, 1000)
    yi = interpolate_linear(y, x, 100000)
    xi = x[0] + np.arange(100000) * (x[-1] - x[0]) / 99999
    seg = np.clip(np.searchsorted(x, xi, side="right") - 1, 0, x.size - 2)
    lo = np.minimum(y[seg], y[seg + 1])
    hi = np.maximum(y[seg], y[seg + 1])
    assert np.all(yi >= lo - 1e-9) and np.all(yi <= hi + 1e-9)
    assert yi[-1] == y[-1]
    with pytest.raises(ValueError):
        interpolate_linear(y, x, 10)
    np.testing.assert_array_equal(interpolate_linear([3.0], [1.0], 5), np.full(5, 3.0))


def test_cross_sections_resampling_and_monochromatic():
    from haseongpu_b200 import CrossSectionData

    cs = CrossSectionData([900, 950, 1000], [1e-21, 3e-21, 2e-21], [900, 1000], [5e-21, 1e-20], resolution=11)
    sa, se = cs.resampled()
    assert sa.size == se.size == 11
    assert sa[0] == pytest.approx(1e-21, rel=1e-12) and sa[-1] == 2e-21 and se[-1] == 1e-20
    sa1, se1 = cs.resampled(monochromatic=True)
    assert sa1.tolist() == [1e-21] and se1.tolist() == [5e-21]
    assert cs.maxSigmaA == 3e-21 and cs.maxSigmaE == 1e-20


def test_phiase_validation():
    from haseongpu_b200 import PhiASE

    with pytest.raises(ValueError):
        PhiASE(propagationMode="sideways")
    with pytest.raises(ValueError):
        PhiASE(parallelMode="mpi")
    with pytest.raises(ValueError):
        PhiASE(config={"mseThreshold": 0.1})
    with pytest.raises(ValueError):
        PhiASE(minRays=0)
    with pytest.raises(RuntimeError):
        PhiASE().getResults()
    with pytest.raises(ValueError):
        PhiASE().run()


def test_prism_mesh_layout():
    from conftest import legacy_mesh

    m = legacy_mesh("cylindrical")
    assert m.numberOfSamples == 4210 and m.numberOfPrisms == 812 * 9
    sp = m.samplePoints()
    np.testing.assert_allclose(sp[421 * 3 + 5], [*m.points[5], 3 * m.thickness])
    np.testing.assert_allclose(m.prismVolumes().sum(), m.triangleAreas().sum() * m.thickness * 9)
