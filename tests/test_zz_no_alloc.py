"""The allocation-free entry point, hase_estimate_sample_noalloc.

Some callers cannot allocate device memory: real-time loops whose device
memory is fixed up front (a cudaMalloc can block and synchronise the device
in the middle of the loop), or hosts that reserve the device's memory and
hand it out only from their own pool.  This entry point estimates one sample
point with all scratch in a fixed device array of the library; the tests
call it through the C ABI with device buffers for its input and output,
twice in a row, and check it against hase_calc_phi_ase for the same sample,
seed and ray count -- without and with reflections -- and that the device's
free memory is the same before and after each call.  (Collected last: a
failure here leaves every other test already run.)
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import legacy_mesh, legacy_spectrum

pytestmark = pytest.mark.gpu


def _noalloc_matches(native, ctx, samples, rays, seed, reflections):
    import torch

    lib = native.lib()
    # inputs and outputs first, so that nothing else allocates around the calls
    bufs = []
    for sample in samples:
        weights = ctx.importance_weights(sample, 1, reflections)[0]
        bufs.append((sample, torch.from_numpy(weights).to("cuda"),
                     torch.full((4,), -1.0, dtype=torch.float64, device="cuda")))
    torch.cuda.synchronize()
    # a first call on the device looks up the scratch array's address
    native.check(lib.hase_estimate_sample_noalloc(ctx.handle, samples[0], C.c_void_p(bufs[0][1].data_ptr()), 64, seed,
                                                  1 if reflections else 0, 1, C.c_void_p(bufs[0][2].data_ptr())))
    for call, (sample, d_weights, d_out) in enumerate(bufs):  # calls in a row share the scratch
        free_before = torch.cuda.mem_get_info()[0]
        status = lib.hase_estimate_sample_noalloc(ctx.handle, sample, C.c_void_p(d_weights.data_ptr()), rays, seed,
                                                  1 if reflections else 0, 1, C.c_void_p(d_out.data_ptr()))
        free_after = torch.cuda.mem_get_info()[0]
        native.check(status)
        assert free_after == free_before, (call, free_before - free_after)
        out = d_out.cpu().numpy()
        ref = ctx.calc_phi_ase(minRays=rays, maxRays=rays, rngSeed=seed, minSample=sample, maxSample=sample,
                               useReflections=reflections)
        assert out[2] == ref.totalRays[0] == rays, call
        assert out[3] == ref.droppedRays[0]
        np.testing.assert_allclose(out[0], float(ref.phiAse[0]), rtol=1e-6)
        np.testing.assert_allclose(out[1], ref.relativeStandardError[0], rtol=1e-9)


def test_noalloc_matches_existing_entry_point(native):
    from haseongpu_b200 import DeviceMesh

    mesh = legacy_mesh("cylindrical")
    sa, se = legacy_spectrum("cylindrical")
    with DeviceMesh(mesh, sa, se) as ctx:
        _noalloc_matches(native, ctx, (123, 2050), 50_000, 321, reflections=False)


def test_noalloc_with_reflections_matches_existing_entry_point(native):
    """disc_poly: 16 wavelengths, top/bottom reflectivities 0.3/0.9, five
    reflection slices of 95,874 prisms (479,370 prism-slices, inside the
    scratch limit of 524,288)."""
    from haseongpu_b200 import DeviceMesh
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    sa, se = w.spectra.resampled()
    with DeviceMesh(w.mesh, sa, se) as ctx:
        _noalloc_matches(native, ctx, (777, 4 * w.mesh.numberOfPoints + 9), 40_000, 99, reflections=True)


def test_noalloc_rejects_meshes_beyond_its_scratch(native):
    import torch

    from haseongpu_b200 import DeviceMesh, PrismMesh
    from haseongpu_b200.mesh import delaunay_triangles, disc_points

    pts = disc_points(1.0, 31, np.random.default_rng(0))
    tri = delaunay_triangles(pts)
    levels = 21  # 20 layers: 5 reflection slices x prisms > 524,288
    assert 5 * tri.shape[0] * (levels - 1) > (1 << 19)
    mesh = PrismMesh(points=pts, triangles=tri, numberOfLevels=levels, thickness=0.05,
                     betaVolume=np.full(tri.shape[0] * (levels - 1), 0.1), nTot=1e20, crystalTFluo=1e-3)
    lib = native.lib()
    with DeviceMesh(mesh, [1e-21], [2e-20]) as ctx:
        d_w = torch.ones(5 * mesh.numberOfPrisms, dtype=torch.float32, device="cuda")
        d_out = torch.zeros(4, dtype=torch.float64, device="cuda")
        status = lib.hase_estimate_sample_noalloc(ctx.handle, 0, C.c_void_p(d_w.data_ptr()), 1000, 1, 1, 1,
                                                  C.c_void_p(d_out.data_ptr()))
        assert status == native.HASE_INVALID_ARGUMENT
        assert b"allocation-free limit" in lib.hase_last_error_message()
        # without reflections the same mesh fits
        d_w1 = torch.ones(mesh.numberOfPrisms, dtype=torch.float32, device="cuda")
        native.check(lib.hase_estimate_sample_noalloc(ctx.handle, 0, C.c_void_p(d_w1.data_ptr()), 1000, 1, 0, 1,
                                                      C.c_void_p(d_out.data_ptr())))
        assert d_out.cpu().numpy()[2] == 1000
