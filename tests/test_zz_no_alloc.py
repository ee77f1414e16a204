"""The allocation-free entry point, hase_estimate_sample_noalloc.

Some callers cannot allocate device memory: code running while a stream is
captured into a CUDA graph, real-time loops whose memory is fixed up front,
or hosts that only hand out device memory from their own pool.  This entry
point estimates one sample point with all scratch in a fixed device array of
the library; the test calls it through the C ABI with device buffers for its
input and output, twice in a row, and checks it against hase_calc_phi_ase for
the same sample, seed and ray count.  (Collected last: a failure here leaves
every other test already run.)
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import legacy_mesh, legacy_spectrum

pytestmark = pytest.mark.gpu


def test_noalloc_matches_existing_entry_point(native):
    import torch

    from haseongpu_b200 import DeviceMesh

    lib = native.lib()
    mesh = legacy_mesh("cylindrical")
    sa, se = legacy_spectrum("cylindrical")
    rays, seed = 50_000, 321
    with DeviceMesh(mesh, sa, se) as ctx:
        for call, sample in enumerate((123, 2050)):  # two calls in a row share the scratch
            weights = ctx.importance_weights(sample, 1)[0]
            d_weights = torch.from_numpy(weights).to("cuda")
            d_out = torch.full((4,), -1.0, dtype=torch.float64, device="cuda")
            status = lib.hase_estimate_sample_noalloc(ctx.handle, sample, C.c_void_p(d_weights.data_ptr()), rays, seed,
                                                      0, 1, C.c_void_p(d_out.data_ptr()))
            native.check(status)
            out = d_out.cpu().numpy()
            ref = ctx.calc_phi_ase(minRays=rays, maxRays=rays, rngSeed=seed, minSample=sample, maxSample=sample)
            assert out[2] == ref.totalRays[0] == rays, call
            assert out[3] == ref.droppedRays[0]
            np.testing.assert_allclose(out[0], float(ref.phiAse[0]), rtol=1e-6)
            np.testing.assert_allclose(out[1], ref.relativeStandardError[0], rtol=1e-9)


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
