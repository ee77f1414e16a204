"""Autotuner for the ray kernel's launch shape (single-medium and batched solves).

Sweeps every launch shape libhase_b200 compiles (block size, idle lanes that
trigger a batched refill, occupancy target; ``hase_ray_kernel_variant_name``)
and the work-item size (rays per lane of a work item) on a short, fixed-ray
solve of the caller's own workload, timing only the ray kernel with the CUDA
events the library records, and returns the fastest pair.  Results are
cached per process by (device, mesh size, reflections, wavelengths).
"""

from __future__ import annotations

from dataclasses import dataclass

from . import _native as N

RAYS_PER_LANE = (16, 32, 64, 128)  # work items of 512 .. 4096 rays

_cache: dict = {}


@dataclass
class TuneResult:
    rayKernelVariant: int
    raysPerThread: int
    name: str
    milliseconds: float
    table: list
    importanceLayers: int = 0
    importanceMilliseconds: float = 0.0

    def kwargs(self) -> dict:
        return {"rayKernelVariant": self.rayKernelVariant, "raysPerThread": self.raysPerThread,
                "importanceLayers": self.importanceLayers}


def variant_names() -> list[str]:
    lib = N.lib()
    return [lib.hase_ray_kernel_variant_name(i).decode() for i in range(lib.hase_ray_kernel_variant_count())]


def pinned(name: str, raysPerThread: int = 16, importanceLayers: int = 0) -> TuneResult:
    """A launch shape chosen by name instead of by a sweep (to time or profile
    one exact kernel); raises ValueError for a name the library does not have."""
    names = variant_names()
    if name not in names:
        raise ValueError(f"unknown ray-kernel launch shape {name!r}; known: {', '.join(names)}")
    return TuneResult(names.index(name), raysPerThread, name, 0.0, [], importanceLayers, 0.0)


def autotune(ctx, *, firstSample: int, samples: int, rays: int, useReflections: bool, monochromatic: bool,
             nearFieldSampling: bool = True, repeats: int = 2, device: int = 0) -> TuneResult:
    mesh = ctx.mesh
    key = (device, mesh.numberOfTriangles, mesh.numberOfLevels, bool(useReflections), ctx.numberOfWavelengths,
           bool(monochromatic), samples, rays)
    if key in _cache:
        return _cache[key]
    names = variant_names()
    table = []
    best = None
    for v, name in enumerate(names):
        for rpt in RAYS_PER_LANE:
            t = min(ctx.calc_phi_ase(minRays=rays, maxRays=rays, useReflections=useReflections,
                                     monochromatic=monochromatic, nearFieldSampling=nearFieldSampling,
                                     rngSeed=17 + k, minSample=firstSample, maxSample=firstSample + samples - 1,
                                     rayKernelVariant=v, raysPerThread=rpt).rayMilliseconds
                    for k in range(repeats))
            table.append({"variant": v, "name": name, "raysPerThread": rpt, "ray_ms": t})
            if best is None or t < best[2]:
                best = (v, rpt, t)
    imp = []
    for layers in (0, 2, 4, 8):  # 0: the line-team kernel
        t = min(ctx.calc_phi_ase(minRays=1, maxRays=1, useReflections=useReflections, monochromatic=monochromatic,
                                 nearFieldSampling=nearFieldSampling, rngSeed=3, minSample=firstSample,
                                 maxSample=firstSample + samples - 1, importanceLayers=layers).importanceMilliseconds
                for _ in range(repeats))
        imp.append((t, layers))
        table.append({"importanceLayers": layers, "importance_ms": t})
    result = TuneResult(best[0], best[1], names[best[0]], best[2], table, min(imp)[1], min(imp)[0])
    _cache[key] = result
    return result


def autotune_batch(batch, media, *, rays: int, useReflections: bool = False, monochromatic: bool = False,
                   nearFieldSampling: bool = True, repeats: int = 2, workspaceBytes: int = 0) -> TuneResult:
    """The same sweep for the pooled ray kernel of a batched solve
    (``MediaBatch.solve``): every launch shape x work-item size on a fixed-ray
    solve of the caller's media, timed by the ray launches' device time."""
    names = variant_names()
    table = []
    best = None
    for v, name in enumerate(names):
        for rpt in RAYS_PER_LANE:
            t = min(batch.solve(media, minRays=rays, maxRays=rays, useReflections=useReflections,
                                monochromatic=monochromatic, nearFieldSampling=nearFieldSampling, rngSeed=31 + k,
                                rayKernelVariant=v, raysPerThread=rpt, workspaceBytes=workspaceBytes)[1].rayMilliseconds
                    for k in range(repeats))
            table.append({"variant": v, "name": name, "raysPerThread": rpt, "ray_ms": t})
            if best is None or t < best[2]:
                best = (v, rpt, t)
    return TuneResult(best[0], best[1], names[best[0]], best[2], table)
