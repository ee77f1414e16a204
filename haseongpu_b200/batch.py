"""Many gain media in one phi-ASE solve (include/hase_b200_batch.h).

``MediaBatch.solve`` takes device meshes (``DeviceMesh``) with a sample range
each and solves them together: one pooled workspace, one persistent ray
launch per adaptive pass over the active sample points of every medium, the
whole schedule captured as one CUDA graph.  Medium i uses the Philox key
``rngSeed + i``, so its result equals ``DeviceMesh.calc_phi_ase`` with that
seed, bit for bit.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .simulation import DeviceMesh, Result


@dataclass
class BatchStats:
    raysTraced: int
    crossings: int
    rows: int
    chunks: int
    passes: int
    unconvergedSamples: int
    kernelLaunches: int
    graphNodes: int
    importanceMilliseconds: float
    rayMilliseconds: float
    totalMilliseconds: float
    captureMilliseconds: float
    setupMilliseconds: float
    hostMilliseconds: float
    fallbackSamples: int
    status: int = 0


class MediaBatch:
    """A batched-solve workspace on one device (hase_batch)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib().hase_batch_create(int(device), C.byref(h)))
        self.handle = h
        self.device = device

    def solve(self, media, *, minRays, maxRays=None, mseThreshold=0.0, useReflections=False, monochromatic=False,
              nearFieldSampling=True, adaptiveSteps=0, rngSeed=5489, raysPerThread=0, workspaceBytes=0,
              rayKernelVariant=0, importanceLayers=0, net=None, mixture=0.0, fallbackVariance=0.0):
        """media: DeviceMesh objects, or (DeviceMesh, minSample, maxSample)
        tuples (maxSample None = last).  net: a ProposalNet whose learned
        proposal replaces the importance weights of every medium (mixture:
        weight of the beta V / d^2 prior, 0 = 0.1; fallbackVariance: per-ray
        variance above which a sample restarts with the importance weights
        after the first pass, 0 = never).  Returns
        ([Result per medium], BatchStats)."""
        items = []
        for m in media:
            if isinstance(m, DeviceMesh):
                items.append((m, 0, None))
            else:
                ctx, lo, hi = m
                items.append((ctx, int(lo), hi))
        if not items:
            raise ValueError("no media")
        outs, descs, keep = [], (N.BatchInstance * len(items))(), []
        ex = cp = None
        for i, (ctx, lo, hi) in enumerate(items):
            out, e, c, r, _ = ctx._descs(minRays, maxRays, mseThreshold, useReflections, monochromatic,
                                         nearFieldSampling, adaptiveSteps, 1, rngSeed, lo, hi, raysPerThread, 0,
                                         workspaceBytes, rayKernelVariant, importanceLayers)
            ex, cp = (e, c) if ex is None else (ex, cp)
            keep.append(r)
            descs[i].context = ctx.handle
            descs[i].minSample = lo
            descs[i].maxSample = ctx.mesh.numberOfSamples - 1 if hi is None else int(hi)
            descs[i].result = C.pointer(r)
            outs.append(out)
        st = N.BatchStats()
        if net is None:
            rc = N.lib().hase_calc_phi_ase_batch(self.handle, descs, len(items), C.byref(ex), C.byref(cp), C.byref(st))
        else:
            rc = N.lib().hase_calc_phi_ase_batch_learned(self.handle, descs, len(items), C.byref(ex), C.byref(cp),
                                                         net.handle, float(mixture), float(fallbackVariance),
                                                         C.byref(st))
        status = N.check(rc, allow_warnings=True)
        for out, r in zip(outs, keep):
            DeviceMesh._fill(out, r, status)
        stats = BatchStats(*(getattr(st, f) for f, _ in N.BatchStats._fields_), status=status)
        return outs, stats

    def close(self):
        if getattr(self, "handle", None):
            N.lib().hase_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve_sequential(media, **kw) -> list[Result]:
    """The same media solved one after another with ``DeviceMesh.calc_phi_ase``
    (medium i with seed rngSeed + i): the unbatched path the batch replaces."""
    seed = int(kw.pop("rngSeed", 5489))
    outs = []
    for i, m in enumerate(media):
        ctx, lo, hi = (m, 0, None) if isinstance(m, DeviceMesh) else m
        outs.append(ctx.calc_phi_ase(rngSeed=(seed + i) & 0xFFFFFFFF, minSample=lo, maxSample=hi, **kw))
    return outs
