"""The learned-proposal protocol: seeded pump fields on one geometry, training
sets logged by the importance-sampled method, training on the GPU, and the
comparison against the method without the network.

Geometry and spectra are the small disc (``configs.disc_small``).  Training
uses 32 seeded beta fields; evaluation uses unseen fields drawn from the same
family with other seeds.  A field is a Gaussian pump
beta = base + peak exp(-r^2 / waist^2) exp(-z / depth) at the prism centres,
times (1 + U(-0.05, 0.05)) noise, with base ~ U(0.02, 0.08),
peak ~ U(0.15, 0.35), waist ~ U(0.25, 0.6) cm, depth ~ U(0.3, 1.0) cm.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import PrismMesh, gaussian_pump_beta
from .proposal import ProposalNet

TRAIN_SEED = 20261204
EVAL_SEED = 20261205


def pump_field(mesh: PrismMesh, rng: np.random.Generator) -> np.ndarray:
    beta = gaussian_pump_beta(mesh.points, mesh.triangles, mesh.numberOfLevels, mesh.thickness,
                              waist=rng.uniform(0.25, 0.6), depth=rng.uniform(0.3, 1.0),
                              base=rng.uniform(0.02, 0.08), peak=rng.uniform(0.15, 0.35))
    return beta * (1.0 + rng.uniform(-0.05, 0.05, beta.size))


def pump_fields(mesh: PrismMesh, n: int, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    return [pump_field(mesh, rng) for _ in range(n)]


@dataclass
class TrainingSet:
    offsets: np.ndarray   # [groups + 1]
    features: np.ndarray  # [rows, 12]
    targets: np.ndarray   # [rows]
    rays: int             # rays logged per group
    importanceVariance: np.ndarray | None = None  # [groups] per-ray variance of the importance-weighted solves

    @property
    def groups(self) -> int:
        return self.offsets.size - 1

    def fallback_limit(self, quantile: float = 1.0) -> float:
        """The plain method as the judge: a per-ray relative variance limit
        (``fallbackVariance`` of the learned solve) at the given quantile of
        what the importance weights reached on the logged samples."""
        if self.importanceVariance is None or self.importanceVariance.size == 0:
            return 0.0
        return float(np.quantile(self.importanceVariance, quantile))


def training_set(ctx, fields, *, samples_per_field=32, rays=100_000, monochromatic=True, useReflections=False,
                 seed=TRAIN_SEED) -> TrainingSet:
    """Per field: a block of consecutive sample points solved with the
    importance weights, every ray's contribution summed per (slice, prism)
    (the targets), and the features of the same pairs.  Pairs without a
    source (beta = 0) are left out: the proposal gives them no rays."""
    rng = np.random.default_rng(seed)
    S = ctx.mesh.numberOfSamples
    feats, targs, offs, var = [], [], [0], []
    for k, beta in enumerate(fields):
        ctx.update_beta(beta)
        first = int(rng.integers(0, max(1, S - samples_per_field)))
        res, con = ctx.log_contributions(minRays=rays, monochromatic=monochromatic, useReflections=useReflections,
                                         rngSeed=seed + k, minSample=first, maxSample=first + samples_per_field - 1)
        var.append(per_ray_variance(res))
        f = ctx.proposal_features(first, samples_per_field, useReflections=useReflections,
                                  monochromatic=monochromatic)
        for i in range(samples_per_field):
            keep = f[i, :, 7] > 0
            feats.append(f[i][keep])
            targs.append(np.maximum(con[i][keep], 0.0))
            offs.append(offs[-1] + int(keep.sum()))
    return TrainingSet(np.asarray(offs, np.uint32), np.concatenate(feats), np.concatenate(targs).astype(np.float32),
                       rays, np.concatenate(var))


def training_set_media(ctxs, *, samples_per_medium=16, rays=100_000, monochromatic=False, useReflections=False,
                       seed=TRAIN_SEED) -> TrainingSet:
    """The training set of a family of media: per medium (a DeviceMesh with
    its own mesh, beta and spectrum) a seeded block of consecutive sample
    points solved with the importance weights, contributions logged per
    (slice, prism) as the targets, and the features of the same pairs."""
    rng = np.random.default_rng(seed)
    feats, targs, offs, var = [], [], [0], []
    for k, ctx in enumerate(ctxs):
        S = ctx.mesh.numberOfSamples
        n = min(samples_per_medium, S)
        first = int(rng.integers(0, max(1, S - n)))
        res, con = ctx.log_contributions(minRays=rays, monochromatic=monochromatic, useReflections=useReflections,
                                         rngSeed=seed + k, minSample=first, maxSample=first + n - 1)
        var.append(per_ray_variance(res))
        f = ctx.proposal_features(first, n, useReflections=useReflections, monochromatic=monochromatic)
        for i in range(n):
            keep = f[i, :, 7] > 0
            feats.append(f[i][keep])
            targs.append(np.maximum(con[i][keep], 0.0))
            offs.append(offs[-1] + int(keep.sum()))
    return TrainingSet(np.asarray(offs, np.uint32), np.concatenate(feats), np.concatenate(targs).astype(np.float32),
                       rays, np.concatenate(var))


def train_proposal(data: TrainingSet, *, steps=3000, groups_per_step=16, learning_rate=2e-3, device=0, seed=1):
    """A proposal network trained on `data` (Adam on the device); returns
    (net, loss history)."""
    net = ProposalNet(device=device, seed=seed)
    order = np.random.default_rng(seed).permutation(data.groups)
    off, feats, targs = reorder(data, order)
    hist = net.train(off, feats, targs, steps=steps, groups_per_step=groups_per_step, learning_rate=learning_rate)
    return net, hist


def reorder(data: TrainingSet, order):
    """The groups of `data` in `order` (training steps take consecutive groups);
    returns (offsets, features, targets)."""
    sizes = np.diff(data.offsets.astype(np.int64))
    idx = np.concatenate([np.arange(data.offsets[g], data.offsets[g + 1]) for g in order])
    off = np.concatenate([[0], np.cumsum(sizes[order])]).astype(np.uint32)
    return off, data.features[idx], data.targets[idx]


def per_ray_variance(result) -> np.ndarray:
    """rays x relative error^2 per sample: the variance of one ray's
    contribution relative to the mean squared (ray budget for a target error
    eps is this / eps^2)."""
    return result.totalRays.astype(np.float64) * result.relativeStandardError ** 2


def warm_started_series(ctx, net, pump, time, *, rays, useReflections=True, monochromatic=False, log_samples=32,
                        log_rays=20_000, train_steps=20, groups_per_step=8, learning_rate=1e-3, fallback="logged",
                        rngSeed=5489):
    """The time-stepped rate equations with the learned proposal warm-started
    from step to step (the time loop of include/core/timeSteppedSimulation.hpp:
    132-617, one step per hase_simulate call): before the phi-ASE solve of
    step k > 0 the network ``net`` is fine-tuned on the current beta --
    ``train_steps`` Adam steps on the device over the contributions logged by
    the importance-weighted method for a seeded block of ``log_samples``
    consecutive sample points (``log_rays`` rays each) -- and the step then
    solves every sample point with ``rays`` rays per sample and the network.
    ``fallback``: the per-ray variance above which the plain importance
    weights take over a sample after the first pass -- "logged" (the largest
    the importance-weighted log solve of the step reached on its block: the
    plain method as the judge), a number, or 0 (never).  The pump runs
    for ``time["pumpSteps"]`` steps and phi-ASE for ``time["aseSteps"]``.
    With the context's local proposal set, the network weights the candidate
    entries and the far prior keeps its share.  Returns the per-step series
    and the device and host times."""
    import time as clock

    steps = int(time["steps"])
    pump_steps = int(time.get("pumpSteps", steps))
    ase_steps = int(time.get("aseSteps", steps))
    S = ctx.mesh.numberOfSamples
    n = min(int(log_samples), S)
    rng = np.random.default_rng(rngSeed)
    out = {"meanBeta": [], "meanPhi": [], "pumpAbsorbed": [], "loss": [], "aseMilliseconds": 0.0,
           "pumpMilliseconds": 0.0, "totalMilliseconds": 0.0, "raysTraced": 0, "fallbackSamples": 0,
           "trainSeconds": 0.0, "stepSeconds": 0.0}
    fallbackVariance = 0.0 if fallback == "logged" else float(fallback)
    for k in range(steps):
        t0 = clock.perf_counter()
        if k > 0 and ase_steps > k:
            first = int(rng.integers(0, max(1, S - n)))
            res, con = ctx.log_contributions(minRays=log_rays, monochromatic=monochromatic,
                                             useReflections=useReflections, rngSeed=rngSeed + 7919 * k,
                                             minSample=first, maxSample=first + n - 1)
            if fallback == "logged":
                v = per_ray_variance(res)
                fallbackVariance = float(v[np.isfinite(v)].max()) if np.isfinite(v).any() else 0.0
            f = ctx.proposal_features(first, n, useReflections=useReflections, monochromatic=monochromatic)
            feats, targs, offs = [], [], [0]
            for i in range(n):
                keep = (f[i, :, 7] > 0) & (con[i] > 0)
                if keep.sum() < 2:
                    continue
                feats.append(f[i][keep])
                targs.append(con[i][keep])
                offs.append(offs[-1] + int(keep.sum()))
            if len(offs) > 1:
                hist = net.train(np.asarray(offs, np.uint32), np.concatenate(feats),
                                 np.concatenate(targs).astype(np.float32), steps=train_steps,
                                 groups_per_step=min(groups_per_step, len(offs) - 1), learning_rate=learning_rate)
                out["loss"].append(float(hist[-1]))
        t1 = clock.perf_counter()
        step = dict(time, steps=1, pumpSteps=1 if k < pump_steps else 0, aseSteps=1 if k < ase_steps else 0)
        r = ctx.simulate(pump=pump, time=step, net=net, fallbackVariance=fallbackVariance, minRays=rays,
                         useReflections=useReflections, monochromatic=monochromatic, rngSeed=rngSeed + k)
        t2 = clock.perf_counter()
        if k == 0:
            out["meanBeta"].append(float(r["meanBeta"][0]))
        out["meanBeta"].append(float(r["meanBeta"][-1]))
        out["meanPhi"].append(float(r["meanPhi"][-1]))
        out["pumpAbsorbed"].append(float(r["pumpAbsorbed"][-1]))
        for key in ("aseMilliseconds", "pumpMilliseconds", "totalMilliseconds"):
            out[key] += float(r[key])
        out["raysTraced"] += int(r["raysTraced"])
        out["fallbackSamples"] += int(r["fallbackSamples"])
        out["trainSeconds"] += t1 - t0
        out["stepSeconds"] += t2 - t1
    return out
