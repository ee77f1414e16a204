#!/usr/bin/env python3
"""bench.py -- phi-ASE throughput of libhase_b200 on B200.

Default workload ``learned`` (the headline: time to threshold with the
learned proposal against plain importance sampling): the network is trained
(untimed) on contributions logged on 32 seeded pump fields of the disc_small
geometry; a step is one full adaptive phi-ASE solve of every sample point of
one unseen pump field (learned proposal, ray->prism map, ray passes until
every sample's relative error <= threshold or maxRays).  The same fields are
also solved with the reference's plain importance sampling and with the
importance weights + near-field start points.  Metric: time to threshold,
reported as its throughput form -- sample points brought to the threshold per
second over the whole job -- with rays/s and the per-step time beside it.
The line nests the importance-sampled solve of ``disc_poly`` (polychromatic
disc with reflections; ``--workload disc_poly`` prints it as the line) and the
forward Tet4 path (``--path forward``).

``value`` is device-timed (CUDA events recorded by the library on the stream
its kernels run on), inputs resident; ``e2e`` goes through the public API with
host buffers: each step uploads the step's beta field (H2D) and reads the
per-sample results back (D2H).  Under torchrun each rank runs its own sample
batches (weak scaling, no collective on the data path); timing is the max over
ranks.

``--impl reference`` times the CPU restatement of the same method (the oracle,
FP64, OpenMP over all host threads) on a bounded sample of the same workload:
the reference's own CPU backend cannot be built here (alpaka3 / openPMD-api
are not available), and its serial backend throws for this path.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = ("phi-ASE time to per-sample relative error <= threshold on 1 B200, as sample points solved per second "
          "(rays/s alongside)")
FP32_INSTR_PER_CROSSING = 24   # stated per-crossing FP32 instruction count
BYTES_PER_CROSSING = 52        # triangle record 48 B + prism beta 4 B
SMS = 148
LANES_PER_SM = 128
MLP_FLOP_PER_PAIR = 2 * (12 * 64 + 64 * 64 + 64 * 64 + 64 * 1)  # 18,048 FLOP per (sample, prism) inference
# special-function (XU) instructions per pair, from ncu (XU pipe 65.2 % active over 7.44e6 cycles x 148 SMs x 16
# lanes = 1.15e10 for 4.99e7 pairs): 192 SiLUs x 1 (tanh) + ~38 in the features (the float-to-int conversions and
# floors of the 8-point gain-grid lookup, two logarithms, a square root, an exponential, reciprocals)
XU_INSTR_PER_PAIR = 230
XU_LANES_PER_SM = 16
FWD_METRIC = "forward Tet4 phi-ASE source rays traced and tallied per second on 1 B200 (crossings/s alongside)"
FP64_INSTR_PER_TET_CROSSING = 100  # stated per-crossing FP64 instruction count of the forward walk
BYTES_PER_TET_CROSSING = 148       # cell record 128 B + beta 8 B + one vertex tally 8 B + one visit count 4 B
FWD_TRAFFIC_DISC_POLY = 49128192   # DRAM bytes of one fwdRayKernel launch on the disc_poly Tet4 twin (ncu)
FP64_LANES_PER_SM = 64
# DRAM bytes of one learned-solve rayKernel launch on disc_small (5,470 samples x 1e5 rays; ncu): the per-sample
# ray maps (q, offsets) read once and the per-item partial sums written; the walk tables stay in L1/L2
RAY_TRAFFIC_LEARNED = 402847744 + 29695232
# what binds the same launch (ncu --set full of it): instruction issue, with the walk tables in L1 -- thread
# instructions per crossing and per ray of that capture (3.09e10 warp instructions x 24.4 threads, 5.47e8 rays)
RAY_BINDING_LEARNED = "instruction issue (ncu: issue active 85.6 %, top stall 'not selected'; L1 hits 99.2 %)"
RAY_INSTR_LEARNED = {"per_crossing": 97, "per_ray": 1379, "crossings_per_ray": 14.2}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8,
                    help="timed steps; the learned workload solves one unseen pump field per step (config 4: 8)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="learned",
                    help="learned (config 4, the headline), media64 (config 3, batched media), disc_poly or "
                         "disc_small (importance-sampled solve)")
    ap.add_argument("--no-nested", action="store_true", help="learned workload only: skip the disc_poly and forward lines")
    ap.add_argument("--samples", type=int, default=1024, help="sample points per step and rank")
    ap.add_argument("--pulse-backward-rays", type=int, default=2000,
                    help="pulse workload: backward rays per sample point and time step (local proposal)")
    ap.add_argument("--pulse-local-triangles", type=int, default=16,
                    help="pulse workload: candidate triangles per sample point of the local proposal")
    ap.add_argument("--pulse-rays", type=int, default=2_000_000,
                    help="pulse workload: forward source rays per time step")
    ap.add_argument("--media-samples", type=int, default=64,
                    help="media64 workload: sample points per medium (64 media) per step")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="bounded CPU baseline sample")
    ap.add_argument("--path", default="backward", choices=["backward", "forward"],
                    help="backward: importance-sampled prism method (headline); forward: Tet4 source-ray method")
    ap.add_argument("--forward-rays", type=int, default=16_000_000, help="source rays per forward step")
    ap.add_argument("--tally", default="auto", choices=["auto", "global", "shared"],
                    help="vertex tallies of the forward kernel")
    ap.add_argument("--ray-variant", default=None,
                    help="learned and importance workloads: this ray-kernel launch shape (by name) instead of the "
                         "autotuner's choice, e.g. to profile one exact kernel")
    ap.add_argument("--rays-per-lane", type=int, default=16, help="work-item size with --ray-variant")
    return ap.parse_args()


def measured_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text()), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def cpu_baseline(workload, seconds, fields=None, nearField=False):
    """The reference's method on the host cores: the oracle (FP64 restatement
    of the importance-sampled method; uniform start points unless nearField)
    runs the same adaptive solve to the threshold on all host threads,
    `cores` consecutive samples from a random position at a time -- each
    chunk on the next of `fields` (beta per prism) when given -- bounded in
    time (at least one chunk)."""
    import numpy as np

    from oracle import oracle

    w = workload
    sa, se = w.spectra.resampled(w.monochromatic)
    cores = os.cpu_count() or 1
    S = w.mesh.numberOfSamples
    rng = np.random.default_rng(1)
    rays = 0
    n_samples = 0
    chunks = 0
    t0 = time.perf_counter()
    while n_samples == 0 or time.perf_counter() - t0 < seconds:
        first = int(rng.integers(0, S - cores))
        mesh = w.mesh if fields is None else w.mesh.withBeta(fields[chunks % len(fields)])
        r = oracle.phi_ase(mesh, (sa, se), minRays=w.minRays, maxRays=w.maxRays, adaptiveSteps=w.adaptiveSteps,
                           mseThreshold=w.threshold, useReflections=w.useReflections, seed=7, minSample=first,
                           maxSample=first + cores - 1, threads=cores, nearField=nearField)
        rays += int(r["totalRays"].astype(np.int64).sum())
        n_samples += cores
        chunks += 1
    dt = time.perf_counter() - t0
    estimator = ("importance weights, near-field start points" if nearField else
                 "the reference's estimator: importance weights, uniform start points")
    where = f"{min(chunks, len(fields))} of the unseen pump fields" if fields is not None else f"{w.name}"
    return {"value": n_samples / dt, "unit": "samples/s", "rays_per_s": rays / dt, "cores": cores, "kind": "port",
            "sample": f"{n_samples} samples of {where} solved to relative error <= {w.threshold} "
                      f"(rays {w.minRays}-{w.maxRays}, {rays} rays, {estimator}, importance walks included), "
                      f"{dt:.1f} s on {cores} threads"}


def learned_config(w, mesh, n_gpus):
    """The learned workload's config (both arms): what is solved, not how."""
    return {"workload": "learned proposal (config 4): disc_small geometry, 32 training pump fields, "
                        "unseen evaluation pump fields",
            "samples_per_step_per_gpu": mesh.numberOfSamples, "triangles": mesh.numberOfTriangles,
            "levels": mesh.numberOfLevels, "prisms": mesh.numberOfPrisms, "wavelengths": 1,
            "rays_per_sample": [w.minRays, w.maxRays], "threshold": w.threshold,
            "adaptive_steps": w.adaptiveSteps, "parallelism": f"independent fields x{n_gpus}",
            "l2": "flushed (256 MiB write) before every timed step"}


class ClockSampler:
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        finally:
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def setup_ranks():
    """rank, world, local; one process per GPU, NCCL process group for N > 1."""
    import torch
    import torch.distributed as dist

    from haseongpu_b200 import build as _build

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    _build.build_library()
    return rank, world, local


def teardown_ranks(world):
    import torch.distributed as dist

    if world > 1:
        dist.destroy_process_group()


def run_ours(args):
    rank, world, local = setup_ranks()
    line = measure_importance(args, local, rank, world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    teardown_ranks(world)


def measure_importance(args, local, rank=0, world=1, nested=False):
    """The importance-sampled solve to the threshold on ``args.workload``
    (default disc_poly), the plain method beside it; the contract line's
    fields (rank 0; None elsewhere).  nested: no CPU baseline and no forward
    measurement (the caller reports those)."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from haseongpu_b200 import DeviceMesh
    from haseongpu_b200.configs import WORKLOADS

    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]()
    mesh = w.mesh
    sa, se = w.spectra.resampled(w.monochromatic)
    S = mesh.numberOfSamples
    B = min(args.samples, S)
    ctx = DeviceMesh(mesh, sa, se, device=local)
    flush = torch.empty(64 << 20, dtype=torch.int32, device=dev)  # 256 MiB > 126 MB L2

    # launch shape of the ray kernel: the project's autotuner, on this workload (untimed)
    from haseongpu_b200.autotune import autotune, pinned

    if args.ray_variant:
        tuned = pinned(args.ray_variant, args.rays_per_lane)
    else:
        tuned = autotune(ctx, firstSample=0, samples=min(B, 128), rays=w.minRays, useReflections=w.useReflections,
                         monochromatic=w.monochromatic, device=local)

    def run_step(step, beta=None):
        first = ((step * world + rank) * B) % (S - B + 1)
        if beta is not None:
            ctx.update_beta(beta)
        return ctx.calc_phi_ase(minRays=w.minRays, maxRays=w.maxRays, mseThreshold=w.threshold,
                                useReflections=w.useReflections, monochromatic=w.monochromatic,
                                adaptiveSteps=w.adaptiveSteps, rngSeed=1000 + step, minSample=first,
                                maxSample=first + B - 1, **tuned.kwargs())

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for s in range(args.warmup):
        run_step(s)
    barrier()
    dev_ms, ray_ms, rays, crossings, launches, unconverged, steps_ms, solved = 0.0, 0.0, 0, 0, 0, 0, [], 0
    imp_ms = 0.0
    with ClockSampler(local) as clk:
        barrier()
        t0 = time.perf_counter()
        for s in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            r = run_step(args.warmup + s)
            dev_ms += r.totalMilliseconds
            ray_ms += r.rayMilliseconds
            imp_ms += r.importanceMilliseconds
            rays += r.raysTraced
            crossings += r.crossings
            launches += r.kernelLaunches + 1
            unconverged += r.unconvergedSamples
            solved += B
            steps_ms.append(r.totalMilliseconds)
        barrier()
        wall = time.perf_counter() - t0
    clocks = clk.summary()

    # e2e: public API with host buffers (beta upload + results read back every step)
    beta_host = [np.ascontiguousarray(mesh.betaVolume * (1.0 + 0.01 * k)) for k in range(args.steps)]
    barrier()
    t1 = time.perf_counter()
    e2e_rays = 0
    for s in range(args.steps):
        r = run_step(args.warmup + s, beta=beta_host[s])
        e2e_rays += r.raysTraced
    e2e_solved = args.steps * B
    barrier()
    e2e_s = time.perf_counter() - t1
    ctx.update_beta(mesh.betaVolume)

    # crossings of the timed steps' importance walks (an instrumented copy of the kernel, untimed)
    imp_crossings = sum(ctx.importance_crossings(((args.warmup + s) * world + rank) * B % (S - B + 1), B,
                                                 w.useReflections) for s in range(args.steps))
    # the plain method (uniform start points, as the legacy code) on one batch, for comparison
    plain = ctx.calc_phi_ase(minRays=w.minRays, maxRays=w.maxRays, mseThreshold=w.threshold,
                             useReflections=w.useReflections, monochromatic=w.monochromatic,
                             adaptiveSteps=w.adaptiveSteps, rngSeed=1000, minSample=0, maxSample=B - 1,
                             nearFieldSampling=False, **tuned.kwargs())
    # the coarse-grid proposal on the same batch: weights from the gain grid
    # instead of the importance walks (hase_context_set_grid_proposal)
    gkw = dict(minRays=w.minRays, maxRays=w.maxRays, mseThreshold=w.threshold, useReflections=w.useReflections,
               monochromatic=w.monochromatic, adaptiveSteps=w.adaptiveSteps, minSample=0, maxSample=B - 1,
               **tuned.kwargs())
    ctx.set_grid_proposal(True)
    ctx.calc_phi_ase(rngSeed=2000, **gkw)  # warm-up: the grid is built once per beta
    grid_runs = [ctx.calc_phi_ase(rngSeed=2001 + k, **gkw) for k in range(3)]
    ctx.set_grid_proposal(False)
    # the forward Tet4 path on the twin of the same medium (1 GPU runs only; fewer steps)
    fwd = None
    if world == 1 and not nested:
        import argparse as _ap

        fargs = _ap.Namespace(**vars(args))
        fargs.steps, fargs.warmup = max(2, min(args.steps, 3)), max(args.warmup, 3)
        fwd = measure_forward(fargs, local, cpu_seconds=min(args.cpu_seconds, 6.0))
    stats = torch.tensor([dev_ms, float(rays), float(e2e_s), float(e2e_rays), float(crossings), ray_ms,
                          float(solved), float(e2e_solved)], dtype=torch.float64, device=dev)
    if world > 1:
        mx = stats.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = stats.clone()
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        dev_ms_max, e2e_max = float(mx[0]), float(mx[2])
        rays_all, e2e_rays_all, cross_all = float(sm[1]), float(sm[3]), float(sm[4])
        solved_all, e2e_solved_all = float(sm[6]), float(sm[7])
    else:
        dev_ms_max, e2e_max, rays_all, e2e_rays_all, cross_all = dev_ms, e2e_s, float(rays), float(e2e_rays), float(crossings)
        solved_all, e2e_solved_all = float(solved), float(e2e_solved)

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
        r_fp32 = SMS * LANES_PER_SM * f_clk / FP32_INSTR_PER_CROSSING
        from haseongpu_b200 import _native

        l2 = _native.l2_bandwidth(local)
        r_l2 = l2 * 1e9 / BYTES_PER_CROSSING
        achieved = crossings / (ray_ms * 1e-3)
        roof = min(r_fp32, r_l2)
        cpu = cpu_baseline(w, args.cpu_seconds) if world == 1 and not nested else None
        h2d = mesh.numberOfPrisms * 8
        d2h = B * (4 + 8 + 8 + 4 + 8 + 4)
        line = {
            "metric": METRIC,
            "value": solved_all / (dev_ms_max * 1e-3),
            "unit": "samples/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": dev_ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 geometry, f64 sums",
            "data": "synthetic (seeded gain medium, no dataset)",
            "config": {"workload": w.name, "samples_per_step_per_gpu": B, "triangles": mesh.numberOfTriangles,
                       "levels": mesh.numberOfLevels, "prisms": mesh.numberOfPrisms,
                       "wavelengths": int(len(sa)), "reflections": w.useReflections,
                       "rays_per_sample": [w.minRays, w.maxRays], "threshold": w.threshold,
                       "adaptive_steps": w.adaptiveSteps, "parallelism": f"sample batches x{world}",
                       "l2": "flushed (256 MiB write) before every timed step; per-step weights > L2",
                       "ray_kernel": {"variant": tuned.name, "rays_per_item": 32 * tuned.raysPerThread,
                                      "autotuned_ms": tuned.milliseconds},
                       "importance_kernel": {"layers_per_thread": tuned.importanceLayers,
                                             "autotuned_ms": tuned.importanceMilliseconds}},
            "time_to_threshold_ms": statistics.median(steps_ms),
            "breakdown_ms_per_step": {"importance": imp_ms / args.steps, "rays": ray_ms / args.steps,
                                      "map_finalize_copies": (dev_ms - imp_ms - ray_ms) / args.steps},
            "rays_per_s": rays_all / (dev_ms_max * 1e-3),
            "crossings_per_s": cross_all / (dev_ms_max * 1e-3),
            "plain_method": {"time_to_threshold_ms": plain.totalMilliseconds, "rays": plain.raysTraced,
                             "unconverged_samples": plain.unconvergedSamples,
                             "note": "uniform start points in every prism (legacy estimator), same batch size"},
            "unconverged_samples": unconverged,
            "grid_proposal": {
                "time_to_threshold_ms": statistics.median(r.totalMilliseconds for r in grid_runs),
                "weights_ms": statistics.median(r.importanceMilliseconds for r in grid_runs),
                "ray_ms": statistics.median(r.rayMilliseconds for r in grid_runs),
                "rays": grid_runs[-1].raysTraced, "unconverged_samples": grid_runs[-1].unconvergedSamples,
                "speedup_vs_walks": statistics.median(steps_ms) / statistics.median(r.totalMilliseconds for r in grid_runs),
                "note": "the same 1,024-sample batch with the coarse-grid proposal (gain-grid weights with per-bounce "
                        "total reflection instead of the importance walks); device time of calc_phi_ase"},
            "e2e": {"value": e2e_solved_all / e2e_max, "unit": "samples/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "rays_per_s": e2e_rays_all / e2e_max},
            "gpu_launches": launches,
            "roofline": {"bound": "fp32_issue" if r_fp32 <= r_l2 else "l2_gather", "kernel": "rayKernel",
                         "achieved": achieved, "peak": roof, "unit": "crossings/s", "frac": achieved / roof,
                         "traffic": None, "fp32_issue_peak": r_fp32, "l2_gather_peak": r_l2,
                         "l2_read_gbs_live": l2, "clock_mhz": f_clk / 1e6, "peak_source": peak_kind},
            "importance_roofline": {"bound": "fp32_issue" if r_fp32 <= r_l2 else "l2_gather",
                                    "kernel": "importanceTeamKernel" if tuned.importanceLayers == 0
                                    else f"importanceKernel<{tuned.importanceLayers}>",
                                    "achieved": imp_crossings / (imp_ms * 1e-3), "peak": roof, "unit": "crossings/s",
                                    "frac": imp_crossings / (imp_ms * 1e-3) / roof,
                                    "fp32_issue_frac": imp_crossings / (imp_ms * 1e-3) / r_fp32,
                                    "crossings_per_step": imp_crossings / args.steps,
                                    "ms_per_step": imp_ms / args.steps,
                                    "walks_per_step": B * mesh.numberOfPrisms * (5 if w.useReflections else 1),
                                    "note": "crossings: per (sample, slice, prism) line, triangles crossed by its "
                                            "2-D projection plus level planes and reflections (in-kernel counter)"},
            "clocks": clocks,
            "wall_s": wall,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if fwd is not None:
            line["forward_tet4"] = fwd
    ctx.close()
    return line if rank == 0 else None


def forward_cpu_baseline(tet, sa, se, seconds):
    """Forward oracle (FP64, OpenMP over all host threads) on a bounded number
    of source rays of the same Tet4 medium, sized to about `seconds`."""
    from oracle import oracle

    cores = os.cpu_count() or 1
    rays = 200_000
    while True:
        t0 = time.perf_counter()
        r = oracle.forward_phi_ase(tet, (sa, se), minRays=rays, seed=4, threads=cores)
        dt = time.perf_counter() - t0
        if dt >= seconds / 3 or rays >= 50_000_000:
            break
        rays = int(min(rays * max(2.0, min(8.0, seconds / max(dt, 1e-3) / 2)), 50_000_000))
    return {"value": rays / dt, "unit": "rays/s", "cores": cores, "kind": "port",
            "sample": f"{rays} source rays of one launch on the Tet4 medium ({tet.numberOfCells} cells, table build "
                      f"included), "
                      f"{dt:.1f} s on {cores} threads", "launches": int(r["launches"])}


def measure_forward(args, local, rank=0, world=1, cpu_seconds=None):
    """Forward Tet4 path: steps of `--forward-rays` source rays on the Tet4
    twin of the workload medium; device time (CUDA events in the library),
    L2 flushed before every timed step; e2e through the public API with the
    step's beta uploaded from the host and the per-cell results read back."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from haseongpu_b200 import TetDeviceMesh, TetMesh, _native
    from haseongpu_b200.configs import WORKLOADS

    w = WORKLOADS["disc_poly" if args.workload == "learned" else args.workload]()
    tet = TetMesh.fromPrismMesh(w.mesh)
    sa, se = w.spectra.resampled(w.monochromatic)
    dev = torch.device("cuda", local)
    flush = torch.empty(64 << 20, dtype=torch.int32, device=dev)
    ctx = TetDeviceMesh(tet, sa, se, device=local)
    rays = int(args.forward_rays)

    def step(k, beta=None):
        if beta is not None:
            ctx.update_beta(beta)
        return ctx.calc_phi_ase(forwardRayCount=rays, rngSeed=1000 + k * world + rank, monochromatic=w.monochromatic,
                                tallyMode=args.tally)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for k in range(args.warmup):
        step(k)
    barrier()
    dev_ms = ray_ms = 0.0
    cross = traced = launches = 0
    tally = 0
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            r = step(args.warmup + k)
            dev_ms += r.totalMilliseconds
            ray_ms += r.rayMilliseconds
            cross += r.crossings
            traced += r.raysTraced
            launches += r.kernelLaunches + 1
            tally = r.tallyMode
        barrier()
    clocks = clk.summary()
    betas = [np.ascontiguousarray(tet.betaVolume * (1.0 + 0.01 * k)) for k in range(args.steps)]
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        step(args.warmup + k, beta=betas[k])
    barrier()
    e2e_s = time.perf_counter() - t0
    ctx.update_beta(tet.betaVolume)
    srm = None
    if w.useReflections and tet.cellFaceBoundaries is not None:
        # surface-reservoir reflections: every reflected pass relaunches the
        # launch's source-ray count, so a smaller launch keeps the step short
        srm_rays = max(1, rays // 8)
        kw = dict(forwardRayCount=srm_rays, monochromatic=w.monochromatic, tallyMode=args.tally, useReflections=True)
        for k in range(2):
            ctx.calc_phi_ase(rngSeed=50 + k, **kw)
        torch.cuda.synchronize()
        s_ms = s_ray = 0.0
        s_cross = 0
        res_s = None
        for k in range(2):
            flush.zero_()
            torch.cuda.synchronize()
            res_s = ctx.calc_phi_ase(rngSeed=60 + k, **kw)
            s_ms += res_s.totalMilliseconds
            s_ray += res_s.rayMilliseconds
            s_cross += res_s.crossings
        srm = {"source_rays_per_step": srm_rays, "ms_per_step": s_ms / 2, "status": res_s.srmStatus,
               "passes": res_s.srmPasses, "remaining_fraction": res_s.srmRemainingFraction,
               "reflecting_faces": res_s.reflectingFaces, "crossings_per_s": s_cross / (s_ray * 1e-3),
               "kernel_launches_per_step": res_s.kernelLaunches,
               "note": "source pass + reflected passes of the same ray count; crossings of all passes"}
    ctx.close()
    stats = torch.tensor([dev_ms, e2e_s, float(traced), float(cross), ray_ms], dtype=torch.float64, device=dev)
    if world > 1:
        mx, sm = stats.clone(), stats.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        dev_ms_max, e2e_max, traced_all, cross_all = float(mx[0]), float(mx[1]), float(sm[2]), float(sm[3])
    else:
        dev_ms_max, e2e_max, traced_all, cross_all = dev_ms, e2e_s, float(traced), float(cross)
    peaks, peak_kind = measured_peaks()
    f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    r_fp64 = SMS * FP64_LANES_PER_SM * f_clk / FP64_INSTR_PER_TET_CROSSING
    l2 = _native.l2_bandwidth(local)
    r_l2 = l2 * 1e9 / BYTES_PER_TET_CROSSING
    achieved = cross / (ray_ms * 1e-3)
    roof = min(r_fp64, r_l2)
    out = {
        "value": traced_all / (dev_ms_max * 1e-3), "unit": "rays/s", "ms_per_step": dev_ms_max / args.steps,
        "crossings_per_s": cross_all / (dev_ms_max * 1e-3), "crossings_per_ray": cross / max(traced, 1),
        "config": {"workload": f"{w.name} Tet4 twin", "cells": tet.numberOfCells, "points": tet.numberOfPoints,
                   "wavelengths": int(len(sa)), "rays_per_step_per_gpu": rays, "batches": 8,
                   "tally": {1: "device-memory atomics", 2: "shared-memory vertex histogram"}.get(tally),
                   "l2": "flushed (256 MiB write) before every timed step"},
        "e2e": {"value": traced_all / e2e_max, "unit": "rays/s", "h2d_bytes_per_step": tet.numberOfCells * 8,
                "d2h_bytes_per_step": tet.numberOfCells * (4 + 8 + 8 + 4 + 4)},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64_issue" if r_fp64 <= r_l2 else "l2_gather", "kernel": "fwdRayKernel",
                     "achieved": achieved, "peak": roof, "unit": "crossings/s", "frac": achieved / roof,
                     "traffic": FWD_TRAFFIC_DISC_POLY if w.name == "disc_poly" else None,
                     "traffic_note": "resident tables read once per launch; independent of the ray count",
                     "fp64_issue_peak": r_fp64, "l2_gather_peak": r_l2, "l2_read_gbs_live": l2,
                     "clock_mhz": f_clk / 1e6, "peak_source": peak_kind},
        "clocks": clocks,
    }
    if srm is not None:
        out["srm_reflections"] = srm
    if cpu_seconds and world == 1:
        out["cpu_baseline"] = forward_cpu_baseline(tet, sa, se, cpu_seconds)
    return out


def run_forward(args):
    import torch
    import torch.distributed as dist

    from haseongpu_b200 import build as _build

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    _build.build_library()
    f = measure_forward(args, local, rank, world, cpu_seconds=args.cpu_seconds)
    if rank == 0:
        line = {"metric": FWD_METRIC, "value": f["value"], "unit": "rays/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": f["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded gain medium, no dataset)"}
        line.update({k: v for k, v in f.items() if k not in line})
        line["config"]["parallelism"] = f"independent ray launches x{world}"
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


MEDIA_METRIC = ("batched phi-ASE over 64 independent gain media (config 3) with the learned proposal to per-sample "
                "relative error <= threshold on 1 B200, as sample points solved per second (rays/s alongside; "
                "importance-weighted batched, sequential and plain importance sampling beside it)")


def measure_media(args, local, steps, warmup):
    """Config 3: 64 seeded media (triangles 200..20,000, levels 5..40, 1..8
    wavelengths), a seeded block of ``--media-samples`` sample points per
    medium, rays 1e4 -> 1e7, relative error 0.001.  Untimed: a proposal
    network trained on 24 other seeded media of the family.  Timed (one graph
    per solve: pooled proposal or importance weights, one persistent ray
    launch per pass over all media): the learned proposal + batching (the
    value), the importance weights with near-field start points + batching,
    the same media solved one after another (identical rays), and the
    reference's plain importance sampling one medium after another."""
    import numpy as np
    import torch

    from haseongpu_b200 import DeviceMesh, MediaBatch, _native
    from haseongpu_b200 import learned as LP
    from haseongpu_b200.autotune import autotune_batch
    from haseongpu_b200.batch import solve_sequential
    from haseongpu_b200.configs import media64, media_training

    w = media64()
    ctxs = [DeviceMesh(m.mesh, *m.spectra.resampled(False), device=local) for m in w.media]
    rng = np.random.default_rng(5)
    K = args.media_samples
    items = []
    for c in ctxs:
        S = c.mesh.numberOfSamples
        lo = int(rng.integers(0, max(1, S - K)))
        items.append((c, lo, min(S - 1, lo + K - 1)))
    rows = sum(hi - lo + 1 for _, lo, hi in items)
    flush = torch.empty(64 << 20, dtype=torch.int32, device=torch.device("cuda", local))
    ws = 32 << 30
    t0 = time.perf_counter()
    trainers = [DeviceMesh(m.mesh, *m.spectra.resampled(False), device=local) for m in media_training()]
    data = LP.training_set_media(trainers, samples_per_medium=16, rays=100_000)
    t1 = time.perf_counter()
    net, hist = LP.train_proposal(data, steps=3000, device=local)
    t2 = time.perf_counter()
    for c in trainers:
        c.close()
    batch = MediaBatch(local)
    tune = autotune_batch(batch, items, rays=100_000, repeats=3, workspaceBytes=ws)
    kw = dict(minRays=w.minRays, maxRays=w.maxRays, mseThreshold=w.threshold, adaptiveSteps=w.adaptiveSteps,
              monochromatic=False, workspaceBytes=ws, rayKernelVariant=tune.rayKernelVariant,
              raysPerThread=tune.raysPerThread)

    def timed(fn):
        out, st_all = [], []
        for s_ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            res, st = fn(1000 + 64 * s_)
            out.append(res)
            st_all.append(st)
        return out, st_all

    # the plain method judges the learned proposal: the largest per-ray variance
    # the importance weights reached on the logged training samples
    fallback = data.fallback_limit(1.0)
    for k in range(warmup):
        batch.solve(items, rngSeed=100 + 64 * k, net=net, fallbackVariance=fallback, **kw)
        batch.solve(items, rngSeed=100 + 64 * k, **kw)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        lt, lst = timed(lambda seed: batch.solve(items, rngSeed=seed, net=net, fallbackVariance=fallback, **kw))
        bt, bst = timed(lambda seed: batch.solve(items, rngSeed=seed, **kw))
        for c in ctxs:  # the coarse-grid proposal for every medium, same batched graph
            c.set_grid_proposal(True)
        try:
            batch.solve(items, rngSeed=999, **kw)  # warm-up: each medium's gain grid is built once per beta
            gt, gst = timed(lambda seed: batch.solve(items, rngSeed=seed, **kw))
        finally:
            for c in ctxs:
                c.set_grid_proposal(False)
    clocks = clk.summary()
    seq_ms, wall_s, same = 0.0, 0.0, True
    for s_ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        t_s = time.perf_counter()
        seq = solve_sequential(items, rngSeed=1000 + 64 * s_, **kw)
        wall_s += time.perf_counter() - t_s
        seq_ms += sum(r.totalMilliseconds for r in seq)
        same = same and all(np.array_equal(a.phiAse, b.phiAse) for a, b in zip(bt[s_], seq))
    # the reference's estimator (importance weights, uniform start points) on
    # the same media, one medium after another: the plain importance-sampled
    # GPU path
    plain_ms, plain_rays, plain_unconv, plain_var = 0.0, 0, 0, None
    pkw = dict(kw, rayKernelVariant=0, raysPerThread=0, nearFieldSampling=False)
    for s_ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        pr = solve_sequential(items, rngSeed=1000 + 64 * s_, **pkw)
        plain_ms += sum(r.totalMilliseconds for r in pr)
        plain_rays += sum(r.raysTraced for r in pr)
        plain_unconv += sum(r.unconvergedSamples for r in pr)
        plain_var = np.concatenate([LP.per_ray_variance(r) for r in pr])
    # e2e: beta of every medium uploaded from host and every result read back, each step
    betas = [c.mesh.betaVolume for c in ctxs]
    torch.cuda.synchronize()
    te = time.perf_counter()
    for s_ in range(steps):
        for c, b in zip(ctxs, betas):
            c.update_beta(b)
        batch.solve(items, rngSeed=1000 + 64 * s_, net=net, fallbackVariance=fallback, **kw)
    e2e_s = time.perf_counter() - te

    def agg(st_all):
        return {"ms": sum(st.totalMilliseconds for st in st_all), "ray_ms": sum(st.rayMilliseconds for st in st_all),
                "imp_ms": sum(st.importanceMilliseconds for st in st_all),
                "rays": sum(st.raysTraced for st in st_all), "cross": sum(st.crossings for st in st_all),
                "unconverged": sum(st.unconvergedSamples for st in st_all),
                "capture_ms": sum(st.captureMilliseconds for st in st_all)}

    L, B, G = agg(lst), agg(bst), agg(gst)
    gv = np.concatenate([LP.per_ray_variance(r) for r in gt[-1]])
    lv = np.concatenate([LP.per_ray_variance(r) for r in lt[-1]])
    nv = np.concatenate([LP.per_ray_variance(r) for r in bt[-1]])
    peaks, peak_kind = measured_peaks()
    f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
    r_fp32 = SMS * LANES_PER_SM * f_clk / FP32_INSTR_PER_CROSSING
    l2 = _native.l2_bandwidth(local)
    r_l2 = l2 * 1e9 / BYTES_PER_CROSSING
    roof = min(r_fp32, r_l2)
    per_ray = np.concatenate([r.totalRays.astype(np.int64) for r in lt[-1]])
    out = {
        "value": steps * rows / (L["ms"] * 1e-3), "unit": "samples/s", "ms_per_step": L["ms"] / steps,
        "rays_per_s": L["rays"] / (L["ms"] * 1e-3), "crossings_per_s": L["cross"] / (L["ray_ms"] * 1e-3),
        "config": {"workload": "media64 (config 3): 64 seeded gain media in one batched solve, learned proposal",
                   "media": len(ctxs), "samples_per_medium": K, "samples_per_step": rows,
                   "triangles": [min(c.mesh.numberOfTriangles for c in ctxs),
                                 max(c.mesh.numberOfTriangles for c in ctxs)],
                   "levels": [min(c.mesh.numberOfLevels for c in ctxs), max(c.mesh.numberOfLevels for c in ctxs)],
                   "prisms_total": sum(c.mesh.numberOfPrisms for c in ctxs),
                   "wavelengths": [m.wavelengths for m in w.media], "rays_per_sample": [w.minRays, w.maxRays],
                   "threshold": w.threshold, "adaptive_steps": w.adaptiveSteps,
                   "l2": "flushed (256 MiB write) before every timed step",
                   "ray_kernel": {"variant": tune.name, "rays_per_lane": tune.raysPerThread,
                                  "autotuned_over": len(tune.table)}},
        "breakdown_ms_per_step": {"proposal_and_mixture": L["imp_ms"] / steps,
                                  "map_ray_finalise_passes": L["ray_ms"] / steps,
                                  "graph_capture_host": L["capture_ms"] / steps},
        "rays_per_sample": {"min": int(per_ray.min()), "median": float(np.median(per_ray)), "max": int(per_ray.max())},
        "unconverged_samples": L["unconverged"],
        "fallback": {"per_ray_variance_limit": fallback, "samples": sum(st.fallbackSamples for st in lst),
                     "rule": "first-pass per-ray variance above the largest the importance weights reached on "
                             "the logged training samples"},
        "per_ray_variance": {"learned_median": float(np.median(lv)), "learned_max": float(lv.max()),
                             "importance_nearfield_median": float(np.median(nv)),
                             "importance_nearfield_max": float(nv.max()),
                             "plain_is_median": float(np.median(plain_var)), "plain_is_max": float(plain_var.max())},
        "training": {"media": 24, "samples_per_medium": 16, "groups": data.groups, "rows": int(data.offsets[-1]),
                     "rays_logged": data.groups * data.rays, "log_s": t1 - t0, "train_s": t2 - t1,
                     "loss_first_50": float(hist[:50].mean()), "loss_last_200": float(hist[-200:].mean()),
                     "note": "24 media of the same generator on another seed (<= 3,000 triangles); the timed media "
                             "are unseen"},
        "grid_batched": {"value": steps * rows / (G["ms"] * 1e-3), "unit": "samples/s", "ms_per_step": G["ms"] / steps,
                         "weights_ms_per_step": G["imp_ms"] / steps, "rays": G["rays"],
                         "unconverged_samples": G["unconverged"], "median_per_ray_variance": float(np.median(gv)),
                         "speedup_vs_learned_batched": L["ms"] / G["ms"],
                         "note": "the coarse-grid proposal for every medium (no walks, no network), near-field "
                                 "start points, the same batched graph"},
        "importance_batched": {"value": steps * rows / (B["ms"] * 1e-3), "unit": "samples/s",
                               "ms_per_step": B["ms"] / steps, "rays": B["rays"],
                               "unconverged_samples": B["unconverged"],
                               "note": "importance weights with near-field start points, the same batched graph"},
        "importance_sequential": {"ms_per_step": seq_ms / steps, "wall_ms_per_step": wall_s * 1e3 / steps,
                                  "identical_to_batched": bool(same),
                                  "note": "the same media, one calc_phi_ase per medium (host-synchronised passes)"},
        "plain_is_sequential": {"value": steps * rows / (plain_ms * 1e-3), "unit": "samples/s",
                                "ms_per_step": plain_ms / steps, "rays": plain_rays,
                                "unconverged_samples": plain_unconv,
                                "note": "the reference's importance weights with uniform start points, one medium "
                                        "after another"},
        "speedup_vs_plain_is_sequential": plain_ms / L["ms"],
        "speedup_vs_importance_batched": B["ms"] / L["ms"],
        "speedup_batched_vs_sequential": seq_ms / B["ms"],
        "e2e": {"value": steps * rows / e2e_s, "unit": "samples/s",
                "h2d_bytes_per_step": sum(c.mesh.numberOfPrisms * 8 for c in ctxs),
                "d2h_bytes_per_step": rows * (4 + 8 + 8 + 4 + 8 + 4)},
        "gpu_launches": sum(st.kernelLaunches for st in lst),
        "graph": {"kernels": lst[-1].kernelLaunches, "nodes": lst[-1].graphNodes, "chunks": lst[-1].chunks},
        "roofline": {"bound": "fp32_issue" if r_fp32 <= r_l2 else "l2_gather", "kernel": "rayKernel (pooled)",
                     "achieved": L["cross"] / (L["ray_ms"] * 1e-3), "peak": roof, "unit": "crossings/s",
                     "frac": L["cross"] / (L["ray_ms"] * 1e-3) / roof, "traffic": None, "peak_source": peak_kind,
                     "note": "ray time includes the map and finalise launches of every pass"},
        "clocks": clocks,
    }
    batch.close()
    net.close()
    for c in ctxs:
        c.close()
    return out


def run_media(args):
    """Config 3 on its own line; with N ranks every rank solves its own copy
    of the 64 media (replicas), timed as the maximum over ranks."""
    import torch
    import torch.distributed as dist

    rank, world, local = setup_ranks()
    m = measure_media(args, local, args.steps, args.warmup)
    ms = torch.tensor([m["ms_per_step"]], dtype=torch.float64, device=torch.device("cuda", local))
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms[0])
    if rank == 0:
        rows = m["config"]["samples_per_step"]
        line = {"metric": MEDIA_METRIC, "value": world * rows / (ms_max * 1e-3), "unit": "samples/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 geometry, f64 sums", "data": "synthetic (seeded gain media, no dataset)"}
        line.update({k: v for k, v in m.items() if k not in ("value", "ms_per_step")})
        print(json.dumps(line), flush=True)
    teardown_ranks(world)


PULSE_METRIC = ("pump-pulse time series (config 5): 50 rate-equation steps of a 1 ms pump with a forward phi-ASE "
                "solve (surface-reservoir reflections) per step on 1 B200, as time steps per second")


def measure_pulse(args, local):
    """Config 5 at its stated size: the ~20,000-triangle x 30-level disc (its
    Tet4 twin: 1.64 M cells), 8 wavelengths, reflectivity 0.3 / 0.9 with
    total internal reflection, beta from 0 through a 1 ms pump in 50 steps;
    every step one forward solve of ``--pulse-rays`` source rays with the
    surface-reservoir passes, then the pump and the RK4 rate-equation update
    on the device.  Timed: the whole series (device time of the solves and of
    the pump/update kernels).  After it, one more forward solve at the final
    beta reports the per-cell relative error that budget reaches."""
    import numpy as np
    import torch

    from haseongpu_b200 import DeviceMesh, TetDeviceMesh, TetMesh
    from haseongpu_b200.configs import pulse

    w = pulse()
    sa, se = w.spectra.resampled(False)
    tet = TetMesh.fromPrismMesh(w.mesh)
    rays = int(args.pulse_rays)
    kw = dict(forwardRayCount=rays, monochromatic=False, useReflections=True)
    with DeviceMesh(w.mesh, sa, se, device=local) as ctx, TetDeviceMesh(tet, sa, se, device=local) as twin:
        warm = dict(w.time, steps=3, pumpSteps=3, aseSteps=3)
        ctx.simulate_forward(twin, pump=w.pump, time=warm, rngSeed=7, **kw)
        ctx.update_beta(w.mesh.betaVolume)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = ctx.simulate_forward(twin, pump=w.pump, time=w.time, rngSeed=11, **kw)
        wall = time.perf_counter() - t0
        final = twin.calc_phi_ase(forwardRayCount=rays, rngSeed=13, monochromatic=False, useReflections=True)
    gain = out["betaVolume"] > 0
    rse = np.repeat(final.relativeStandardError.reshape(-1, 3).max(axis=1), 1)[gain]
    return {
        "value": w.time["steps"] / (out["totalMilliseconds"] * 1e-3), "unit": "time steps/s",
        "ms_per_series": out["totalMilliseconds"], "wall_ms_per_series": wall * 1e3,
        "ase_ms": out["aseMilliseconds"], "pump_and_update_ms": out["pumpMilliseconds"],
        "rays_per_s": out["raysTraced"] / (out["aseMilliseconds"] * 1e-3),
        "source_rays": out["raysTraced"],
        "config": {"workload": "pulse (config 5): disc of 18,816 triangles x 30 levels, Tet4 twin 1,636,992 cells",
                   "wavelengths": int(len(sa)), "reflectivity": [0.3, 0.9], "steps": w.time["steps"],
                   "time_step_s": w.time["timeStep"], "pump_s": w.time["timeStep"] * w.time["pumpSteps"],
                   "forward_rays_per_step": rays, "phi_method": "forward Tet4 with surface-reservoir reflections"},
        "mean_beta": {"start": float(out["meanBeta"][0]), "mid": float(out["meanBeta"][25]),
                      "end": float(out["meanBeta"][-1])},
        "mean_phi_end": float(out["meanPhi"][-1]),
        "pump_absorbed_fraction_end": float(out["pumpAbsorbed"][-1]),
        "final_solve": {"srm_status": final.srmStatus, "srm_passes": final.srmPasses,
                        "median_cell_rse_gain": float(np.median(rse)) if rse.size else None,
                        "ms": final.totalMilliseconds, "crossings_per_s": final.crossings / (final.rayMilliseconds * 1e-3)},
    }


def _rse_summary(res, rays):
    import numpy as np

    g = res.phiAse > 0
    r = res.relativeStandardError[g]
    return {"rays_per_sample": rays, "median_sample_rse": float(np.median(r)), "p90_sample_rse": float(np.percentile(r, 90)),
            "max_sample_rse": float(r.max()), "per_ray_variance_median": float(np.median(rays * r ** 2)),
            "ms": res.totalMilliseconds}


# far-prior share of the config-5 backward series: at the end-of-pump beta the
# per-ray variance of the local proposal (K = 16) is 0.215 at 0.97 against 0.28 at 0.9
FAR_SHARE = 0.97


def measure_pulse_backward(args, local):
    """Config 5 with the backward method: every time step solves all 287,310
    sample points (9,577 points x 30 levels) with the local proposal (per
    point its ``--pulse-local-triangles`` nearest triangles x 29 layers x 5
    slices weighted by the importance walks, FAR_SHARE of the rays from the
    far beta V gain / d^2 prior; unbiased mixture weights), ``--pulse-backward-rays``
    rays per sample, 8 wavelengths, reflections.  Two series of 50 steps:
    the plain local proposal (device time of hase_simulate) and the learned
    proposal warm-started from step to step (fine-tuned before every step
    on the contributions the importance-weighted method logs for a block of
    32 sample points, plain importance weights as the fallback above the
    per-ray variance the logged block reached).  Then at the plain series'
    final beta: the per-sample error the budget reaches, and an adaptive
    solve to relative error 1e-3 of 2,048 sample points (a block of the
    middle level) whose device time, scaled to all sample points, is the
    cost of one time step at the stated accuracy."""
    import time as clock

    import numpy as np

    from haseongpu_b200 import DeviceMesh
    from haseongpu_b200.configs import pulse
    from haseongpu_b200.learned import warm_started_series
    from haseongpu_b200.proposal import ProposalNet

    w = pulse()
    sa, se = w.spectra.resampled(False)
    rays, K = int(args.pulse_backward_rays), int(args.pulse_local_triangles)
    S = w.mesh.numberOfSamples
    out = {"config": {"local_triangles": K, "far_fraction": FAR_SHARE, "rays_per_sample_and_step": rays, "samples": S,
                      "steps": w.time["steps"], "wavelengths": int(len(sa)), "phi_method": "backward, local proposal"}}
    with DeviceMesh(w.mesh, sa, se, device=local) as ctx:
        ctx.set_local_proposal(K, FAR_SHARE)
        ctx.calc_phi_ase(minRays=1000, useReflections=True, minSample=0, maxSample=63)  # candidate tables
        t0 = clock.perf_counter()
        ser = ctx.simulate(pump=w.pump, time=w.time, minRays=rays, useReflections=True, rngSeed=11)
        wall = clock.perf_counter() - t0
        fin = ctx.calc_phi_ase(minRays=rays, useReflections=True, rngSeed=13)
        first = (w.mesh.numberOfLevels // 2) * w.mesh.numberOfPoints
        thr = ctx.calc_phi_ase(minRays=16000, maxRays=4_000_000, mseThreshold=1e-3, adaptiveSteps=6,
                               useReflections=True, rngSeed=17, minSample=first, maxSample=first + 2047)
        out["plain_local"] = {
            "ms_per_series": ser["totalMilliseconds"], "wall_ms_per_series": wall * 1e3,
            "value": w.time["steps"] / (ser["totalMilliseconds"] * 1e-3), "unit": "time steps/s",
            "ase_ms": ser["aseMilliseconds"], "rays_traced": ser["raysTraced"],
            "mean_beta_end": float(ser["meanBeta"][-1]), "mean_phi_end": float(ser["meanPhi"][-1]),
            "final_beta_solve": _rse_summary(fin, rays)}
        out["to_rse_1e-3"] = {
            "samples": 2048, "ms": thr.totalMilliseconds, "unconverged": thr.unconvergedSamples,
            "mean_rays_per_sample": float(thr.totalRays.mean()),
            "median_sample_rse": float(np.median(thr.relativeStandardError)),
            "ms_per_time_step_all_samples": thr.totalMilliseconds * S / 2048.0,
            "note": "adaptive 16,000 -> 4e6 rays (6 increases) at the series' final beta; scaled by samples"}
    with DeviceMesh(w.mesh, sa, se, device=local) as ctx, ProposalNet(device=local, seed=3) as net:
        ctx.set_local_proposal(K, FAR_SHARE)
        ctx.calc_phi_ase(minRays=1000, useReflections=True, minSample=0, maxSample=63)
        t0 = clock.perf_counter()
        ws = warm_started_series(ctx, net, w.pump, w.time, rays=rays, rngSeed=11, fallback="logged")
        wall = clock.perf_counter() - t0
        fin = ctx.calc_phi_ase_learned(net, minRays=rays, useReflections=True, rngSeed=13)
        out["learned_warm_started"] = {
            "ms_per_series": ws["totalMilliseconds"], "wall_ms_per_series": wall * 1e3,
            "value": w.time["steps"] / (ws["totalMilliseconds"] * 1e-3), "unit": "time steps/s",
            "fine_tune_s": ws["trainSeconds"], "fallback_samples": ws["fallbackSamples"],
            "mean_beta_end": ws["meanBeta"][-1], "mean_phi_end": ws["meanPhi"][-1],
            "loss_last": ws["loss"][-1] if ws["loss"] else None,
            "final_beta_solve": _rse_summary(fin, rays),
            "note": "device time of the 50 hase_simulate steps; fine-tuning and logging are host-timed (fine_tune_s)"}
    return out


def run_pulse(args):
    """Config 5 on its own line; with N ranks every rank runs its own series
    (replicas), timed as the maximum over ranks."""
    import torch
    import torch.distributed as dist

    rank, world, local = setup_ranks()
    m = measure_pulse(args, local)
    m["backward"] = measure_pulse_backward(args, local)
    ms = torch.tensor([m["ms_per_series"]], dtype=torch.float64, device=torch.device("cuda", local))
    if world > 1:
        dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms_max = float(ms[0])
    if rank == 0:
        steps = m["config"]["steps"]
        line = {"metric": PULSE_METRIC, "value": world * steps / (ms_max * 1e-3), "unit": m["unit"], "n_gpus": world,
                "steps": 1, "warmup": 1, "ms_per_step": ms_max, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 walk and sums",
                "data": "synthetic (seeded gain medium and pump, no dataset)"}
        line.update({k: v for k, v in m.items() if k not in ("value", "unit")})
        print(json.dumps(line), flush=True)
    teardown_ranks(world)


LEARNED_METRIC = ("phi-ASE time to per-sample relative error <= threshold with the learned proposal, as sample points "
                  "solved per second (plain importance sampling on the same fields beside it; rays/s alongside)")


def run_learned(args):
    """Config 4: the learned proposal on the disc_small geometry.  Untimed:
    logging 32 seeded training fields with the importance weights and
    training the network (Adam, device).  Timed: each step solves every
    sample point of one unseen pump field to the threshold (rays 1e5 -> 1e6,
    relative error 0.005) with the learned proposal; the same fields are then
    solved with the reference's plain importance sampling (uniform start
    points) and with the importance weights + near-field start points."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from haseongpu_b200 import DeviceMesh, _native
    from haseongpu_b200 import learned as LP
    from haseongpu_b200.configs import disc_small

    rank, world, local = setup_ranks()
    dev = torch.device("cuda", local)
    w = disc_small()
    mesh = w.mesh
    sa, se = w.spectra.resampled(True)
    S = mesh.numberOfSamples
    ctx = DeviceMesh(mesh, sa, se, device=local)
    flush = torch.empty(64 << 20, dtype=torch.int32, device=dev)  # 256 MiB > 126 MB L2

    t0 = time.perf_counter()
    data = LP.training_set(ctx, LP.pump_fields(mesh, 32, LP.TRAIN_SEED))
    t1 = time.perf_counter()
    net, hist = LP.train_proposal(data, steps=3000, device=local)
    t2 = time.perf_counter()
    fields = LP.pump_fields(mesh, args.warmup + args.steps, LP.EVAL_SEED + 7919 * rank)
    # launch shape of the ray kernel and importance layers: the project's
    # autotuner on this geometry (untimed), shared by every arm
    from haseongpu_b200.autotune import autotune, pinned

    ctx.update_beta(fields[0])
    if args.ray_variant:
        tuned = pinned(args.ray_variant, args.rays_per_lane)
    else:
        tuned = autotune(ctx, firstSample=0, samples=min(S, 1024), rays=w.minRays, useReflections=False,
                         monochromatic=True, device=local)
    kw = dict(minRays=w.minRays, maxRays=w.maxRays, mseThreshold=w.threshold, adaptiveSteps=w.adaptiveSteps,
              monochromatic=True, minSample=0, maxSample=S - 1, rayKernelVariant=tuned.rayKernelVariant,
              raysPerThread=tuned.raysPerThread)
    ikw = dict(importanceLayers=tuned.importanceLayers)

    # the plain method judges the learned proposal: a sample whose first-pass
    # per-ray variance exceeds the worst the importance weights reached on the
    # logged training samples restarts with the importance weights
    fallback = data.fallback_limit(1.0)

    def solve(kind, k):
        ctx.update_beta(fields[k])
        if kind == "learned":
            return ctx.calc_phi_ase_learned(net, rngSeed=3000 + k, fallbackVariance=fallback, **kw)
        if kind == "grid":  # the coarse-grid proposal: weights from the gain grid, no walks, no network
            ctx.set_grid_proposal(True)
            try:
                return ctx.calc_phi_ase(rngSeed=3000 + k, **kw)
            finally:
                ctx.set_grid_proposal(False)
        return ctx.calc_phi_ase(rngSeed=3000 + k, nearFieldSampling=(kind == "nearfield"), **kw, **ikw)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for k in range(args.warmup):
        solve("learned", k)
    barrier()
    acc = {"learned": [], "plain": [], "nearfield": [], "grid": []}
    with ClockSampler(local) as clk:
        for kind in ("learned", "plain", "nearfield", "grid"):
            for s_ in range(args.steps):
                ctx.update_beta(fields[args.warmup + s_])
                flush.zero_()
                torch.cuda.synchronize()
                acc[kind].append(solve(kind, args.warmup + s_))
        barrier()
    clocks = clk.summary()
    # e2e: the public API with host buffers (beta upload and per-sample results read back every step)
    barrier()
    te = time.perf_counter()
    for s_ in range(args.steps):
        solve("learned", args.warmup + s_)
    barrier()
    e2e_s = time.perf_counter() - te

    def agg(rs):
        ms = sum(r.totalMilliseconds for r in rs)
        return {"ms": ms, "rays": sum(r.raysTraced for r in rs), "crossings": sum(r.crossings for r in rs),
                "ray_ms": sum(r.rayMilliseconds for r in rs), "proposal_ms": sum(r.importanceMilliseconds for r in rs),
                "unconverged": sum(r.unconvergedSamples for r in rs), "launches": sum(r.kernelLaunches + 1 for r in rs)}

    a = {k: agg(v) for k, v in acc.items()}
    stats = torch.tensor([a["learned"]["ms"], a["plain"]["ms"], a["nearfield"]["ms"], e2e_s,
                          float(a["learned"]["rays"]), float(args.steps * S), a["grid"]["ms"]], dtype=torch.float64,
                         device=dev)
    if world > 1:
        mx, sm = stats.clone(), stats.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        ms_l, ms_p, ms_n, e2e_max = float(mx[0]), float(mx[1]), float(mx[2]), float(mx[3])
        rays_all, solved_all = float(sm[4]), float(sm[5])
        ms_g = float(mx[6])
    else:
        ms_l, ms_p, ms_n, e2e_max = a["learned"]["ms"], a["plain"]["ms"], a["nearfield"]["ms"], e2e_s
        ms_g = a["grid"]["ms"]
        rays_all, solved_all = float(a["learned"]["rays"]), float(args.steps * S)
    disc_poly = fwd = media = pulse_line = None
    if world == 1 and not args.no_nested:
        import argparse as _ap

        nargs = _ap.Namespace(**vars(args))
        nargs.workload, nargs.samples = "disc_poly", 1024
        nargs.steps, nargs.warmup = max(2, min(args.steps, 3)), max(args.warmup, 3)
        disc_poly = measure_importance(nargs, local, rank, world, nested=True)
        media = measure_media(nargs, local, steps=2, warmup=3)
        pulse_line = measure_pulse(nargs, local)
        # the backward series at a quarter of the pulse workload's budget
        # (--workload pulse runs --pulse-backward-rays)
        bargs = _ap.Namespace(**vars(nargs))
        bargs.pulse_backward_rays = max(1, args.pulse_backward_rays // 4)
        pulse_line["backward"] = measure_pulse_backward(bargs, local)
        fwd = measure_forward(nargs, local, cpu_seconds=min(args.cpu_seconds, 6.0))
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        f_clk = float(peaks.get("sm_max_mhz", 1965.0)) * 1e6
        r_fp32 = SMS * LANES_PER_SM * f_clk / FP32_INSTR_PER_CROSSING
        l2 = _native.l2_bandwidth(local)
        r_l2 = l2 * 1e9 / BYTES_PER_CROSSING
        roof = min(r_fp32, r_l2)
        achieved = a["learned"]["crossings"] / (a["learned"]["ray_ms"] * 1e-3)
        rows = args.steps * S * mesh.numberOfPrisms
        prop_tflops = rows * MLP_FLOP_PER_PAIR / (a["learned"]["proposal_ms"] * 1e-3) / 1e12
        bf16 = float(peaks.get("bf16_tflops", 1590.0))
        lv = np.concatenate([LP.per_ray_variance(r) for r in acc["learned"]])
        pv = np.concatenate([LP.per_ray_variance(r) for r in acc["plain"]])
        nv = np.concatenate([LP.per_ray_variance(r) for r in acc["nearfield"]])
        gv = np.concatenate([LP.per_ray_variance(r) for r in acc["grid"]])
        cpu = cpu_baseline(w, args.cpu_seconds, fields=fields[args.warmup:]) if world == 1 else None
        l1 = _native.l1_bandwidth(local)
        smem = _native.l1_bandwidth(local, shared=True)
        r_l1 = l1 * 1e9 / BYTES_PER_CROSSING
        line = {
            "metric": LEARNED_METRIC,
            "value": solved_all / (ms_l * 1e-3),
            "unit": "samples/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_l / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 geometry, f64 sums, bf16 proposal network (f32 accumulation)",
            "data": "synthetic (seeded gain media and pump fields, no dataset)",
            "config": learned_config(w, mesh, world),
            "ray_kernel": {"variant": tuned.name, "rays_per_lane": tuned.raysPerThread,
                           "importance_layers": tuned.importanceLayers, "autotuned_over": len(tuned.table)},
            "time_to_threshold_ms": ms_l / args.steps,
            "plain_is": {"value": solved_all / (ms_p * 1e-3), "unit": "samples/s", "ms_per_step": ms_p / args.steps,
                         "rays": a["plain"]["rays"], "unconverged_samples": a["plain"]["unconverged"],
                         "median_per_ray_variance": float(np.median(pv)), "max_per_ray_variance": float(pv.max()),
                         "note": "the reference's importance weights with uniform start points (legacy estimator)"},
            "importance_nearfield": {"value": solved_all / (ms_n * 1e-3), "unit": "samples/s",
                                     "ms_per_step": ms_n / args.steps, "rays": a["nearfield"]["rays"],
                                     "unconverged_samples": a["nearfield"]["unconverged"],
                                     "median_per_ray_variance": float(np.median(nv))},
            "grid_proposal": {"value": solved_all / (ms_g * 1e-3), "unit": "samples/s", "ms_per_step": ms_g / args.steps,
                              "rays": a["grid"]["rays"], "unconverged_samples": a["grid"]["unconverged"],
                              "weights_ms_per_step": a["grid"]["proposal_ms"] / args.steps,
                              "median_per_ray_variance": float(np.median(gv)), "speedup_vs_learned": ms_l / ms_g,
                              "note": "importance weights from the coarse gain grid (no walks, no network), "
                                      "near-field start points; the same fields"},
            "learned": {"rays": a["learned"]["rays"], "unconverged_samples": a["learned"]["unconverged"],
                        "median_per_ray_variance": float(np.median(lv)), "max_per_ray_variance": float(lv.max()),
                        "proposal_ms_per_step": a["learned"]["proposal_ms"] / args.steps,
                        "ray_ms_per_step": a["learned"]["ray_ms"] / args.steps,
                        "training": {"groups": data.groups, "rows": int(data.offsets[-1]),
                                     "rays_logged": data.groups * data.rays, "log_s": t1 - t0, "train_s": t2 - t1,
                                     "adam_steps": 3000, "loss_first_50": float(hist[:50].mean()),
                                     "loss_last_200": float(hist[-200:].mean())},
                        "speedup_vs_plain_is": ms_p / ms_l, "speedup_vs_importance_nearfield": ms_n / ms_l,
                        "fallback": {"per_ray_variance_limit": fallback,
                                     "samples": sum(r.fallbackSamples for r in acc["learned"]),
                                     "rule": "first-pass per-ray variance above the largest the importance weights "
                                             "reached on the logged training samples"}},
            "rays_per_s": rays_all / (ms_l * 1e-3),
            "e2e": {"value": solved_all / e2e_max, "unit": "samples/s", "h2d_bytes_per_step": mesh.numberOfPrisms * 8,
                    "d2h_bytes_per_step": S * (4 + 8 + 8 + 4 + 8 + 4)},
            "gpu_launches": a["learned"]["launches"],
            "roofline": {"bound": "fp32_issue" if r_fp32 <= r_l2 else "l2_gather", "kernel": tuned.name,
                         "achieved": achieved, "peak": roof, "unit": "crossings/s", "frac": achieved / roof,
                         "traffic": RAY_TRAFFIC_LEARNED,
                         "traffic_note": "DRAM bytes per launch (ncu): the per-sample ray maps read once and the "
                                         "per-item partial sums; the walk tables stay in L1 (99 % hits) and L2",
                         "fp32_issue_peak": r_fp32, "l2_gather_peak": r_l2, "l1_gather_peak": r_l1,
                         "fp32_issue_frac": achieved / r_fp32, "l1_gather_frac": achieved / r_l1,
                         "l2_read_gbs_live": l2, "l1_read_gbs_live": l1, "smem_read_gbs_live": smem,
                         "binding": RAY_BINDING_LEARNED, "ncu_thread_instructions": RAY_INSTR_LEARNED,
                         "clock_mhz": f_clk / 1e6, "peak_source": peak_kind},
            "proposal_roofline": {"bound": "xu", "kernel": "proposalKernel",
                                  "achieved": rows / (a["learned"]["proposal_ms"] * 1e-3),
                                  "peak": SMS * XU_LANES_PER_SM * f_clk / XU_INSTR_PER_PAIR, "unit": "pairs/s",
                                  "frac": rows / (a["learned"]["proposal_ms"] * 1e-3)
                                  / (SMS * XU_LANES_PER_SM * f_clk / XU_INSTR_PER_PAIR),
                                  "tensor_tflops": prop_tflops, "tensor_frac_of_bf16": prop_tflops / bf16,
                                  "flop_per_pair": MLP_FLOP_PER_PAIR, "xu_instr_per_pair": XU_INSTR_PER_PAIR,
                                  "pairs": rows, "peak_source": peak_kind},
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if disc_poly is not None:
            line["importance_disc_poly"] = {k: disc_poly[k] for k in (
                "value", "unit", "ms_per_step", "config", "time_to_threshold_ms", "breakdown_ms_per_step",
                "rays_per_s", "crossings_per_s", "plain_method", "unconverged_samples", "grid_proposal", "e2e", "roofline",
                "importance_roofline")}
        if fwd is not None:
            line["forward_tet4"] = fwd
        if pulse_line is not None:
            line["pulse_time_series"] = pulse_line
        if media is not None:
            line["batched_media"] = {k: media[k] for k in (
                "value", "unit", "ms_per_step", "config", "rays_per_s", "crossings_per_s", "breakdown_ms_per_step",
                "rays_per_sample", "unconverged_samples", "fallback", "per_ray_variance", "training", "grid_batched",
                "importance_batched",
                "importance_sequential", "plain_is_sequential", "speedup_vs_plain_is_sequential",
                "speedup_vs_importance_batched", "speedup_batched_vs_sequential", "graph", "e2e", "roofline")}
            line["learned_batched_target"] = {
                "target": "learned proposal + persistent batching >= 5x less time to every sample's threshold than "
                          "the plain importance-sampled GPU path",
                "workload": "media64 (config 3), unseen media",
                "learned_batched_ms": media["ms_per_step"],
                "plain_is_sequential_ms": media["plain_is_sequential"]["ms_per_step"],
                "plain_is_unconverged_samples_per_step": media["plain_is_sequential"]["unconverged_samples"] / 2,
                "learned_batched_unconverged_samples_per_step": media["unconverged_samples"] / 2,
                "samples_per_step": media["config"]["samples_per_step"],
                "ratio": media["speedup_vs_plain_is_sequential"],
                "met": bool(media["speedup_vs_plain_is_sequential"] >= 5.0)}
        print(json.dumps(line), flush=True)
    net.close()
    ctx.close()
    teardown_ranks(world)


def run_reference(args):
    """The reference arm: the reference's method (importance weights, uniform
    start points) in its CPU restatement, the oracle, on all host threads
    (rank 0 only), on the same workload as this build's arm.  For the learned
    workload each step solves a bounded sample of the sample points of the
    same unseen evaluation pump field this build's rank 0 solves in that
    step, with the same rays and threshold, and the line carries this build's
    config."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return
    from haseongpu_b200.configs import WORKLOADS, disc_small

    per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
    if args.workload == "learned":
        from haseongpu_b200 import learned as LP

        w = disc_small()
        fields = LP.pump_fields(w.mesh, args.warmup + args.steps, LP.EVAL_SEED)
        for k in range(args.warmup):
            cpu_baseline(w, 0.0, fields=[fields[k]])
        vals = [cpu_baseline(w, per_step, fields=[fields[args.warmup + k]]) for k in range(args.steps)]
        config, metric = learned_config(w, w.mesh, args.gpus), LEARNED_METRIC
    else:
        w = WORKLOADS[args.workload]()
        for _ in range(args.warmup):
            cpu_baseline(w, 0.0)
        vals = [cpu_baseline(w, per_step) for _ in range(args.steps)]
        config, metric = {"workload": w.name, "threshold": w.threshold, "reflections": w.useReflections}, METRIC
    value = statistics.median(v["value"] for v in vals)
    cores = vals[0]["cores"]
    line = {
        "metric": metric, "value": value, "unit": "samples/s",
        "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded gain medium and pump fields, no dataset)",
        "impl": "reference", "config": config,
        "rays_per_s": statistics.median(v["rays_per_s"] for v in vals),
        "cpu_baseline": {"value": value, "unit": "samples/s", "cores": cores, "kind": "port",
                         "sample": vals[0]["sample"]},
        "e2e": {"value": value, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.path == "forward":
        run_forward(args)
    elif args.workload == "learned":
        run_learned(args)
    elif args.workload == "media64":
        run_media(args)
    elif args.workload == "pulse":
        run_pulse(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
