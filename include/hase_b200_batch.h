/*
 * hase_b200_batch.h -- many gain media in one phi-ASE solve of
 * libhase_b200.so.
 *
 * The reference serves one mesh per calcPhiASE call and spreads the sample
 * points of that mesh over devices (MPI ranks or host threads:
 * include/core/forwardPhiAseEvaluator.hpp:302-339, calcPhiAseMpi.hpp).  Here
 * the sample points of many independent gain media (each a hase_context:
 * its own mesh, beta and spectrum) share one device:
 *
 *   - the importance weights of every medium are computed into one pooled
 *     workspace (one importance launch per medium);
 *   - every adaptive pass maps the rays of all still-active sample points and
 *     walks them in ONE persistent ray launch, whose warps take work items
 *     (a run of rays of one sample point of one medium) from one global
 *     queue, so media of a few hundred prisms and of a million prisms fill
 *     the GPU together and the uneven per-sample budgets of the adaptive
 *     passes balance across media;
 *   - the active counts stay on the device (map, ray and finalise launches
 *     read them there), so the whole adaptive schedule is one captured CUDA
 *     graph without a host synchronisation between passes.
 *
 * Each medium's rays use the Philox key (rngSeed + instance index, 0): the
 * result of instance i is bit-identical to hase_calc_phi_ase on its context
 * with compute.rngSeed = rngSeed + i and the same sample range, experiment
 * and launch shape.
 */
#ifndef HASE_B200_BATCH_H
#define HASE_B200_BATCH_H

#include "hase_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hase_batch hase_batch;

/* One gain medium of a batch: its context (all contexts on the batch's
 * device), its inclusive sample range (maxSample UINT32_MAX = last sample) and
 * caller-allocated result arrays of (maxSample - minSample + 1) entries.  The
 * scalar fields of result are filled per medium (raysTraced, crossings,
 * unconvergedSamples, passes); the millisecond fields and kernelLaunches
 * carry the whole batch's figures. */
typedef struct {
    hase_context* context;
    uint32_t minSample;
    uint32_t maxSample;
    hase_result* result;
} hase_batch_instance;

typedef struct {
    uint64_t raysTraced;
    uint64_t crossings;
    uint32_t rows;                      /* sample points solved */
    uint32_t chunks;                    /* workspace chunks (one graph launch each) */
    uint32_t passes;                    /* adaptive passes that had active samples */
    uint32_t unconvergedSamples;
    uint32_t kernelLaunches;            /* kernel nodes of the graphs launched */
    uint32_t graphNodes;                /* all nodes (kernels, memsets, copies, events) */
    double importanceMilliseconds;      /* device time (events inside the graphs) */
    double rayMilliseconds;             /* map + ray + finalise launches of all passes */
    double totalMilliseconds;           /* graph launch to completion, all chunks */
    double captureMilliseconds;         /* host time spent capturing and instantiating graphs */
    double setupMilliseconds;           /* host time before the first graph launch (tables, views, uploads) */
    double hostMilliseconds;            /* host time of the whole call */
    uint32_t fallbackSamples;           /* learned solve: samples that restarted with the importance weights */
} hase_batch_stats;

hase_status hase_batch_create(int device, hase_batch** out);
hase_status hase_batch_destroy(hase_batch* batch);

/* Solves every instance's sample range to experiment->mseThreshold (shared
 * ray schedule minRays -> maxRays over compute->adaptiveSteps passes).  Of
 * compute, adaptiveSteps, rngSeed, raysPerThread, workspaceBytes,
 * rayKernelVariant (hase_ray_kernel_variant_name) and importanceLayers are
 * used; minSample / maxSample come from the instances.  Returns
 * HASE_DROPPED_RAYS / HASE_NOT_CONVERGED as hase_calc_phi_ase does, over the
 * whole batch.  stats may be NULL. */
hase_status hase_calc_phi_ase_batch(hase_batch* batch, const hase_batch_instance* instances, uint32_t count,
                                    const hase_experiment_desc* experiment, const hase_compute_desc* compute,
                                    hase_batch_stats* stats);

struct hase_proposal; /* include/hase_b200_proposal.h */

/* The same batched solve with the learned proposal of `net` (on the batch's
 * device) in place of every medium's importance weights:
 * q = (1 - mixture) softmax(network logits) + mixture (beta V R_j / d^2
 * prior), mixture 0 = 0.1, one network for all media (its features are
 * normalised by each medium's radius and height).  fallbackVariance > 0:
 * after the first pass, every sample still above the threshold whose per-ray
 * relative variance (rays x relative error^2) exceeds it restarts with the
 * importance weights, on the device (hase_learned_desc.fallbackVariance).
 * Medium i equals hase_calc_phi_ase_learned on its context with seed
 * rngSeed + i. */
hase_status hase_calc_phi_ase_batch_learned(hase_batch* batch, const hase_batch_instance* instances, uint32_t count,
                                            const hase_experiment_desc* experiment, const hase_compute_desc* compute,
                                            struct hase_proposal* net, float mixture, float fallbackVariance,
                                            hase_batch_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* HASE_B200_BATCH_H */
