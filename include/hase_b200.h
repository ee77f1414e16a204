/*
 * hase_b200.h -- C ABI of libhase_b200.so, the B200 (sm_100a) implementation
 * of HASEonGPU's adaptive Monte Carlo phi-ASE computation on extruded
 * triangle-prism meshes (backward, importance-sampled method).
 *
 * Plain C types only; no exceptions cross this boundary.  Every entry point
 * returns a hase_status; on failure hase_last_error_message() (thread-local)
 * says why.  One context per host thread / stream; calls on one context must
 * be serialised by the caller.
 *
 * What each entry point replaces in HASEonGPU v2.2.0 (paths inside the
 * reference project):
 *   hase_context_create       - HostMesh construction + device upload
 *                               (include/core/mesh.hpp:509-768,
 *                                include/core/forwardPhiAseEvaluator.hpp:184-204)
 *   hase_context_update_beta  - dynamic beta update without re-sending topology
 *                               (ForwardPhiAseDeviceContext::rebuildBetaVolumePrefix,
 *                                include/core/calcForwardPhiAse.hpp:337-380)
 *   hase_calc_phi_ase         - hase::core::startSimulation<false>(experiment,
 *                               compute, result, mesh)
 *                               (include/core/simulation.hpp:42-47), i.e. the
 *                               calcPhiASE entry point behind PhiASE.run
 *                               (pyInclude/simulation.py:452-483)
 *   hase_result               - hase::core::Result (include/core/types.hpp:201-246)
 *   hase_experiment_desc      - hase::core::ExperimentParameters
 *                               (include/core/types.hpp:248-331)
 *   hase_compute_desc         - hase::core::ComputeParameters (adaptiveSteps,
 *                               repetitions, rngSeed, sample range)
 */
#ifndef HASE_B200_H
#define HASE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HASE_B200_ABI_VERSION 2

typedef enum {
    HASE_OK = 0,
    HASE_INVALID_ARGUMENT = 1, /* std::invalid_argument / std::out_of_range in the reference */
    HASE_CUDA_ERROR = 2,       /* a CUDA runtime call failed */
    HASE_OUT_OF_MEMORY = 3,
    HASE_DEVICE_TIMEOUT = 4,   /* a bounded device wait gave up */
    HASE_DROPPED_RAYS = 5,     /* warning: some rays could not be walked (counted in droppedRays) */
    HASE_NOT_CONVERGED = 6,    /* warning: some samples stayed above the MSE threshold at maxRays */
    HASE_NO_DEVICE = 7         /* no CUDA device (the reference returns non-zero when no backend matched) */
} hase_status;

typedef struct hase_context hase_context;

/* Extruded triangle-prism gain medium (legacy HASEonGPU mesh layout).
 * Prism (triangle t, layer l) has index t + l * numberOfTriangles; sample
 * point (point p, level l) has index p + l * numberOfPoints. */
typedef struct {
    uint32_t numberOfPoints;            /* 2-D mesh points */
    uint32_t numberOfTriangles;         /* T */
    uint32_t numberOfLevels;            /* z levels (>= 2); layers = levels - 1 */
    const double* points;               /* [numberOfPoints][2] x, y (cm) */
    const uint32_t* triangles;          /* [T][3] point indices */
    double thickness;                   /* level spacing (cm) */
    const double* betaVolume;           /* [levels-1][T] excited fraction per prism */
    const double* betaCells;            /* [levels][numberOfPoints] per sample point (dndt only); may be NULL */
    const uint32_t* claddingCellTypes;  /* [T] or NULL */
    uint32_t claddingNumber;            /* triangles with this type are cladding */
    double claddingAbsorption;          /* cladding absorption coefficient (cm^-1) */
    double nTot;                        /* doping density (cm^-3) */
    double crystalTFluo;                /* fluorescence lifetime (s) */
    const double* reflectivities;       /* [T][2]: t*2+0 bottom, t*2+1 top; NULL = 0 */
    const double* refractiveIndices;    /* [4]: bottom inside, bottom outside, top inside, top outside; NULL = 1 */
} hase_mesh_desc;

/* Cross sections on a common wavelength grid.  phi-ASE is the mean over the
 * wavelengths: every ray of a polychromatic solve contributes its gain
 * averaged over all of them (its walk keeps the path integrals every
 * wavelength's exponent is linear in), so no wavelength is drawn per ray. */
typedef struct {
    uint32_t numberOfWavelengths;       /* >= 1 */
    const double* sigmaA;               /* absorption cross sections (cm^2) */
    const double* sigmaE;               /* emission cross sections (cm^2) */
} hase_spectrum_desc;

typedef struct {
    uint32_t minRays;                   /* rays per sample in the first pass */
    uint32_t maxRays;                   /* cap of the adaptive schedule */
    double mseThreshold;                /* stop when the relative standard error <= this */
    uint32_t useReflections;            /* 0/1: top/bottom reflections of order <= 2 */
    uint32_t monochromatic;             /* 1: use only the first (sigmaA, sigmaE) pair */
    uint32_t nearFieldSampling;         /* 1: solid-angle start points in the prisms touching the sample
                                           (bounded weights); 0: uniform start points in every prism, as
                                           the legacy method */
} hase_experiment_desc;

typedef struct {
    uint32_t adaptiveSteps;             /* geometric ray-target increases minRays -> maxRays */
    uint32_t repetitions;               /* accepted for interface compatibility (passes pool their rays) */
    uint32_t rngSeed;
    uint32_t minSample;                 /* inclusive */
    uint32_t maxSample;                 /* inclusive; UINT32_MAX = last sample */
    uint32_t raysPerThread;             /* rays per lane of a ray-kernel work item (item = 32 x this);
                                           0 = default (1024-ray items) */
    uint32_t blockSize;                 /* 0 = default / autotuned */
    uint64_t workspaceBytes;            /* 0 = default device workspace budget */
    uint32_t rayKernelVariant;          /* launch shape of the ray kernel, 0 = default; see
                                           hase_ray_kernel_variant_name (chosen by the autotuner) */
    uint32_t importanceLayers;          /* importance kernel: 0 = line teams (a team of lanes per (sample,
                                           triangle) shares the 2-D walk); 2, 4, 8 = that many prism layers
                                           per thread; the same weights either way */
} hase_compute_desc;

/* Caller-allocated host arrays of (maxSample - minSample + 1) entries; any
 * pointer may be NULL to skip that output. */
typedef struct {
    float* phiAse;
    double* standardError;
    double* relativeStandardError;      /* the legacy "mse" */
    uint32_t* totalRays;
    double* dndtAse;
    uint32_t* droppedRays;
    /* scalar outputs */
    uint64_t raysTraced;
    uint64_t crossings;                 /* prism crossings walked by the ray kernel */
    double importanceMilliseconds;      /* device time, CUDA events */
    double rayMilliseconds;
    double totalMilliseconds;
    uint32_t passes;
    uint32_t unconvergedSamples;
    uint32_t kernelLaunches;            /* kernels this call launched */
} hase_result;

const char* hase_last_error_message(void);
const char* hase_status_string(hase_status status);
int hase_abi_version(void);
/* Launch shapes of the ray kernel (hase_compute_desc.rayKernelVariant). */
int hase_ray_kernel_variant_count(void);
const char* hase_ray_kernel_variant_name(uint32_t variant);

hase_status hase_context_create(const hase_mesh_desc* mesh, const hase_spectrum_desc* spectrum, int device,
                                hase_context** out);
hase_status hase_context_update_beta(hase_context* ctx, const double* betaVolume, const double* betaCells);
hase_status hase_calc_phi_ase(hase_context* ctx, const hase_experiment_desc* experiment,
                              const hase_compute_desc* compute, hase_result* result);
hase_status hase_context_destroy(hase_context* ctx);

/* Local proposal for media too large for a weight per (sample, slice,
 * prism) pair (no reference counterpart; the reference weights every prism).
 * With triangles = K > 0, every backward solve of the context (plain or
 * learned), hase_importance_weights, hase_learned_weights,
 * hase_log_contributions and hase_proposal_features use per sample point its
 * K nearest triangles (by centroid distance) x layers x slices as the
 * candidate entries of the weight rows (entry j (layers K) + l K + k).  A
 * fraction farFraction (0: 0.9) of each pass's rays is drawn instead from a
 * prior over every (slice, prism): beta V times a two-point gain estimate
 * over the squared distance to the slice's image of the sample point, on a
 * grid of about 8 triangles per cell.  Each ray is weighted by the mixture
 * of both sources' probabilities, so the estimate is unbiased with O(K)
 * weights per sample instead of O(prisms).  Logged contributions
 * (hase_log_contributions) are those of every ray in a candidate prism.
 * triangles = 0 restores the full proposal; triangles >= the mesh's
 * triangles uses every triangle as a candidate and no far rays.  Batched
 * media (hase_calc_phi_ase_batch) reject a context in local mode. */
hase_status hase_context_set_local_proposal(hase_context* ctx, uint32_t triangles, float farFraction);

/* Coarse-grid proposal (no reference counterpart; the reference walks every
 * (sample, slice, prism) line for its importance weights).  With enable = 1
 * the context's plain backward solves (hase_calc_phi_ase, hase_simulate)
 * take their weights from the importance function beta V R / d^2 e^G with
 * the straight-line gain G estimated on the coarse gain grid of the learned
 * proposal's features (8 points along the line, reflections folded) instead
 * of a walk, and the reflection factor R of a slice taken per bounce from the
 * pair's own direction: 1 beyond the surface's critical angle, its mean
 * reflectivity otherwise.  Any positive proposal leaves the estimate unbiased;
 * this one costs a fraction of the walks.  With the local proposal set, it
 * weights the candidate rows; a batched solve without a network uses it for
 * the media whose context has it set.  Learned solves keep the network's
 * weights.  enable = 0 restores the walks. */
hase_status hase_context_set_grid_proposal(hase_context* ctx, uint32_t enable);

/* ---- kernel-level entry points (the four hot-path kernels, one at a time) ----
 * Used by the parity tests and the benchmark; no reference counterpart beyond
 * the kernels they expose (importance weights, ray->prism map, ray walk). */

/* Normalised importance weights (max 1) for samples [firstSample, firstSample+count):
 * weights[i][j*P + p] for reflection slice j (slices = 5 with reflections, else 1). */
hase_status hase_importance_weights(hase_context* ctx, uint32_t firstSample, uint32_t count,
                                    uint32_t useReflections, float* weights);

/* The coarse-grid proposal's normalised weights (max 1), laid out as those of
 * hase_importance_weights (the local proposal's candidate rows when it is
 * set); monochromatic: the grid of the first wavelength pair, else of the
 * spectral mean. */
hase_status hase_grid_weights(hase_context* ctx, uint32_t firstSample, uint32_t count, uint32_t useReflections,
                              uint32_t monochromatic, float* weights);

/* Crossings of the importance walks of samples [firstSample, firstSample +
 * count): per (sample, reflection slice, prism) line, the triangles its 2-D
 * projection crosses plus the level planes and reflections on the way -- the
 * work unit of the importance kernel's roofline (counted by an instrumented
 * copy of the kernel; the walks are those of hase_calc_phi_ase). */
hase_status hase_importance_crossings(hase_context* ctx, uint32_t firstSample, uint32_t count,
                                      uint32_t useReflections, uint64_t* crossings);

/* The prism walk records hase_context_create builds on the host (no device
 * needed; the reference derives the same neighbour table in
 * pyInclude/geometry/core.py:733 _derived_topology): per triangle 12 floats, the outward
 * unit normal and line constant (nx, ny, c) of its three edges followed by
 * the three neighbour codes as int bits (neighbour << 2 | the edge's index in
 * the neighbour, -1 at the mesh boundary), edge e joining the triangle's
 * points e and e + 1.  `tri` receives the records as given, `walk` the walks'
 * copy with NaN normals on the boundary edges; either may be NULL. */
hase_status hase_mesh_tables(const hase_mesh_desc* mesh, float* tri, float* walk);

/* Ray->prism map of `rows` weight rows of length n: q[row][n] (quantised
 * weights), offsets[row][n+1] (exclusive ray offsets), Q[row]. */
hase_status hase_ray_map(uint32_t rows, uint32_t n, const float* weights, uint32_t rays, const uint32_t* phases,
                         uint32_t* q, uint32_t* offsets, uint64_t* Q);

/* ln(gain) and distance of explicit rays from start[i] (x,y,z) in prism
 * (tri[i], level[i]) to sample[i] through reflection slice[i] at wavelength
 * index `wavelength`. dropped[i] = 1 if the walk failed. */
hase_status hase_trace_rays(hase_context* ctx, uint32_t n, const float* start, const uint32_t* tri,
                            const uint32_t* level, const uint32_t* sample, const uint32_t* slice,
                            uint32_t wavelength, float* lnGain, float* distance, uint32_t* dropped);

/* Allocation-free estimate of one sample point (no counterpart in the
 * reference).  For callers that must not allocate device memory -- real-time
 * loops whose memory is fixed up front (a cudaMalloc can block and
 * synchronise the device mid-loop), or hosts that reserve the device's memory
 * and hand it out only through their own pool -- this entry point calls no
 * cudaMalloc/cudaFree and no allocating library routine.  The caller passes device pointers:
 * `deviceWeights` [slices * prisms] non-negative importance weights (slices =
 * 5 with reflections, else 1; e.g. from hase_importance_weights) and
 * `deviceResult` [4] doubles receiving phiAse, relative standard error, rays
 * and dropped rays.  One pass of `rays` rays over all wavelengths of the
 * context, like hase_calc_phi_ase with minRays = maxRays = rays for that
 * single sample.  Scratch lives in a fixed ~4.2 MiB device array inside the
 * library, so slices * prisms may be at most 524,288 (larger meshes are
 * rejected with HASE_INVALID_ARGUMENT).  The first call on a device looks up
 * the array's device address; make that first call before any stream
 * capture.  All calls on one device share the array: calls that overlap on
 * the GPU (other host threads, other contexts on the same device) race and
 * must be serialised by the caller.  It synchronises the context's stream
 * and returns once the result is written. */
hase_status hase_estimate_sample_noalloc(hase_context* ctx, uint32_t sample, const float* deviceWeights, uint32_t rays,
                                         uint32_t rngSeed, uint32_t useReflections, uint32_t nearFieldSampling,
                                         double* deviceResult);

/* ---- time-stepped rate equations (pump pulse, fluorescence, ASE) ----
 * Replaces the reference's compiled time loop, hase::core time-stepped
 * simulation (include/core/timeSteppedSimulation.hpp:132-617, stages
 * include/kernels/timeIntegrationUpdateKernels.hpp:21-127, derivative
 * include/kernels/derivativeComposition.hpp:27-93), on the prism mesh:
 *   d beta/dt = pump(beta) - [beta (sigma_e + sigma_a) - sigma_a] Phi - beta / tau
 * per gain prism (cladding prisms keep their beta), Phi the prism's mean
 * phi-ASE over its six vertices, the ASE cross sections the first pair
 * (monochromatic) or the largest pair.  The pump is a collimated
 * super-Gaussian beam entering the bottom surface along +z (the reference
 * example's SurfacePumpInjector with a collimated angular distribution),
 * optionally retro-reflected at the top: per triangle column an exact
 * Beer-Lambert integration with g_p = N_tot [beta (sigma_a + sigma_e) -
 * sigma_a] at the pump wavelength, absorbed photons / (N_tot h) per layer
 * (cladding prisms attenuate with claddingAbsorption). */
typedef struct {
    double peakIntensity;       /* W/cm^2 at the profile centre */
    double radius;              /* super-Gaussian radius (cm) */
    double exponent;            /* super-Gaussian exponent */
    double centerX;             /* profile centre (cm) */
    double centerY;
    double wavelength;          /* pump wavelength (m): photon energy h c / lambda */
    double sigmaA;              /* pump cross sections (cm^2) */
    double sigmaE;
    uint32_t retroreflect;      /* 1: the beam returns down from the top surface */
} hase_pump_desc;

typedef struct {
    double timeStep;            /* s */
    uint32_t steps;             /* simulation steps */
    uint32_t pumpSteps;         /* steps with the pump on, from the first */
    uint32_t aseSteps;          /* steps with a phi-ASE solve, from the first (0: pump and fluorescence only) */
    uint32_t integrator;        /* the reference's time integrators (include/core/timeSteppedSimulation.hpp:321-415):
                                   0 frozen-phi-ase-runge-kutta-4 (phi-ASE solved at the step start only),
                                   1 explicit-euler, 2 heun, 3 midpoint, 4 runge-kutta-4,
                                   5 implicit-euler (fixed-point iterations), 6 exponential-euler;
                                   2, 3, 4 and 5 re-solve phi-ASE at every stage they evaluate */
    uint32_t implicitIterations; /* implicit-euler iterations (0: the reference's default, 8) */
} hase_time_desc;

typedef struct {
    double* betaVolume;         /* out [prisms] beta after the last step, or NULL */
    double* meanBeta;           /* out [steps + 1] mean beta of the gain prisms, or NULL */
    double* meanPhi;            /* out [steps] mean phi-ASE of the samples (0 without a solve), or NULL */
    double* pumpAbsorbed;       /* out [steps] absorbed fraction of the pump power (first stage), or NULL */
    float* phiHistory;          /* out [aseSteps x solves per step][samples] phi-ASE of every solve, in order,
                                   or NULL; solves per step: 1 (integrators 0, 1, 6), 2 (2, 3), 4 (4),
                                   implicitIterations (5) */
    double aseMilliseconds;     /* device time of the phi-ASE solves */
    double pumpMilliseconds;    /* device time of pump, derivative and stage kernels */
    double totalMilliseconds;
    uint64_t raysTraced;
    uint32_t fallbackSamples;
} hase_time_result;

/* `proposal` (hase_b200_proposal.h): NULL solves with the importance
 * weights; otherwise with the learned proposal (its fallback limit
 * `fallbackVariance`).  The context's beta is advanced in place. */
struct hase_proposal;
hase_status hase_simulate(hase_context* ctx, struct hase_proposal* proposal, float fallbackVariance,
                          const hase_experiment_desc* experiment, const hase_compute_desc* compute,
                          const hase_pump_desc* pump, const hase_time_desc* time, hase_time_result* result);

/* Measurement support (no reference counterpart): L2 read bandwidth of
 * `device` in GB/s, from `reps` passes over an L2-resident buffer of `bytes`. */
hase_status hase_probe_l2_bandwidth(int device, uint64_t bytes, uint32_t reps, double* gbPerSecond);

/* Measured L1 (sharedMemory = 0) or shared-memory (1) read bandwidth of the
 * whole device in GB/s: two 1024-thread blocks per SM read a resident 32 KB
 * `reps` times with 16-byte loads (the on-chip bound of a walk whose tables
 * stay in L1 or shared memory). */
hase_status hase_probe_l1_bandwidth(int device, uint32_t sharedMemory, uint32_t reps, double* gbPerSecond);

/* Philox4x32-10 on the device: out[i] = philox(ctr[i], key). */
hase_status hase_philox(uint32_t n, const uint32_t* ctr, const uint32_t key[2], uint32_t* out);

#ifdef __cplusplus
}
#endif

#endif /* HASE_B200_H */
