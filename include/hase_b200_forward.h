/*
 * hase_b200_forward.h -- C ABI of the forward Tet4 phi-ASE path of
 * libhase_b200.so: HASEonGPU v2.2.0's current calcPhiASE method (source rays
 * drawn from the excited volume, walked out of a tetrahedral mesh, their
 * track-length tallies collected at the mesh vertices), on sm_100a.
 *
 * Same conventions as hase_b200.h (whose hase_status, hase_spectrum_desc,
 * hase_last_error_message and hase_status_string this header reuses): plain
 * C types, no exceptions across the boundary, one context per host thread,
 * calls on one context serialised by the caller.
 *
 * What each entry point replaces in the reference (paths inside its tree):
 *   hase_tet_context_create      - Tet4 HostMesh construction, barycentric
 *                                  face planes and neighbour tables, device
 *                                  upload (include/core/mesh.hpp:509-768,
 *                                  :657-727; DeviceMeshContainer and
 *                                  ForwardPhiAseDeviceContext,
 *                                  include/core/calcForwardPhiAse.hpp:61-130)
 *   hase_tet_context_update_beta - ForwardPhiAseDeviceContext::rebuildBetaVolumePrefix
 *                                  (include/core/calcForwardPhiAse.hpp:337-380)
 *   hase_tet_calc_phi_ase        - the forward evaluator behind
 *                                  hase::core::startSimulation<false>
 *                                  (include/core/forwardPhiAseEvaluator.hpp:114-178,
 *                                  kernels include/kernels/forward/accumulation.hpp:369-453
 *                                  and include/kernels/forwardPhiAseMapping.hpp:51-150)
 *   hase_forward_result          - the forward fields of hase::core::Result
 *                                  (include/core/types.hpp:201-246): phiAse,
 *                                  relative standard error, dndtAse,
 *                                  totalRays (= cell ray visits,
 *                                  include/core/calcForwardPhiAse.hpp:258),
 *                                  droppedRays
 *   useReflections (SRM)         - the surface-reservoir reflection passes
 *                                  (include/core/forwardSrm.hpp:100-365,
 *                                  include/kernels/forward/accumulation.hpp:455-833,
 *                                  reflectance include/kernels/reflection.hpp:21-47,
 *                                  surfaces include/core/mesh.hpp:301-332)
 *   hase_tet_trace               - one ray through the mesh, as the reference's
 *                                  traversal tests drive nextFaceIntersection /
 *                                  transitionAcrossIntersection
 *                                  (tests/forwardRayTraversal.cpp:98-153)
 */
#ifndef HASE_B200_FORWARD_H
#define HASE_B200_FORWARD_H

#include "hase_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hase_tet_context hase_tet_context;

/* Tet4 gain medium.  Local face f of a cell is the face opposite its vertex f. */
typedef struct {
    uint32_t numberOfPoints;
    uint32_t numberOfCells;
    const double* points;               /* [numberOfPoints][3] x, y, z (cm) */
    const uint32_t* cells;              /* [numberOfCells][4] point indices */
    const double* betaVolume;           /* [numberOfCells] excited fraction per cell */
    const uint32_t* claddingCellTypes;  /* [numberOfCells] or NULL */
    uint32_t claddingNumber;            /* cells with this type are cladding */
    double claddingAbsorption;          /* cladding absorption coefficient (cm^-1) */
    double nTot;                        /* doping density (cm^-3) */
    double crystalTFluo;                /* fluorescence lifetime (s) */
    /* Reflecting boundary surfaces (used with hase_forward_desc.useReflections).
     * A boundary face whose surface id is > 0 reflects: its reflectivity is
     * surfaceReflectivities[id] when id < numberOfSurfaces, else the legacy
     * reflectivities[cell * 2 + face % 2] (0 when NULL); its refractive
     * indices likewise come from the per-surface arrays or the legacy
     * refractiveIndices[2 * (face % 2)] (inside) and [2 * (face % 2) + 1]
     * (outside), 1 when NULL.  Total internal reflection (reflectance 1) when
     * (n_in / n_out)^2 sin^2(incidence) > 1.  All pointers may be NULL. */
    const int32_t* cellFaceBoundaries;             /* [numberOfCells][4] surface id per local face */
    uint32_t numberOfSurfaces;
    const double* surfaceReflectivities;           /* [numberOfSurfaces] */
    const double* surfaceRefractiveIndexInside;    /* [numberOfSurfaces] */
    const double* surfaceRefractiveIndexOutside;   /* [numberOfSurfaces] */
    const double* reflectivities;                  /* legacy [numberOfCells][2] */
    const double* refractiveIndices;               /* legacy [4] */
} hase_tet_mesh_desc;

typedef struct {
    uint32_t forwardRayCount;           /* rays of the first launch */
    uint32_t maxRays;                   /* cap of the adaptive schedule (<= forwardRayCount: one launch) */
    uint32_t adaptiveSteps;             /* geometric increases forwardRayCount -> maxRays */
    double relativeStandardErrorThreshold; /* stop when every cell's relative error <= this */
    uint32_t monochromatic;             /* 1: use only the first (sigmaA, sigmaE) pair */
    uint32_t rngSeed;
    uint32_t batches;                   /* statistical batches of the relative error; 0 = 8, at most 64 */
    uint32_t blockSize;                 /* threads per block of the ray kernel; 0 = default */
    uint32_t tallyMode;                 /* 0 = automatic, 1 = device-memory atomics,
                                           2 = per-block shared-memory vertex tallies */
    /* Surface-reservoir method (SRM): rays leaving through a reflecting face
     * deposit weight x gain x reflectance into a per-face reservoir of
     * reflected directions; every launch then runs reflected passes of the
     * same ray count from the reservoir (start at the face centroid) until the
     * reflected weight converges, stabilises, diverges or the pass limit is
     * reached.  Every statistical batch runs its own chain. */
    uint32_t useReflections;
    uint32_t reflectionMaxIterations;   /* reflected passes per launch; 0 = 40 */
    double reflectionTolerance;         /* 0 = 1e-4 */
    uint32_t surfaceReservoirSize;      /* reservoir slots per reflecting face; 0 = 32 */
    uint32_t divergenceStreak;          /* passes of growing weight that end a chain as diverged; 0 = 3 */
} hase_forward_desc;

/* Caller-allocated host arrays of numberOfCells entries; any pointer may be
 * NULL to skip that output. */
typedef struct {
    float* phiAse;
    double* relativeStandardError;
    double* dndtAse;
    uint32_t* totalRays;                /* ray segments tallied in the cell (the reference's cell visits) */
    uint32_t* droppedRays;
    /* scalar outputs */
    uint64_t raysTraced;
    uint64_t crossings;                 /* cell crossings walked by the ray kernel */
    double rayMilliseconds;             /* device time of the ray kernels, CUDA events */
    double totalMilliseconds;
    uint32_t launches;                  /* adaptive launches */
    uint32_t unconvergedCells;
    uint32_t kernelLaunches;            /* kernels this call launched */
    uint32_t tallyMode;                 /* tally mode used (1 or 2) */
    /* SRM outputs of the last launch (include/core/types.hpp:174-246): the
     * worst status over the batches (0 disabled, 1 converged, 2 stable,
     * 3 diverged, 4 max_iterations; worst = diverged > max_iterations >
     * stable > converged), the most passes, the largest remaining fraction
     * of the first reflected weight */
    uint32_t srmStatus;
    uint32_t srmPasses;
    double srmRemainingFraction;
    uint32_t srmMaxIterations;
    uint32_t srmDivergenceStreak;
    uint32_t reflectingFaces;           /* boundary faces with a reflecting surface */
} hase_forward_result;

hase_status hase_tet_context_create(const hase_tet_mesh_desc* mesh, const hase_spectrum_desc* spectrum, int device,
                                    hase_tet_context** out);
hase_status hase_tet_context_update_beta(hase_tet_context* ctx, const double* betaVolume);
/* Sizes of the context's mesh (either pointer may be NULL). */
hase_status hase_tet_context_info(hase_tet_context* ctx, uint32_t* numberOfCells, uint32_t* numberOfPoints);
hase_status hase_tet_calc_phi_ase(hase_tet_context* ctx, const hase_forward_desc* forward,
                                  hase_forward_result* result);
hase_status hase_tet_context_destroy(hase_tet_context* ctx);

/* Device tables of the context: neighbours [C][4] (-1 at the boundary),
 * neighbour local face [C][4], face planes [C][4][4] (lambda_f(x) =
 * a.x + b.y + c.z + d; the device keeps faces 1..3, face 0 is returned as
 * lambda_0 = 1 - lambda_1 - lambda_2 - lambda_3), volumes [C].  Any pointer
 * may be NULL. */
hase_status hase_tet_tables(hase_tet_context* ctx, int32_t* neighbors, int32_t* neighborFace, double* planes,
                            double* volumes);

/* n single rays through the mesh (no tally): ray i starts at origin[i] in
 * startCell[i] along the unit direction[i].  segments[i] = cells crossed, a
 * zero-length step included; cells / lengths [n][maxSegments] the first
 * maxSegments of them (either may be NULL); lnGain[i] = sum of g l at spectral
 * pair `wavelength`; endPoint[i] where the walk stopped; status[i] 0 = left
 * the mesh, 1 = walk failed. */
hase_status hase_tet_trace(hase_tet_context* ctx, uint32_t n, const uint32_t* startCell, const double* origin,
                           const double* direction, uint32_t wavelength, uint32_t maxSegments, uint32_t* segments,
                           uint32_t* cells, double* lengths, double* lnGain, double* endPoint, int32_t* status);

/* hase_simulate (include/hase_b200.h) with the ASE term from the forward
 * method instead of the backward solve: `twin` is the Tet4 twin of the prism
 * mesh of `prism` (cell 3p + k, k < 3, belongs to prism p, the split of
 * TetMesh.fromPrismMesh).  Every ASE step copies the prisms' beta to their
 * cells, runs one forward solve with `forward` (surface-reservoir reflections
 * when forward->useReflections), and takes a prism's phi as the
 * volume-weighted mean of its three cells' phi; pump and rate equations are
 * those of hase_simulate.  result->phiHistory (may be NULL) is
 * [aseSteps][prisms]; result->meanPhi is the mean over the gain prisms. */
hase_status hase_simulate_forward(hase_context* prism, hase_tet_context* twin, const hase_forward_desc* forward,
                                  const hase_pump_desc* pump, const hase_time_desc* time, hase_time_result* result);

#ifdef __cplusplus
}
#endif

#endif /* HASE_B200_FORWARD_H */
