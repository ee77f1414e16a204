/*
 * hase_oracle.h -- CPU (FP64, OpenMP) restatement of HASEonGPU's backward,
 * importance-sampled prism phi-ASE method.  TEST INFRASTRUCTURE ONLY: the
 * product library never links or calls this code; tests, smoke() and the CPU
 * baseline leg of bench.py use it as the checker.
 *
 * The reference (HASEonGPU v2.2.0) retired the backward prism kernels; this
 * restatement follows the method as published (Eckert et al., Comput. Phys.
 * Commun. 207 (2016) 362) and the anchors that survive in the reference tree:
 *   - prism tables:        pyInclude/geometry/core.py:670-774
 *   - gain coefficient:    include/kernels/forward/rayWalk.hpp:170-182
 *   - cladding segments:   tests/data/laserPumpCladding/true_cladding_no_reflection_phiase_reference/README.md:27-33
 *   - legacy reflectivity index (cell*2 + face%2): include/core/mesh.hpp:301-332
 *   - adaptive ray target: include/core/types.hpp:333-354
 *   - dndt = (beta*(sigmaE+sigmaA) - sigmaA) * phi: include/core/forwardPhiAseUtilities.hpp:16-25
 *   - golden outputs:      tests/data/compareSerial/phiase_reference.npz,
 *                          tests/data/laserPumpCladding/true_cladding_no_reflection_phiase_reference/phiase_reference.npz
 * Parity is pinned against those golden outputs by tests/test_oracle_golden.py.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t numberOfPoints;      /* 2-D mesh points */
    uint32_t numberOfTriangles;   /* T */
    uint32_t numberOfLevels;      /* z levels; prisms = T * (levels - 1) */
    const double* points;         /* [numberOfPoints][2] x, y */
    const uint32_t* triangles;    /* [T][3] */
    double thickness;             /* level spacing h */
    const double* betaVolume;     /* [levels-1][T]: prism = t + level * T */
    const double* betaCells;      /* [levels][numberOfPoints] (dndt only), may be NULL */
    const uint32_t* claddingCellTypes; /* [T] or NULL */
    uint32_t claddingNumber;
    double claddingAbsorption;
    double nTot;
    double crystalTFluo;
    const double* reflectivities; /* [T][2]: t*2 + 0 bottom, t*2 + 1 top; NULL = 0 */
    const double* refractiveIndices; /* [4]: bottom in/out, top in/out; NULL = 1 */
} oracle_mesh;

typedef struct {
    uint32_t numberOfWavelengths;
    const double* sigmaA;
    const double* sigmaE;
} oracle_spectrum;

typedef struct {
    uint32_t minRays;
    uint32_t maxRays;
    uint32_t adaptiveSteps;
    double mseThreshold;
    uint32_t useReflections;      /* 0/1: top/bottom reflections of order <= 2 */
    uint32_t seed;
    uint32_t minSample;           /* inclusive */
    uint32_t maxSample;           /* inclusive */
    uint32_t nearField;           /* solid-angle start points in prisms touching the (image) sample */
} oracle_experiment;

typedef struct {
    double* phiAse;       /* [nSamples] */
    double* mse;          /* relative standard error of phiAse */
    uint32_t* totalRays;
    double* dndtAse;
    uint32_t* droppedRays;
    double* gainSum;      /* sum of per-ray contributions (FP64) */
    double* gainSumSquare;
} oracle_result;

/* Philox4x32-10 (Salmon et al., SC'11): out = philox(ctr, key). */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Per-triangle tables (row-major [t][e]); edge e runs from vertex e to e+1.
 * normals are outward unit normals, c = n . (edge start point). */
int oracle_build_tables(uint32_t numberOfPoints, const double* points, uint32_t numberOfTriangles,
                        const uint32_t* triangles, int32_t* neighbors, int32_t* forbiddenEdge,
                        double* normalX, double* normalY, double* edgeC, double* centerX,
                        double* centerY, double* area);

/* ln(gain) of straight rays from start (x,y,z) in prism (tri, level) to sample
 * point `sample` (index point + level * numberOfPoints) through reflection
 * slice `slice` (0 direct, 1 bottom, 2 top, 3 bottom+top, 4 top+bottom),
 * for wavelength `wavelength`.  Reflection factors are included; a zero
 * reflectivity yields -inf.  dropped[i] = 1 when the walk failed. */
int oracle_trace(const oracle_mesh* mesh, const oracle_spectrum* spectrum, uint32_t wavelength,
                 uint32_t n, const double* start, const uint32_t* tri, const uint32_t* level,
                 const uint32_t* sample, const uint32_t* slice, double* lnGain, double* distance,
                 uint32_t* dropped);

/* Importance weights w[slice*P + prism] for one sample. */
int oracle_importance(const oracle_mesh* mesh, const oracle_spectrum* spectrum, uint32_t sample,
                      uint32_t slices, double* weights);

/* Integer ray->prism map from weights: q = ceil(w * 2^24 / max w) (0 for w <= 0),
 * Q = sum q, offsets[b] = floor((C_b * N * 2^32 + phase * Q) / (Q * 2^32)),
 * C_b the exclusive prefix sum of q.  Returns Q (0 if all weights vanish). */
uint64_t oracle_ray_map(uint32_t n, const float* weights, uint32_t rays, uint32_t phase,
                        uint32_t* q, uint32_t* offsets);

/* Full adaptive method over samples [minSample, maxSample].
 * weightsOverride: NULL, or [nSamples][slices*P] FP32 importance weights
 * (lets tests replay the GPU's weights so both walk identical rays). */
int oracle_phi_ase(const oracle_mesh* mesh, const oracle_spectrum* spectrum,
                   const oracle_experiment* experiment, const float* weightsOverride,
                   int threads, oracle_result* result);


/* ---- forward Tet4 estimator (the reference's current calcPhiASE) ----
 * Restates include/kernels/forward/accumulation.hpp:369-453 (source rays by
 * stratified beta*V CDF, uniform point in the tet, isotropic direction,
 * stratified wavelength bin; walk out of the mesh; per crossed cell the
 * track-length tally weight * G * (exp(g l) - 1)/g split to the cell's four
 * material vertices by the segment-midpoint barycentric weights) and the
 * finaliser include/kernels/forwardPhiAseMapping.hpp:51-150 (vertex -> cell
 * density through lumped vertex volumes, estimate S B / (N V) * N_tot/tau,
 * relative error of the batch means). */
typedef struct {
    uint32_t numberOfPoints;
    uint32_t numberOfCells;
    const double* points;              /* [Np][3] */
    const uint32_t* cells;             /* [C][4] */
    const double* betaVolume;          /* [C] */
    const uint32_t* claddingCellTypes; /* [C] or NULL */
    uint32_t claddingNumber;
    double claddingAbsorption;
    double nTot;
    double crystalTFluo;
    /* reflecting boundary surfaces (include/core/mesh.hpp:301-332,
     * include/kernels/reflection.hpp:21-47); all may be NULL */
    const int32_t* cellFaceBoundaries;             /* [C][4] surface id (> 0: a reflecting surface) */
    uint32_t numberOfSurfaces;
    const double* surfaceReflectivities;           /* [numberOfSurfaces] */
    const double* surfaceRefractiveIndexInside;    /* [numberOfSurfaces] */
    const double* surfaceRefractiveIndexOutside;   /* [numberOfSurfaces] */
    const double* reflectivities;                  /* legacy [C][2], by local face % 2 */
    const double* refractiveIndices;               /* legacy [4] */
} oracle_tet_mesh;

typedef struct {
    uint32_t minRays;
    uint32_t maxRays;
    uint32_t adaptiveSteps;
    double rseThreshold;
    uint32_t seed;
    uint32_t batches;          /* statistical batches (reference default 8) */
    /* surface-reservoir reflections (include/core/forwardSrm.hpp:100-365) */
    uint32_t useReflections;
    uint32_t reflectionMaxIterations;
    double reflectionTolerance;
    uint32_t surfaceReservoirSize;
    uint32_t divergenceStreak;
} oracle_forward_experiment;

typedef struct {
    double* phiAse;            /* [C] */
    double* relativeStandardError;
    double* dndtAse;
    uint32_t* droppedRays;     /* [C] */
    uint32_t* rayVisits;       /* [C] segments tallied per cell (the reference's forward totalRays), or NULL */
    uint64_t totalRays;
    uint32_t launches;
    /* SRM outputs of the last launch: worst status over the batches
     * (0 disabled, 1 converged, 2 stable, 3 diverged, 4 max_iterations), most
     * passes, largest remaining weight fraction */
    uint32_t srmStatus;
    uint32_t srmPasses;
    double srmRemainingFraction;
} oracle_forward_result;

/* Tet tables: neighbours [C][4] (-1 boundary), neighbour local face [C][4],
 * barycentric gradients [C][4][3] (lambda_f(x) = delta_f0 + grad_f.(x - v0)),
 * volumes [C]. */
int oracle_tet_tables(const oracle_tet_mesh* mesh, int32_t* neighbors, int32_t* neighborFace, double* gradients,
                      double* volumes);

int oracle_forward_phi_ase(const oracle_tet_mesh* mesh, const oracle_spectrum* spectrum,
                           const oracle_forward_experiment* experiment, int threads, oracle_forward_result* result);

/* Single rays through the Tet4 mesh (no tally): ray i starts at origin[i] in
 * startCell[i] along the unit direction[i].  segments[i] = cells crossed (a
 * zero-length step counts), cells/lengths [n][maxSegments] the first
 * maxSegments of them (either may be NULL), lnGain[i] = sum g l at
 * `wavelength`, endPoint[i] where the walk stopped, status[i] 0 = left the
 * mesh, 1 = walk failed. */
int oracle_tet_trace(const oracle_tet_mesh* mesh, const oracle_spectrum* spectrum, uint32_t wavelength, uint32_t n,
                     const uint32_t* startCell, const double* origin, const double* direction, uint32_t maxSegments,
                     uint32_t* segments, uint32_t* cells, double* lengths, double* lnGain, double* endPoint,
                     int32_t* status);

#ifdef __cplusplus
}
#endif
