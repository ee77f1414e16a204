"""ctypes binding of libhase_b200.so (the C ABI declared in include/hase_b200.h,
include/hase_b200_forward.h and include/hase_b200_proposal.h).

The shared library is built in-tree (``haseongpu_b200/libhase_b200.so``) by
``haseongpu_b200.build.build_library()``.  There is no CPU fallback: every
entry point runs on a CUDA device and reports ``HASE_NO_DEVICE`` otherwise.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

PACKAGE_DIR = Path(__file__).resolve().parent
LIB_PATH = PACKAGE_DIR / "libhase_b200.so"

HASE_OK = 0
HASE_INVALID_ARGUMENT = 1
HASE_CUDA_ERROR = 2
HASE_OUT_OF_MEMORY = 3
HASE_DEVICE_TIMEOUT = 4
HASE_DROPPED_RAYS = 5
HASE_NOT_CONVERGED = 6
HASE_NO_DEVICE = 7
WARNINGS = (HASE_DROPPED_RAYS, HASE_NOT_CONVERGED)

# Every symbol include/hase_b200.h declares.
EXPORTED_SYMBOLS = (
    "hase_last_error_message",
    "hase_status_string",
    "hase_abi_version",
    "hase_ray_kernel_variant_count",
    "hase_ray_kernel_variant_name",
    "hase_context_create",
    "hase_context_update_beta",
    "hase_calc_phi_ase",
    "hase_context_destroy",
    "hase_context_set_local_proposal",
    "hase_context_set_grid_proposal",
    "hase_grid_weights",
    "hase_importance_weights",
    "hase_importance_crossings",
    "hase_ray_map",
    "hase_mesh_tables",
    "hase_trace_rays",
    "hase_philox",
    "hase_probe_l2_bandwidth",
    "hase_probe_l1_bandwidth",
    "hase_estimate_sample_noalloc",
    "hase_simulate",
    # include/hase_b200_forward.h
    "hase_tet_context_create",
    "hase_tet_context_update_beta",
    "hase_tet_context_info",
    "hase_simulate_forward",
    "hase_tet_calc_phi_ase",
    "hase_tet_context_destroy",
    "hase_tet_tables",
    "hase_tet_trace",
    # include/hase_b200_proposal.h
    "hase_proposal_create",
    "hase_proposal_destroy",
    "hase_proposal_get_params",
    "hase_proposal_set_params",
    "hase_proposal_forward",
    "hase_proposal_loss_grad",
    "hase_proposal_train",
    "hase_calc_phi_ase_learned",
    "hase_log_contributions",
    "hase_proposal_features",
    "hase_learned_weights",
    # include/hase_b200_batch.h
    "hase_batch_create",
    "hase_batch_destroy",
    "hase_calc_phi_ase_batch",
    "hase_calc_phi_ase_batch_learned",
)
PROPOSAL_FEATURES = 12
PROPOSAL_PARAMS = 12 * 64 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 + 1

_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)


class MeshDesc(C.Structure):
    _fields_ = [
        ("numberOfPoints", C.c_uint32),
        ("numberOfTriangles", C.c_uint32),
        ("numberOfLevels", C.c_uint32),
        ("points", _f64p),
        ("triangles", _u32p),
        ("thickness", C.c_double),
        ("betaVolume", _f64p),
        ("betaCells", _f64p),
        ("claddingCellTypes", _u32p),
        ("claddingNumber", C.c_uint32),
        ("claddingAbsorption", C.c_double),
        ("nTot", C.c_double),
        ("crystalTFluo", C.c_double),
        ("reflectivities", _f64p),
        ("refractiveIndices", _f64p),
    ]


class SpectrumDesc(C.Structure):
    _fields_ = [("numberOfWavelengths", C.c_uint32), ("sigmaA", _f64p), ("sigmaE", _f64p)]


class ExperimentDesc(C.Structure):
    _fields_ = [
        ("minRays", C.c_uint32),
        ("maxRays", C.c_uint32),
        ("mseThreshold", C.c_double),
        ("useReflections", C.c_uint32),
        ("monochromatic", C.c_uint32),
        ("nearFieldSampling", C.c_uint32),
    ]


class ComputeDesc(C.Structure):
    _fields_ = [
        ("adaptiveSteps", C.c_uint32),
        ("repetitions", C.c_uint32),
        ("rngSeed", C.c_uint32),
        ("minSample", C.c_uint32),
        ("maxSample", C.c_uint32),
        ("raysPerThread", C.c_uint32),
        ("blockSize", C.c_uint32),
        ("workspaceBytes", C.c_uint64),
        ("rayKernelVariant", C.c_uint32),
        ("importanceLayers", C.c_uint32),
    ]


class ResultDesc(C.Structure):
    _fields_ = [
        ("phiAse", _f32p),
        ("standardError", _f64p),
        ("relativeStandardError", _f64p),
        ("totalRays", _u32p),
        ("dndtAse", _f64p),
        ("droppedRays", _u32p),
        ("raysTraced", C.c_uint64),
        ("crossings", C.c_uint64),
        ("importanceMilliseconds", C.c_double),
        ("rayMilliseconds", C.c_double),
        ("totalMilliseconds", C.c_double),
        ("passes", C.c_uint32),
        ("unconvergedSamples", C.c_uint32),
        ("kernelLaunches", C.c_uint32),
    ]


class TetMeshDesc(C.Structure):
    _fields_ = [
        ("numberOfPoints", C.c_uint32),
        ("numberOfCells", C.c_uint32),
        ("points", _f64p),
        ("cells", _u32p),
        ("betaVolume", _f64p),
        ("claddingCellTypes", _u32p),
        ("claddingNumber", C.c_uint32),
        ("claddingAbsorption", C.c_double),
        ("nTot", C.c_double),
        ("crystalTFluo", C.c_double),
        ("cellFaceBoundaries", C.POINTER(C.c_int32)),
        ("numberOfSurfaces", C.c_uint32),
        ("surfaceReflectivities", _f64p),
        ("surfaceRefractiveIndexInside", _f64p),
        ("surfaceRefractiveIndexOutside", _f64p),
        ("reflectivities", _f64p),
        ("refractiveIndices", _f64p),
    ]


class ForwardDesc(C.Structure):
    _fields_ = [
        ("forwardRayCount", C.c_uint32),
        ("maxRays", C.c_uint32),
        ("adaptiveSteps", C.c_uint32),
        ("relativeStandardErrorThreshold", C.c_double),
        ("monochromatic", C.c_uint32),
        ("rngSeed", C.c_uint32),
        ("batches", C.c_uint32),
        ("blockSize", C.c_uint32),
        ("tallyMode", C.c_uint32),
        ("useReflections", C.c_uint32),
        ("reflectionMaxIterations", C.c_uint32),
        ("reflectionTolerance", C.c_double),
        ("surfaceReservoirSize", C.c_uint32),
        ("divergenceStreak", C.c_uint32),
    ]


class ForwardResultDesc(C.Structure):
    _fields_ = [
        ("phiAse", _f32p),
        ("relativeStandardError", _f64p),
        ("dndtAse", _f64p),
        ("totalRays", _u32p),
        ("droppedRays", _u32p),
        ("raysTraced", C.c_uint64),
        ("crossings", C.c_uint64),
        ("rayMilliseconds", C.c_double),
        ("totalMilliseconds", C.c_double),
        ("launches", C.c_uint32),
        ("unconvergedCells", C.c_uint32),
        ("kernelLaunches", C.c_uint32),
        ("tallyMode", C.c_uint32),
        ("srmStatus", C.c_uint32),
        ("srmPasses", C.c_uint32),
        ("srmRemainingFraction", C.c_double),
        ("srmMaxIterations", C.c_uint32),
        ("srmDivergenceStreak", C.c_uint32),
        ("reflectingFaces", C.c_uint32),
    ]


SRM_STATUS = ("disabled", "converged", "stable", "diverged", "max_iterations")


class ProposalBatch(C.Structure):
    _fields_ = [
        ("groups", C.c_uint32),
        ("offsets", _u32p),
        ("features", _f32p),
        ("targets", _f32p),
        ("groupWeights", _f32p),
    ]


class ProposalTrainDesc(C.Structure):
    _fields_ = [
        ("steps", C.c_uint32),
        ("groupsPerStep", C.c_uint32),
        ("learningRate", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("epsilon", C.c_float),
    ]


class LearnedDesc(C.Structure):
    _fields_ = [
        ("mixture", C.c_float),
        ("fallbackVariance", C.c_float),
        ("fallbackSamples", C.c_uint32),
    ]


class PumpDesc(C.Structure):
    _fields_ = [
        ("peakIntensity", C.c_double),
        ("radius", C.c_double),
        ("exponent", C.c_double),
        ("centerX", C.c_double),
        ("centerY", C.c_double),
        ("wavelength", C.c_double),
        ("sigmaA", C.c_double),
        ("sigmaE", C.c_double),
        ("retroreflect", C.c_uint32),
    ]


class TimeDesc(C.Structure):
    _fields_ = [
        ("timeStep", C.c_double),
        ("steps", C.c_uint32),
        ("pumpSteps", C.c_uint32),
        ("aseSteps", C.c_uint32),
        ("integrator", C.c_uint32),
        ("implicitIterations", C.c_uint32),
    ]


class TimeResultDesc(C.Structure):
    _fields_ = [
        ("betaVolume", _f64p),
        ("meanBeta", _f64p),
        ("meanPhi", _f64p),
        ("pumpAbsorbed", _f64p),
        ("phiHistory", _f32p),
        ("aseMilliseconds", C.c_double),
        ("pumpMilliseconds", C.c_double),
        ("totalMilliseconds", C.c_double),
        ("raysTraced", C.c_uint64),
        ("fallbackSamples", C.c_uint32),
    ]


class BatchInstance(C.Structure):
    _fields_ = [
        ("context", C.c_void_p),
        ("minSample", C.c_uint32),
        ("maxSample", C.c_uint32),
        ("result", C.POINTER(ResultDesc)),
    ]


class BatchStats(C.Structure):
    _fields_ = [
        ("raysTraced", C.c_uint64),
        ("crossings", C.c_uint64),
        ("rows", C.c_uint32),
        ("chunks", C.c_uint32),
        ("passes", C.c_uint32),
        ("unconvergedSamples", C.c_uint32),
        ("kernelLaunches", C.c_uint32),
        ("graphNodes", C.c_uint32),
        ("importanceMilliseconds", C.c_double),
        ("rayMilliseconds", C.c_double),
        ("totalMilliseconds", C.c_double),
        ("captureMilliseconds", C.c_double),
        ("setupMilliseconds", C.c_double),
        ("hostMilliseconds", C.c_double),
        ("fallbackSamples", C.c_uint32),
    ]


class HaseError(RuntimeError):
    """A libhase_b200 call failed; ``status`` is the hase_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_lib = None


def lib():
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing; build it with haseongpu_b200.build.build_library()")
        L = C.CDLL(str(LIB_PATH))
        L.hase_last_error_message.restype = C.c_char_p
        L.hase_status_string.restype = C.c_char_p
        L.hase_status_string.argtypes = [C.c_int]
        L.hase_abi_version.restype = C.c_int
        L.hase_ray_kernel_variant_count.restype = C.c_int
        L.hase_ray_kernel_variant_name.restype = C.c_char_p
        L.hase_ray_kernel_variant_name.argtypes = [C.c_uint32]
        L.hase_context_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(SpectrumDesc), C.c_int,
                                          C.POINTER(C.c_void_p)]
        L.hase_context_update_beta.argtypes = [C.c_void_p, _f64p, _f64p]
        L.hase_calc_phi_ase.argtypes = [C.c_void_p, C.POINTER(ExperimentDesc), C.POINTER(ComputeDesc),
                                        C.POINTER(ResultDesc)]
        L.hase_context_destroy.argtypes = [C.c_void_p]
        L.hase_context_set_local_proposal.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.hase_context_set_grid_proposal.argtypes = [C.c_void_p, C.c_uint32]
        L.hase_grid_weights.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _f32p]
        L.hase_importance_weights.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, _f32p]
        L.hase_importance_crossings.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, _u64p]
        L.hase_ray_map.argtypes = [C.c_uint32, C.c_uint32, _f32p, C.c_uint32, _u32p, _u32p, _u32p, _u64p]
        L.hase_trace_rays.argtypes = [C.c_void_p, C.c_uint32, _f32p, _u32p, _u32p, _u32p, _u32p, C.c_uint32,
                                      _f32p, _f32p, _u32p]
        L.hase_philox.argtypes = [C.c_uint32, _u32p, _u32p, _u32p]
        L.hase_probe_l2_bandwidth.argtypes = [C.c_int, C.c_uint64, C.c_uint32, _f64p]
        L.hase_probe_l1_bandwidth.argtypes = [C.c_int, C.c_uint32, C.c_uint32, _f64p]
        L.hase_estimate_sample_noalloc.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32,
                                                   C.c_uint32, C.c_uint32, C.c_void_p]
        _i32p = C.POINTER(C.c_int32)
        L.hase_tet_context_create.argtypes = [C.POINTER(TetMeshDesc), C.POINTER(SpectrumDesc), C.c_int,
                                              C.POINTER(C.c_void_p)]
        L.hase_tet_context_update_beta.argtypes = [C.c_void_p, _f64p]
        L.hase_tet_context_info.argtypes = [C.c_void_p, _u32p, _u32p]
        L.hase_simulate_forward.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(ForwardDesc), C.POINTER(PumpDesc),
                                            C.POINTER(TimeDesc), C.POINTER(TimeResultDesc)]
        L.hase_tet_calc_phi_ase.argtypes = [C.c_void_p, C.POINTER(ForwardDesc), C.POINTER(ForwardResultDesc)]
        L.hase_tet_context_destroy.argtypes = [C.c_void_p]
        L.hase_tet_tables.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, _f64p]
        L.hase_tet_trace.argtypes = [C.c_void_p, C.c_uint32, _u32p, _f64p, _f64p, C.c_uint32, C.c_uint32, _u32p,
                                     _u32p, _f64p, _f64p, _f64p, _i32p]
        L.hase_proposal_create.argtypes = [C.c_int, C.c_uint32, C.POINTER(C.c_void_p)]
        L.hase_proposal_destroy.argtypes = [C.c_void_p]
        L.hase_proposal_get_params.argtypes = [C.c_void_p, _f32p]
        L.hase_proposal_set_params.argtypes = [C.c_void_p, _f32p]
        L.hase_proposal_forward.argtypes = [C.c_void_p, C.c_uint32, _f32p, _f32p]
        L.hase_proposal_loss_grad.argtypes = [C.c_void_p, C.POINTER(ProposalBatch), _f32p, _f32p]
        L.hase_proposal_train.argtypes = [C.c_void_p, C.POINTER(ProposalBatch), C.POINTER(ProposalTrainDesc), _f32p]
        L.hase_calc_phi_ase_learned.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(ExperimentDesc),
                                                C.POINTER(ComputeDesc), C.POINTER(LearnedDesc), C.POINTER(ResultDesc)]
        L.hase_log_contributions.argtypes = [C.c_void_p, C.POINTER(ExperimentDesc), C.POINTER(ComputeDesc), _f32p,
                                             C.POINTER(ResultDesc)]
        L.hase_proposal_features.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _f32p]
        L.hase_learned_weights.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                           C.c_float, _f32p]
        L.hase_simulate.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.POINTER(ExperimentDesc), C.POINTER(ComputeDesc),
                                    C.POINTER(PumpDesc), C.POINTER(TimeDesc), C.POINTER(TimeResultDesc)]
        L.hase_batch_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.hase_batch_destroy.argtypes = [C.c_void_p]
        L.hase_calc_phi_ase_batch.argtypes = [C.c_void_p, C.POINTER(BatchInstance), C.c_uint32,
                                              C.POINTER(ExperimentDesc), C.POINTER(ComputeDesc), C.POINTER(BatchStats)]
        L.hase_calc_phi_ase_batch_learned.argtypes = [C.c_void_p, C.POINTER(BatchInstance), C.c_uint32,
                                                      C.POINTER(ExperimentDesc), C.POINTER(ComputeDesc), C.c_void_p,
                                                      C.c_float, C.c_float, C.POINTER(BatchStats)]
        for name in EXPORTED_SYMBOLS:
            if name not in ("hase_last_error_message", "hase_status_string", "hase_abi_version",
                            "hase_ray_kernel_variant_count", "hase_ray_kernel_variant_name"):
                getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def check(status: int, *, allow_warnings: bool = False) -> int:
    if status == HASE_OK or (allow_warnings and status in WARNINGS):
        return status
    msg = lib().hase_last_error_message().decode(errors="replace")
    name = lib().hase_status_string(status).decode()
    raise HaseError(status, f"libhase_b200: {name}: {msg}")


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


def philox(ctr, key):
    """Device Philox4x32-10 of counters ``ctr`` [n, 4] under ``key`` (2 words)."""
    c = np.ascontiguousarray(np.asarray(ctr, np.uint32).reshape(-1, 4))
    k = np.ascontiguousarray(np.asarray(key, np.uint32).reshape(2))
    out = np.empty_like(c)
    check(lib().hase_philox(c.shape[0], ptr(c, _u32p), ptr(k, _u32p), ptr(out, _u32p)))
    return out


def l2_bandwidth(device=0, bytes_=48 << 20, reps=40) -> float:
    """Measured L2 read bandwidth (GB/s) of `device`."""
    out = C.c_double(0.0)
    check(lib().hase_probe_l2_bandwidth(int(device), int(bytes_), int(reps), C.byref(out)))
    return out.value


def l1_bandwidth(device=0, shared=False, reps=2000) -> float:
    """Measured L1 (or shared-memory) read bandwidth (GB/s) of `device`."""
    out = C.c_double(0.0)
    check(lib().hase_probe_l1_bandwidth(int(device), 1 if shared else 0, int(reps), C.byref(out)))
    return out.value


def ray_map(weights, rays, phases):
    """Device ray->prism map of weight rows ``weights`` [rows, n] (float32)."""
    w = np.ascontiguousarray(np.atleast_2d(np.asarray(weights, np.float32)))
    rows, n = w.shape
    ph = np.ascontiguousarray(np.asarray(phases, np.uint32).reshape(rows))
    q = np.empty((rows, n), np.uint32)
    off = np.empty((rows, n + 1), np.uint32)
    Q = np.empty(rows, np.uint64)
    check(lib().hase_ray_map(rows, n, ptr(w, _f32p), int(rays), ptr(ph, _u32p), ptr(q, _u32p), ptr(off, _u32p),
                             ptr(Q, _u64p)))
    return Q, q, off
