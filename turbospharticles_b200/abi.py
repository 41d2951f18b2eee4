"""ctypes mirror of include/tsp_b200.h and loader of the in-tree CUDA library.

The structs here are byte-for-byte the C structs of the C ABI; both the product backend
(`libtsp_b200.so`) and the test oracle use them.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "_build", "libtsp_b200.so")

TSP_OK = 0
STATUS_NAMES = {
    -1: "TSP_ERR_INVALID", -2: "TSP_ERR_CUDA", -3: "TSP_ERR_OVERFLOW", -4: "TSP_ERR_FRAME",
    -5: "TSP_ERR_NEIGHBOR_LIST", -6: "TSP_ERR_RIGID", -7: "TSP_ERR_UNSUPPORTED",
    -8: "TSP_ERR_NO_DEVICE",
}

TERM_FIXED_ITERS, TERM_REL_ERR_RAW, TERM_REL_ERR_POS, TERM_REL_ERR_ABS = 0, 1, 2, 3
SPECIES_F, SPECIES_B, SPECIES_R = 0, 1, 2
LIST_FF, LIST_FB, LIST_FR, LIST_RF, LIST_RB, LIST_RR = range(6)
NOALLOC_MAX_PARTICLES = 1 << 24  # TSP_NOALLOC_MAX_PARTICLES
# Stats::StatMetric (source/eval/stats/metrics.h:23-86), the record of tsp_b200_fill_statistics
STAT_NAMES = ("NumF", "NumB", "NumR", "NumNbrFF_Avg", "NumNbrFF_Min", "NumNbrFF_Max", "NumNbrFF_P99", "NumNbrFB_Avg", "NumNbrFB_Min", "NumNbrFB_Max", "NumNbrFB_P99", "NumNbrFR_Avg", "NumNbrFR_Min", "NumNbrFR_Max", "NumNbrFR_P99", "NumNbrRF_Avg", "NumNbrRF_Min", "NumNbrRF_Max", "NumNbrRF_P99", "NumNbrRB_Avg", "NumNbrRB_Min", "NumNbrRB_Max", "NumNbrRB_P99", "NumNbrRR_Avg", "NumNbrRR_Min", "NumNbrRR_Max", "NumNbrRR_P99", "DensRelError_Raw_Avg", "DensRelError_Pos_Avg", "DensRelError_Abs_Avg", "NumSolverIters", "CFL_Number", "VelMag_Avg", "VelMag_Min", "VelMag_Max")
PHASE_NAMES = ("frame", "sort_reorder_tables", "query_count", "finalize_readback", "query_fill", "density",
               "non_pressure", "source_diag_init", "jacobi_loop", "pressure_acc_final", "integration",
               "stats_readback")
STAGE_DENSITY, STAGE_NON_PRESSURE, STAGE_SOURCE_DIAG_INIT = 1, 2, 3
STAGE_PRESSURE_ACC, STAGE_JACOBI_UPDATE, STAGE_INTEGRATION, STAGE_BOUNDARY_VOLUMES = 4, 5, 6, 7
(FIELD_POS, FIELD_VEL, FIELD_VEL_PRED, FIELD_ACC_PRESS, FIELD_SOURCE, FIELD_DIAG, FIELD_PRESSURE,
 FIELD_DENSITY, FIELD_VOL_B, FIELD_PSI_B, FIELD_VOL_R, FIELD_PSI_R, FIELD_FORCE_R,
 FIELD_BODY_FT) = range(14)
FIELD_COMPONENTS = {FIELD_POS: 3, FIELD_VEL: 3, FIELD_VEL_PRED: 3, FIELD_ACC_PRESS: 3,
                    FIELD_SOURCE: 1, FIELD_DIAG: 1, FIELD_PRESSURE: 1, FIELD_DENSITY: 1,
                    FIELD_VOL_B: 1, FIELD_PSI_B: 1, FIELD_VOL_R: 1, FIELD_PSI_R: 1,
                    FIELD_FORCE_R: 3, FIELD_BODY_FT: 6}

_f = C.c_float
_u32 = C.c_uint32
_pf = C.POINTER(C.c_float)
_pu64 = C.POINTER(C.c_uint64)
_pu32 = C.POINTER(C.c_uint32)


class TspParams(C.Structure):
    _fields_ = [
        ("timeStep", _f), ("particleSizeF", _f), ("particleSizeB", _f),
        ("kernelRadius", _f), ("kernelRadiusSqu", _f), ("restDensity", _f),
        ("massF", _f), ("massB", _f), ("viscosityF", _f), ("viscosityB", _f),
        ("gravity", _f * 3), ("pressGamma", _f), ("jacobiOmega", _f),
        ("jacobiWarmStart", _f), ("densityDevTarget", _f),
        ("fixedIters", _u32), ("minSolverIters", _u32), ("maxSolverIters", _u32),
        ("solverTerminationCond", _u32), ("gridCellSizeRatio", _f), ("boundaryLayers", _u32),
        ("cubicSplineAlphaOverride", _f), ("rigidContactDensityDevTarget", _f),
        ("rigidContactMaxSolverIters", _u32), ("surfaceNbrCountThreshold", _u32), ("reserved", _u32 * 1),
    ]


_STATE_FIELDS = [
    ("N_F", _u32), ("N_B", _u32), ("N_R", _u32), ("N_RB", _u32),
    ("step", C.c_uint64), ("time", C.c_double),
    ("idF", _pu64),
    ("xPosF", _pf), ("yPosF", _pf), ("zPosF", _pf),
    ("xVelF", _pf), ("yVelF", _pf), ("zVelF", _pf),
    ("xVelPredF", _pf), ("yVelPredF", _pf), ("zVelPredF", _pf),
    ("xAccPressF", _pf), ("yAccPressF", _pf), ("zAccPressF", _pf),
    ("sourceTermF", _pf), ("diagElemF", _pf), ("pressureF", _pf), ("densityF", _pf),
    ("idB", _pu64), ("xPosB", _pf), ("yPosB", _pf), ("zPosB", _pf), ("volB", _pf), ("psiB", _pf),
    ("idR", _pu64), ("bodyIdR", _pu32),
    ("xPosRelR", _pf), ("yPosRelR", _pf), ("zPosRelR", _pf), ("volR", _pf), ("psiR", _pf),
    ("xPosR", _pf), ("yPosR", _pf), ("zPosR", _pf),
    ("idRB", _pu64), ("rigidParticleCountRB", _pu32),
    ("xCM", _pf), ("yCM", _pf), ("zCM", _pf),
    ("xVelRB", _pf), ("yVelRB", _pf), ("zVelRB", _pf),
    ("xOmegaRB", _pf), ("yOmegaRB", _pf), ("zOmegaRB", _pf),
    ("xAngMomRB", _pf), ("yAngMomRB", _pf), ("zAngMomRB", _pf),
    ("a00", _pf), ("a01", _pf), ("a02", _pf), ("a10", _pf), ("a11", _pf), ("a12", _pf),
    ("a20", _pf), ("a21", _pf), ("a22", _pf),
    ("massRB", _pf), ("massInvRB", _pf),
    ("iBodyInv00", _pf), ("iBodyInv01", _pf), ("iBodyInv02", _pf),
    ("iBodyInv10", _pf), ("iBodyInv11", _pf), ("iBodyInv12", _pf),
    ("iBodyInv20", _pf), ("iBodyInv21", _pf), ("iBodyInv22", _pf),
]


class TspStateView(C.Structure):
    _fields_ = _STATE_FIELDS


STATE_ARRAY_FIELDS = [name for name, _ in _STATE_FIELDS[6:]]


class TspStepRecord(C.Structure):
    _fields_ = [("step", C.c_uint64), ("ms", C.c_float), ("solverIters", C.c_uint32),
                ("avgRelDensityErrPos", C.c_double)]


class TspStepStats(C.Structure):
    _fields_ = [
        ("step", C.c_uint64), ("time", C.c_double), ("solverIters", _u32), ("reserved0", _u32),
        ("errSumRaw", C.c_double), ("errSumPos", C.c_double), ("errSumAbs", C.c_double),
        ("avgRelDensityErrRaw", _f), ("avgRelDensityErrPos", _f), ("avgRelDensityErrAbs", _f),
        ("frameRebuilds", _u32), ("cellOrig", C.c_int32 * 3), ("cellDims", _u32 * 3),
        ("keyBits", _u32), ("nCellsF", _u32), ("nCellsB", _u32), ("nCellsR", _u32),
        ("nNbrFF", C.c_uint64), ("nNbrFB", C.c_uint64), ("nNbrFR", C.c_uint64),
        ("nNbrRF", C.c_uint64), ("nNbrRB", C.c_uint64), ("nNbrRR", C.c_uint64),
        ("sellPackedBytes", C.c_uint64), ("lastStepMs", _f), ("lastNeighborMs", _f),
        ("lastJacobiMs", _f), ("reserved1", _u32),
    ]


# every exported entry point of include/tsp_b200.h, with its ctypes signature
class TspContactReport(C.Structure):
    """tsp_contact_report (CPU::RigidContactReport, rigid_solver.h:25-30, + contact counts)."""
    _fields_ = [("solverIters", _u32), ("avgDensityError", _f), ("converged", _u32), ("reserved", _u32),
                ("nContacts", C.c_uint64), ("nContactBoundary", C.c_uint64)]


class TspExportSnapshot(C.Structure):
    """tsp_export_snapshot (Sync::ExportSnapshot, snapshots.h:37-66)."""
    _fields_ = [("simStep", C.c_uint64), ("simTime", C.c_double), ("N_F", _u32), ("N_B", _u32), ("N_R", _u32),
                ("reserved", _u32)] + [(n, _pf) for n in ("xPosF", "yPosF", "zPosF", "velMagF", "xPosB", "yPosB",
                                                           "zPosB", "volB")] + \
               [("isMeshB", C.POINTER(C.c_uint8)), ("bodyIdR", _pu32)] + \
               [(n, _pf) for n in ("xPosR", "yPosR", "zPosR", "volR")]


NO_MESH_ID = (1 << 64) - 1
TSP_ERR_INVALID, TSP_ERR_OVERFLOW = -1, -3


class TspSurfaceSamplingParams(C.Structure):
    """tsp_surface_sampling_params (parameters_sim.h:122-139)."""
    _fields_ = [("minDistance", _f), ("maxDistance", _f), ("coverageProbeSpacing", _f), ("particleSizeF", _f),
                ("candidateMultiplier", _u32), ("reserved", _u32), ("seed", C.c_uint64)]


class TspSurfaceSamplingStats(C.Structure):
    """tsp_surface_sampling_stats (SurfaceSamplingStats, surface_sampling.h:18-26)."""
    _fields_ = [("N_candidates", C.c_uint64), ("N_initialSamples", _u32), ("N_coverageRepairs", _u32),
                ("N_coverageProbes", C.c_uint64), ("surfaceArea", _f), ("reserved", _u32)]

_VP = C.c_void_p
EXPORTS = {
    "tsp_b200_create": (C.c_int, [C.POINTER(TspParams), C.c_int, C.POINTER(_VP)]),
    "tsp_b200_destroy": (C.c_int, [_VP]),
    "tsp_b200_name": (C.c_char_p, [_VP]),
    "tsp_b200_last_error": (C.c_char_p, [_VP]),
    "tsp_b200_set_domain": (C.c_int, [_VP, _pf, _pf]),
    "tsp_b200_pull_state": (C.c_int, [_VP, C.POINTER(TspStateView), C.POINTER(TspParams)]),
    "tsp_b200_push_state": (C.c_int, [_VP, C.POINTER(TspStateView)]),
    "tsp_b200_get_counts": (C.c_int, [_VP, _pu32, _pu32, _pu32, _pu32]),
    "tsp_b200_neighbor_search": (C.c_int, [_VP, C.POINTER(TspParams)]),
    "tsp_b200_step": (C.c_int, [_VP, C.POINTER(TspParams), _u32]),
    "tsp_b200_get_stats": (C.c_int, [_VP, C.POINTER(TspStepStats)]),
    "tsp_b200_read_cell_ids": (C.c_int, [_VP, _u32, _pu64, _u32]),
    "tsp_b200_read_permutation": (C.c_int, [_VP, _u32, _pu32, _u32]),
    "tsp_b200_read_cell_table": (C.c_int, [_VP, _u32, _pu64, _pu32, _u32, _pu32]),
    "tsp_b200_read_sell32_meta": (C.c_int, [_VP, _u32, C.POINTER(C.c_uint16),
                                            C.POINTER(C.c_uint16), C.POINTER(C.c_uint8), _pu32,
                                            _pu32, _pu64, _u32, _pu64, _pu64]),
    "tsp_b200_read_sell32_words": (C.c_int, [_VP, _u32, C.POINTER(C.c_uint16), C.c_uint64,
                                             _pu32, C.c_uint64]),
    "tsp_b200_read_rows": (C.c_int, [_VP, _u32, _pu64, _u32, _pu32, C.c_uint64, _pu64]),
    "tsp_b200_run_stage": (C.c_int, [_VP, C.POINTER(TspParams), _u32, C.POINTER(C.c_double)]),
    "tsp_b200_read_field": (C.c_int, [_VP, _u32, _VP, _u32]),
    "tsp_b200_write_field": (C.c_int, [_VP, _u32, _VP, _u32]),
    "tsp_b200_time_stage": (C.c_int, [_VP, C.POINTER(TspParams), _u32, _u32, _pf]),
    "tsp_b200_get_launch_count": (C.c_int, [_VP, C.POINTER(C.c_uint64)]),
    "tsp_b200_get_step_time_total": (C.c_int, [_VP, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "tsp_b200_get_step_history": (C.c_int, [_VP, C.POINTER(TspStepRecord), _u32, C.POINTER(_u32)]),
    "tsp_b200_get_stream": (C.c_int, [_VP, C.POINTER(_VP)]),
    "tsp_b200_fill_statistics": (C.c_int, [_VP, C.POINTER(TspParams), C.POINTER(C.c_double), C.c_uint32]),
    "tsp_b200_get_contact_report": (C.c_int, [_VP, C.POINTER(TspContactReport)]),
    "tsp_b200_pack_export_snapshot": (C.c_int, [_VP, C.POINTER(TspParams), C.c_int, C.c_uint64,
                                                C.POINTER(TspExportSnapshot)]),
    "tsp_b200_sample_surface": (C.c_int, [C.c_int, _pf, _u32, _pu32, _u32, C.POINTER(TspSurfaceSamplingParams), _pf,
                                          C.c_uint64, _pu64, C.POINTER(TspSurfaceSamplingStats)]),
    "tsp_b200_get_phase_times": (C.c_int, [_VP, C.POINTER(C.c_float), C.c_uint32, C.POINTER(C.c_uint32)]),
    "tsp_b200_try_build_cell_frame": (C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                                 C.POINTER(C.c_uint32)]),
    "tsp_b200_batch_create": (C.c_int, [C.POINTER(TspParams), C.c_int, C.c_uint64, C.POINTER(_VP)]),
    "tsp_b200_batch_destroy": (C.c_int, [_VP]),
    "tsp_b200_batch_last_error": (C.c_char_p, [_VP]),
    "tsp_b200_admit": (C.c_int, [_VP, C.POINTER(TspStateView), _pf, _pf, C.POINTER(C.c_uint32)]),
    "tsp_b200_retire": (C.c_int, [_VP, C.c_uint32, C.POINTER(TspStateView)]),
    "tsp_b200_substep_all": (C.c_int, [_VP, C.POINTER(TspParams), C.c_uint32]),
    "tsp_b200_batch_push": (C.c_int, [_VP, C.c_uint32, C.POINTER(TspStateView)]),
    "tsp_b200_batch_stats": (C.c_int, [_VP, C.c_uint32, C.POINTER(TspStepStats)]),
    "tsp_b200_batch_info": (C.c_int, [_VP, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                      C.POINTER(C.c_uint64), C.POINTER(C.c_float), C.POINTER(C.c_uint64)]),
    "tsp_b200_batch_scene_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_uint64]),
    "tsp_b200_set_autotune": (C.c_int, [C.c_int]),
    "tsp_b200_reset_tuning": (C.c_int, []),
    "tsp_b200_set_tuning": (C.c_int, [C.c_int, C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint32]),
    "tsp_b200_get_tuning": (C.c_int, [C.c_int, C.c_char_p, C.c_uint32, C.POINTER(C.c_uint32)]),
    "tsp_b200_noalloc_setup": (C.c_int, []),
    "tsp_b200_build_cell_table_noalloc": (C.c_int, [_VP, C.c_uint32, _VP, _VP, _VP, _VP]),
    "tsp_b200_noalloc_last_error": (C.c_char_p, []),
}


class TspError(RuntimeError):
    """Raised when a C-ABI call returns a negative status (the reference throws
    std::runtime_error from GPU::Check, source/simulation/GPU/gpu_utils.h:24-45)."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_LIB = None


def load_library(path: str | None = None) -> C.CDLL:
    """Loads the in-tree CUDA library; raises if it is missing (there is no CPU fallback)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `python -m turbospharticles_b200.build` "
            "(the B200 backend has no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def set_autotune(enabled: bool) -> None:
    """Autotuner on (default) or off (every launch uses the untuned configuration)."""
    load_library().tsp_b200_set_autotune(1 if enabled else 0)


def reset_tuning() -> None:
    load_library().tsp_b200_reset_tuning()


def tuning(device: int = 0) -> dict:
    """The autotuner's choices on a device: {"kernel/nN": {slots, min_blocks, ms, untuned_ms,
    worst_ms, candidates}}."""
    import json
    L = load_library()
    n = C.c_uint32()
    L.tsp_b200_get_tuning(device, None, 0, C.byref(n))
    buf = C.create_string_buffer(n.value + 1)
    L.tsp_b200_get_tuning(device, buf, n.value + 1, C.byref(n))
    return json.loads(buf.value.decode() or "{}")


def pin_tuning(table: dict, device: int = 0) -> None:
    """Pins the configurations of a tuning report (the dict `tuning()` returns) on a device."""
    L = load_library()
    for key, v in table.items():
        kernel, n = key.split("/n")
        rc = L.tsp_b200_set_tuning(device, kernel.encode(), int(n), int(v["slots"]), int(v["min_blocks"]))
        if rc != 0:
            raise TspError(rc, f"cannot pin {key}: {v}")
