"""ctypes view of the engine's C ABI (include/g4b.h, include/g4b_scheduler.h, include/g4b_synth.h).

Loads g4go_b200/_lib/libg4b.so, the sm_100a build of the engine. There is no
fallback: if the library is missing it is built with nvcc, and if that is
impossible importing the engine fails.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

import numpy as np

from . import build as _build

ABI_VERSION = 1
INVALID_ID = 0xFFFFFFFF

OK = 0
ERR_INVALID_ARGUMENT = -1
ERR_OVERFLOW = -2
ERR_LOGIC = -3
ERR_CUDA = -4
ERR_CAPACITY = -5
ERR_TIMEOUT = -6
ERR_NO_SCENE = -7
ERR_UNSUPPORTED = -8
ERR_NO_DEVICE = -9

PRECISION_FP32 = 0
PRECISION_FP64 = 1
FORM_BATCHED = 0
FORM_PLAIN = 1

EMISSION_DIRECT = 0
EMISSION_CERENKOV = 1
EMISSION_SCINTILLATION = 2

SURFACE_DIELECTRIC_DIELECTRIC = 0
SURFACE_DIELECTRIC_METAL = 1
MODEL_GLISUR = 0
MODEL_UNIFIED = 1
FINISH_POLISHED = 0
FINISH_GROUND = 1

FIELD_GENERATED = 0
FIELD_CAPTURED = 1
FIELD_DETECTED = 2
FIELD_ABSORBED = 3
FIELD_ESCAPED = 4
FIELD_TRUNCATED = 5
FIELD_MAX_BOUNCE = 6
FIELD_INVALID_STATE = 7
FIELD_ZERO_STEP = 8
FIELD_TRANSPORT_TIME = 9

# 128-byte genstep (OpticalEmission, PhotonTransport.hpp:40-69).
EMISSION_DTYPE = np.dtype(
    [
        ("position_mm", "<f4", (3,)),
        ("time_ns", "<f4"),
        ("direction", "<f4", (3,)),
        ("step_length_mm", "<f4"),
        ("step_delta_mm", "<f4", (3,)),
        ("pre_velocity_mm_per_ns", "<f4"),
        ("polarization", "<f4", (3,)),
        ("delta_velocity_mm_per_ns", "<f4"),
        ("energy_ev", "<f4"),
        ("pre_mean_photon_count", "<f4"),
        ("post_mean_photon_count", "<f4"),
        ("decay_time_ns", "<f4"),
        ("rise_time_ns", "<f4"),
        ("charge", "<f4"),
        ("event_id", "<u4"),
        ("first_photon_id", "<u4"),
        ("photon_count", "<u4"),
        ("volume_id", "<u4"),
        ("material_id", "<u4"),
        ("spectrum_id", "<u4"),
        ("type", "u1"),
        ("reserved", "u1", (15,)),
    ]
)
assert EMISSION_DTYPE.itemsize == 128

# 48-byte detection (PhotonDetection, PhotonTransport.hpp:71-81).
DETECTION_DTYPE = np.dtype(
    [
        ("position_mm", "<f4", (3,)),
        ("time_ns", "<f4"),
        ("direction", "<f4", (3,)),
        ("energy_ev", "<f4"),
        ("event_id", "<u4"),
        ("photon_id", "<u4"),
        ("sensor_id", "<u4"),
        ("reserved", "<u4"),
    ]
)
assert DETECTION_DTYPE.itemsize == 48


class Config(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("device", C.c_int32),
        ("seed", C.c_uint64),
        ("max_bounces_per_photon", C.c_uint32),
        ("boundary_tolerance_mm", C.c_float),
        ("precision", C.c_uint32),
        ("launch_form", C.c_uint32),
        ("enable_performance_diagnostics", C.c_uint32),
        ("ordered_detections", C.c_uint32),
        ("hit_capacity", C.c_uint64),
        ("block_size", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("chunk_photons", C.c_uint32),
        ("use_cuda_graph", C.c_uint32),
        ("record_photon_fates", C.c_uint32),
        ("generation_pass", C.c_uint32),
        ("wave_photons", C.c_uint32),
        ("reserved", C.c_uint32 * 5),
    ]


class Property(C.Structure):
    _fields_ = [
        ("energy_ev", C.POINTER(C.c_float)),
        ("values", C.POINTER(C.c_float)),
        ("count", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class Material(C.Structure):
    _fields_ = [
        ("rindex", Property),
        ("rindex_max", C.c_float),
        ("reserved", C.c_uint32),
        ("group_velocity_mm_per_ns", Property),
        ("abs_length_mm", Property),
        ("rayleigh_length_mm", Property),
        ("scintillation_spectrum", Property * 3),
    ]


class Surface(C.Structure):
    _fields_ = [
        ("type", C.c_uint8),
        ("model", C.c_uint8),
        ("finish", C.c_uint8),
        ("reserved0", C.c_uint8),
        ("model_value", C.c_float),
        ("reflectivity", Property),
        ("efficiency", Property),
        ("transmittance", Property),
        ("rindex", Property),
        ("specular_lobe", Property),
        ("specular_spike", Property),
        ("backscatter", Property),
        ("surface_roughness", Property),
    ]


class Volume(C.Structure):
    _fields_ = [
        ("volume_id", C.c_uint32),
        ("material_id", C.c_uint32),
        ("parent_volume_id", C.c_uint32),
        ("skin_surface_id", C.c_uint32),
        ("sensor_id", C.c_uint32),
        ("reserved", C.c_uint32),
        ("center_mm", C.c_float * 3),
        ("half_size_mm", C.c_float * 3),
    ]


class SurfaceBinding(C.Structure):
    _fields_ = [
        ("from_volume_id", C.c_uint32),
        ("to_volume_id", C.c_uint32),
        ("surface_id", C.c_uint32),
    ]


class Scene(C.Structure):
    _fields_ = [
        ("materials", C.POINTER(Material)),
        ("material_count", C.c_uint32),
        ("surface_count", C.c_uint32),
        ("surfaces", C.POINTER(Surface)),
        ("volumes", C.POINTER(Volume)),
        ("volume_count", C.c_uint32),
        ("binding_count", C.c_uint32),
        ("bindings", C.POINTER(SurfaceBinding)),
        ("world_volume_id", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class Statistics(C.Structure):
    _fields_ = [
        ("valid_fields", C.c_uint32),
        ("reserved", C.c_uint32),
        ("generated_count", C.c_uint64),
        ("captured_count", C.c_uint64),
        ("detected_count", C.c_uint64),
        ("absorbed_count", C.c_uint64),
        ("escaped_count", C.c_uint64),
        ("truncated_count", C.c_uint64),
        ("max_bounce_count", C.c_uint64),
        ("invalid_state_count", C.c_uint64),
        ("zero_step_count", C.c_uint64),
        ("transport_time_ms", C.c_double),
    ]


class EventStatistics(C.Structure):
    _fields_ = [
        ("event_id", C.c_uint32),
        ("reserved", C.c_uint32),
        ("statistics", Statistics),
    ]


class Performance(C.Structure):
    _fields_ = [
        ("host_to_device_ms", C.c_double),
        ("host_to_device_bytes", C.c_uint64),
        ("device_memset_ms", C.c_double),
        ("kernel_ms", C.c_double),
        ("device_hit_compaction_ms", C.c_double),
        ("device_to_host_ms", C.c_double),
        ("device_metadata_to_host_ms", C.c_double),
        ("device_metadata_to_host_bytes", C.c_uint64),
        ("device_hits_to_host_ms", C.c_double),
        ("device_hits_to_host_bytes", C.c_uint64),
        ("host_hit_compaction_ms", C.c_double),
        ("total_bounce_count", C.c_uint64),
        ("coincident_candidate_trace_count", C.c_uint64),
        ("coincident_candidate_hit_count", C.c_uint64),
        ("kernel_launch_count", C.c_uint64),
    ]


class Output(C.Structure):
    _fields_ = [
        ("detections", C.c_void_p),
        ("detection_capacity", C.c_uint64),
        ("detection_count", C.c_uint64),
        ("event_statistics", C.POINTER(EventStatistics)),
        ("event_capacity", C.c_uint32),
        ("event_count", C.c_uint32),
        ("statistics", Statistics),
        ("performance", Performance),
    ]


class SchedulerConfig(C.Structure):
    _fields_ = [
        ("abi_version", C.c_uint32),
        ("target_photons_per_batch", C.c_uint32),
        ("max_events_per_batch", C.c_uint32),
        ("max_queued_photons", C.c_uint32),
        ("max_queued_submissions", C.c_uint32),
        ("batch_collection_timeout_ms", C.c_uint32),
        ("enable_performance_diagnostics", C.c_uint32),
        ("serial", C.c_uint32),
        ("batches_in_flight", C.c_uint32),
        ("reserved", C.c_uint32 * 7),
    ]


class BatchStatistics(C.Structure):
    _fields_ = [
        ("batch_count", C.c_uint64),
        ("event_count", C.c_uint64),
        ("photon_count", C.c_uint64),
        ("max_batch_photon_count", C.c_uint64),
        ("max_batch_event_count", C.c_uint64),
        ("queue_high_water_mark", C.c_uint64),
        ("min_batch_photon_count", C.c_uint64),
        ("total_queue_wait_count", C.c_uint64),
        ("scheduler_input_wait_ms", C.c_double),
        ("scheduler_gpu_wait_ms", C.c_double),
        ("scheduler_queue_wait_ms", C.c_double),
        ("scheduler_batch_flatten_ms", C.c_double),
        ("scheduler_batch_flatten_bytes", C.c_uint64),
        ("overlapped_batch_count", C.c_uint64),
        ("performance", Performance),
    ]


# g4b_transport_ops: a transport the scheduler drives (include/g4b_scheduler.h).
TRANSPORT_ENQUEUE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32,
                                C.POINTER(C.c_uint32))
TRANSPORT_POLL = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_int))
TRANSPORT_QUERY = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32))
TRANSPORT_COMPLETE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(Output))
TRANSPORT_LAST_ERROR = C.CFUNCTYPE(C.c_void_p, C.c_void_p)


class TransportOps(C.Structure):
    _fields_ = [
        ("context", C.c_void_p),
        ("enqueue", TRANSPORT_ENQUEUE),
        ("poll", TRANSPORT_POLL),
        ("query", TRANSPORT_QUERY),
        ("complete", TRANSPORT_COMPLETE),
        ("last_error", TRANSPORT_LAST_ERROR),
    ]


class TuneResult(C.Structure):
    _fields_ = [
        ("block_size", C.c_uint32),
        ("blocks_per_sm", C.c_uint32),
        ("chunk_photons", C.c_uint32),
        ("candidates_tried", C.c_uint32),
        ("best_ms", C.c_double),
        ("worst_ms", C.c_double),
    ]


class GradientRequest(C.Structure):
    _fields_ = [
        ("rindex_material_id", C.c_uint32),
        ("abs_length_material_id", C.c_uint32),
        ("reflectivity_surface_id", C.c_uint32),
        ("edge_band_mm", C.c_float),
        ("edge_index_window", C.c_float),
        ("reserved", C.c_uint32 * 3),
    ]


class Gradients(C.Structure):
    _fields_ = [
        ("detected", C.c_uint64),
        ("replay_mismatches", C.c_uint64),
        ("mean_time_ns", C.c_double),
        ("d_detected", C.c_double * 4),
        ("d_mean_time_ns", C.c_double * 4),
        ("kernel_ms", C.c_double),
    ]


class SynthParams(C.Structure):
    _fields_ = [
        ("event_count", C.c_uint32),
        ("first_event_id", C.c_uint32),
        ("seed", C.c_uint64),
        ("energy_mode", C.c_uint32),
        ("entry_mode", C.c_uint32),
        ("energy_min_mev", C.c_double),
        ("energy_max_mev", C.c_double),
        ("max_incidence_deg", C.c_double),
        ("crystal_center_mm", C.c_float * 3),
        ("crystal_half_size_mm", C.c_float * 3),
        ("step_mm", C.c_double),
        ("density_g_cm3", C.c_double),
        ("scintillation_yield_per_mev", C.c_double),
        ("resolution_scale", C.c_double),
        ("decay_time_ns", C.c_float),
        ("rise_time_ns", C.c_float),
        ("cerenkov", C.c_uint32),
        ("threads", C.c_uint32),
        ("rindex", C.c_double),
        ("cerenkov_energy_min_ev", C.c_double),
        ("cerenkov_energy_max_ev", C.c_double),
        ("volume_id", C.c_uint32),
        ("material_id", C.c_uint32),
        ("spectrum_id", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


# Every symbol include/g4b.h and include/g4b_scheduler.h declare (libg4b.so), with its ctypes signature.
_VP = C.c_void_p
_U32 = C.c_uint32
_U64 = C.c_uint64
_I32 = C.c_int
_PD = C.POINTER(C.c_double)
_PF = C.POINTER(C.c_float)
_PU32 = C.POINTER(C.c_uint32)
_PU64 = C.POINTER(C.c_uint64)
SIGNATURES = {
    "g4b_create": (_I32, [C.POINTER(Config), C.POINTER(_VP)]),
    "g4b_destroy": (_I32, [_VP]),
    "g4b_last_error": (C.c_char_p, [_VP]),
    "g4b_set_scene": (_I32, [_VP, C.POINTER(Scene)]),
    "g4b_enqueue": (_I32, [_VP, _VP, _U32, _PU32, _U32, _PU32]),
    "g4b_relaunch": (_I32, [_VP]),
    "g4b_query_oldest": (_I32, [_VP, _PU64, _PU32]),
    "g4b_poll_oldest": (_I32, [_VP, C.POINTER(C.c_int)]),
    "g4b_complete": (_I32, [_VP, C.POINTER(Output)]),
    "g4b_get_stream": (_I32, [_VP, C.POINTER(_VP)]),
    "g4b_photon_fates": (_I32, [_VP, _PU32, _PD, _U64, _PU64]),
    "g4b_autotune": (_I32, [_VP, _PU32, _U32, _PU32, _U32, _U32, C.POINTER(TuneResult)]),
    "g4b_gradients": (_I32, [_VP, C.POINTER(GradientRequest), C.POINTER(Gradients)]),
    "g4b_eval_fresnel": (_I32, [_I32, _U32, _U32, _PD, _PD, _PD, _PD, _PD, _PD]),
    "g4b_eval_lambertian": (_I32, [_I32, _U32, _U32, _PD, _PD, _PD, _PD]),
    "g4b_eval_math": (_I32, [_I32, _U32, _U32, _PF, _PF]),
    "g4b_eval_uniform": (_I32, [_I32, _U32, _U64, _PU64, _PU32, _PU32, _PU32, _PF]),
    "g4b_host_alloc": (_I32, [C.c_size_t, C.POINTER(_VP)]),
    "g4b_host_free": (_I32, [_VP]),
    "g4b_order_detections_static": (_I32, [_VP, _VP, _U64, _U32, _VP, _VP]),
    "g4b_abi_version": (_U32, []),
    "g4b_scheduler_create": (_I32, [C.POINTER(Config), C.POINTER(Scene), C.POINTER(SchedulerConfig), C.POINTER(_VP)]),
    "g4b_scheduler_create_with_transport": (
        _I32,
        [C.POINTER(TransportOps), _U32, C.POINTER(SchedulerConfig), C.POINTER(_VP)],
    ),
    "g4b_scheduler_submit": (_I32, [_VP, _U32, _VP, _U32, _U64, C.POINTER(Statistics), _PU64]),
    "g4b_scheduler_wait": (_I32, [_VP, _U64, C.c_int64, C.POINTER(Output)]),
    "g4b_scheduler_end_run": (_I32, [_VP]),
    "g4b_scheduler_statistics": (_I32, [_VP, C.POINTER(Statistics), C.POINTER(BatchStatistics)]),
    "g4b_scheduler_destroy": (_I32, [_VP]),
    "g4b_scheduler_replay": (_I32, [_VP, _VP, _PU64, _PU32, _U32, _U32, _U32, _PU64, _PD]),
    "g4b_scheduler_last_error": (C.c_char_p, []),
}
# Every symbol include/g4b_synth.h declares (libg4b_synth.so).
SYNTH_SIGNATURES = {
    "g4b_synth_electrons": (_I32, [C.POINTER(SynthParams), C.POINTER(_VP)]),
    "g4b_synth_isotropic_photons": (
        _I32,
        [_U64, _U32, _U64, _PF, _PF, C.c_double, C.c_double, _U32, _U32, C.POINTER(_VP)],
    ),
    "g4b_synth_view": (
        _I32,
        [_VP, C.POINTER(_VP), _PU32, C.POINTER(_VP), _PU32, C.POINTER(_VP), _PU64],
    ),
    "g4b_synth_free": (None, [_VP]),
    "g4b_synth_last_error": (C.c_char_p, []),
}

_lock = threading.Lock()
_lib: C.CDLL | None = None
_synth: C.CDLL | None = None


def library_path() -> Path:
    return _build.LIBRARY


def load() -> C.CDLL:
    """Loads the engine library, building it first if it is missing or stale."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        try:
            path = _build.build()
        except Exception as error:  # no nvcc, compile error
            if _build.LIBRARY.exists():
                path = _build.LIBRARY
            else:
                raise ImportError(f"the g4b CUDA engine library is missing and cannot be built: {error}") from error
        lib = C.CDLL(str(path))
        for name, (restype, argtypes) in SIGNATURES.items():
            function = getattr(lib, name)
            function.restype = restype
            function.argtypes = argtypes
        if lib.g4b_abi_version() != ABI_VERSION:
            raise ImportError("libg4b.so ABI version does not match the Python binding")
        _lib = lib
        return lib


def load_synth() -> C.CDLL:
    """Loads the seeded genstep source (libg4b_synth.so), building it first if
    it is missing or stale. It needs no GPU and does not load the engine."""
    global _synth
    with _lock:
        if _synth is not None:
            return _synth
        try:
            path = _build.build_synth()
        except Exception as error:
            if _build.SYNTH_LIBRARY.exists():
                path = _build.SYNTH_LIBRARY
            else:
                raise ImportError(f"the genstep source library is missing and cannot be built: {error}") from error
        lib = C.CDLL(str(path))
        for name, (restype, argtypes) in SYNTH_SIGNATURES.items():
            function = getattr(lib, name)
            function.restype = restype
            function.argtypes = argtypes
        _synth = lib
        return lib


def as_ptr(array: np.ndarray, ctype):
    return array.ctypes.data_as(C.POINTER(ctype))
