"""ctypes binding of the CPU oracle (oracle/cpu_transport.cpp) and of the
reference's own boundary physics compiled from the reference tree (oracle/_ref).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine, never the engine.
The record layouts are the engine's ABI types (include/g4b.h), reused here so
both sides read the same bytes.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import threading
from pathlib import Path

import numpy as np

from g4go_b200 import _abi

ORACLE_DIR = Path(__file__).resolve().parent
LIBRARY = ORACLE_DIR / "_build" / "liboracle.so"
REFERENCE_LIBRARY = ORACLE_DIR / "_ref" / "libref_boundary.so"
REFERENCE_TRANSPORT_LIBRARY = ORACLE_DIR / "_ref" / "libref_transport.so"

_lock = threading.Lock()
_lib = None
_ref = None
_ref_transport = None


class OracleResult(C.Structure):
    _fields_ = [
        ("detections", C.c_void_p),
        ("detection_capacity", C.c_uint64),
        ("detection_count", C.c_uint64),
        ("event_statistics", C.POINTER(_abi.EventStatistics)),
        ("event_capacity", C.c_uint32),
        ("event_count", C.c_uint32),
        ("statistics", _abi.Statistics),
        ("total_bounce_count", C.c_uint64),
        ("coincident_candidate_trace_count", C.c_uint64),
        ("coincident_candidate_hit_count", C.c_uint64),
        ("photon_fate", C.POINTER(C.c_uint32)),
        ("photon_time_ns", C.POINTER(C.c_double)),
        ("photon_capacity", C.c_uint64),
        ("photon_count", C.c_uint64),
    ]


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


def load():
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        sources = [ORACLE_DIR / "cpu_transport.cpp", ORACLE_DIR / "g4b_oracle.h"]
        if not LIBRARY.exists() or any(s.stat().st_mtime > LIBRARY.stat().st_mtime for s in sources):
            build()
        lib = C.CDLL(str(LIBRARY))
        f3 = C.POINTER(C.c_float)
        d3 = C.POINTER(C.c_double)
        lib.oracle_transport.restype = C.c_int
        lib.oracle_transport.argtypes = [
            C.POINTER(_abi.Scene), C.POINTER(_abi.Config), C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32,
            C.POINTER(C.c_uint32), C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(OracleResult),
        ]
        lib.oracle_last_error.restype = C.c_char_p
        lib.oracle_take_detections.restype = C.c_uint64
        lib.oracle_take_detections.argtypes = [C.c_void_p, C.c_uint64]
        lib.oracle_fresnel_f.argtypes = [f3, f3, f3, C.c_float, C.c_float, f3]
        lib.oracle_fresnel_d.argtypes = [d3, d3, d3, C.c_double, C.c_double, d3]
        lib.oracle_classify_surface.restype = C.c_int
        lib.oracle_classify_surface.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_float]
        lib.oracle_evaluate_absorption.restype = C.c_int
        lib.oracle_evaluate_absorption.argtypes = [C.c_float, C.c_int, C.c_float]
        lib.oracle_lambertian_f.argtypes = [f3, C.c_float, C.c_float, f3]
        lib.oracle_lambertian_d.argtypes = [d3, C.c_double, C.c_double, d3]
        for name, t in (("log_f", C.c_float), ("exp_f", C.c_float), ("log_d", C.c_double), ("exp_d", C.c_double)):
            fn = getattr(lib, "oracle_" + name)
            fn.restype = t
            fn.argtypes = [t]
        lib.oracle_sincos_turn_f.argtypes = [C.c_float, f3, f3]
        lib.oracle_sincos_turn_d.argtypes = [C.c_double, d3, d3]
        lib.oracle_sample_property_f.restype = C.c_float
        lib.oracle_sample_property_f.argtypes = [f3, f3, C.c_uint32, C.c_float, C.c_float]
        lib.oracle_sample_spectrum_f.restype = C.c_float
        lib.oracle_sample_spectrum_f.argtypes = [f3, f3, C.c_uint32, C.c_float]
        lib.oracle_uniform_f.restype = C.c_float
        lib.oracle_uniform_f.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        lib.oracle_generate.restype = C.c_int
        lib.oracle_generate.argtypes = [C.POINTER(_abi.Scene), C.c_uint64, C.c_uint32, C.c_void_p, C.c_uint32,
                                        C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.c_uint32, d3, d3]
        lib.oracle_spectrum_cdf.restype = C.c_uint32
        lib.oracle_spectrum_cdf.argtypes = [f3, f3, C.c_uint32, f3]
        _lib = lib
        return lib


def load_reference():
    """The reference's OptiXBoundaryPhysics.cuh compiled from its own sources, or None."""
    global _ref
    with _lock:
        if _ref is not None:
            return _ref
        if not REFERENCE_LIBRARY.exists():
            try:
                subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "ref"], check=True)
            except Exception:
                return None
        if not REFERENCE_LIBRARY.exists():
            return None
        lib = C.CDLL(str(REFERENCE_LIBRARY))
        f3 = C.POINTER(C.c_float)
        lib.ref_fresnel.argtypes = [f3, f3, f3, C.c_float, C.c_float, f3]
        lib.ref_classify_surface.restype = C.c_int
        lib.ref_classify_surface.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_float]
        lib.ref_evaluate_absorption.restype = C.c_int
        lib.ref_evaluate_absorption.argtypes = [C.c_float, C.c_int, C.c_float]
        lib.ref_lambertian.argtypes = [f3, C.c_float, C.c_float, f3]
        _ref = lib
        return lib


class RefResult(C.Structure):
    _fields_ = [
        ("fate", C.POINTER(C.c_uint32)),
        ("zero_steps", C.POINTER(C.c_uint32)),
        ("detections", C.c_void_p),
        ("detection_count", C.c_uint64),
        ("event_statistics", C.POINTER(_abi.EventStatistics)),
        ("statistics", _abi.Statistics),
        ("total_bounce_count", C.c_uint64),
        ("coincident_candidate_trace_count", C.c_uint64),
        ("coincident_candidate_hit_count", C.c_uint64),
    ]


def load_reference_transport():
    """The reference's device program (OptiXTransportDevice.cu) compiled for
    the host from its own sources (oracle/Makefile, ref_transport_shim.cpp), or
    None where the reference tree was not there to build it."""
    global _ref_transport
    with _lock:
        if _ref_transport is not None:
            return _ref_transport
        if not REFERENCE_TRANSPORT_LIBRARY.exists():
            try:
                subprocess.run(["make", "-s", "-C", str(ORACLE_DIR), "ref"], check=True)
            except Exception:
                return None
        if not REFERENCE_TRANSPORT_LIBRARY.exists():
            return None
        lib = C.CDLL(str(REFERENCE_TRANSPORT_LIBRARY))
        f = C.POINTER(C.c_float)
        u32 = C.POINTER(C.c_uint32)
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_uniform.restype = C.c_float
        lib.ref_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        lib.ref_sample_property.restype = C.c_float
        lib.ref_sample_property.argtypes = [f, f, C.c_uint32, C.c_uint32, C.c_float, C.c_float]
        lib.ref_sample_spectrum.restype = C.c_float
        lib.ref_sample_spectrum.argtypes = [f, f, C.c_uint32, C.c_float]
        lib.ref_spectrum_cdf.restype = C.c_uint32
        lib.ref_spectrum_cdf.argtypes = [f, f, C.c_uint32, f]
        lib.ref_generate.restype = C.c_int
        lib.ref_generate.argtypes = [C.POINTER(_abi.Scene), C.c_uint64, C.c_void_p, C.c_uint32, u32, u32, C.c_uint32,
                                     f, C.POINTER(C.c_double)]
        lib.ref_transport.restype = C.c_int
        lib.ref_transport.argtypes = [
            C.POINTER(_abi.Scene), C.POINTER(_abi.Config), C.c_void_p, C.c_uint32, u32, C.c_uint32, u32,
            C.c_uint32, C.c_uint64, C.c_uint64, C.POINTER(RefResult),
        ]
        _ref_transport = lib
        return lib


def reference_transport(scene, batch, config, threads: int = 0, photon_range: tuple[int, int] | None = None):
    """The reference's own __raygen__rg over the batch's photons (or a slice):
    detections in flattened order, per-photon fate (outcome | bounces << 3)
    and zero-step counts, per-event and run statistics."""
    lib = load_reference_transport()
    if lib is None:
        raise RuntimeError("the reference's device program was not built (oracle/_ref)")
    c_scene = scene.to_c()
    c_config = config.to_c()
    begin, end = photon_range if photon_range is not None else (0, batch.photon_count)
    span = end - begin
    events = batch.event_ids.shape[0]
    fates = np.zeros(span, dtype=np.uint32)
    zero_steps = np.zeros(span, dtype=np.uint32)
    detections = np.zeros(span, dtype=_abi.DETECTION_DTYPE)
    event_stats = (_abi.EventStatistics * max(events, 1))()
    result = RefResult()
    result.fate = _abi.as_ptr(fates, C.c_uint32)
    result.zero_steps = _abi.as_ptr(zero_steps, C.c_uint32)
    result.detections = detections.ctypes.data
    result.event_statistics = C.cast(event_stats, C.POINTER(_abi.EventStatistics))
    status = lib.ref_transport(C.byref(c_scene.struct), C.byref(c_config), batch.emissions.ctypes.data_as(C.c_void_p),
                               batch.emissions.shape[0], _abi.as_ptr(batch.event_ids, C.c_uint32), events,
                               _abi.as_ptr(batch.emission_event_indices, C.c_uint32), threads, begin, end,
                               C.byref(result))
    if status != 0:
        raise RuntimeError(f"reference transport failed: {lib.ref_last_error().decode()}")
    from g4go_b200.transport import EventStatisticsList

    stats = {name: getattr(result.statistics, name) for name, _ in _abi.Statistics._fields_ if name != "reserved"}
    per_event = EventStatisticsList(np.ctypeslib.as_array(event_stats)[:events].copy())
    out = OracleOutput(detections[: result.detection_count].copy(), per_event, stats, int(result.total_bounce_count),
                       fates, None, (int(result.coincident_candidate_trace_count),
                                     int(result.coincident_candidate_hit_count)))
    out.zero_steps = zero_steps
    return out


def generate(scene, batch, seed: int, emission_index, local, precision: str = "fp32", reference: bool = False):
    """GeneratePhoton for photon local[i] of genstep emission_index[i], by the
    oracle (FP32 or FP64) or by the reference's own code: (rows, time), each
    row position[3], direction[3], polarization[3], energy."""
    index = np.ascontiguousarray(emission_index, dtype=np.uint32)
    local = np.ascontiguousarray(local, dtype=np.uint32)
    n = index.size
    c_scene = scene.to_c()
    times = np.empty(n, dtype=np.float64)
    if reference:
        lib = load_reference_transport()
        if lib is None:
            raise RuntimeError("the reference's device program was not built (oracle/_ref)")
        rows = np.empty((n, 10), dtype=np.float32)
        status = lib.ref_generate(C.byref(c_scene.struct), seed, batch.emissions.ctypes.data_as(C.c_void_p),
                                  batch.emissions.shape[0], _abi.as_ptr(index, C.c_uint32),
                                  _abi.as_ptr(local, C.c_uint32), n, _abi.as_ptr(rows, C.c_float),
                                  _abi.as_ptr(times, C.c_double))
        if status != 0:
            raise RuntimeError(f"reference generation failed: {lib.ref_last_error().decode()}")
        return rows.astype(np.float64), times
    lib = load()
    rows = np.empty((n, 10), dtype=np.float64)
    status = lib.oracle_generate(C.byref(c_scene.struct), seed,
                                 _abi.PRECISION_FP64 if precision == "fp64" else _abi.PRECISION_FP32,
                                 batch.emissions.ctypes.data_as(C.c_void_p), batch.emissions.shape[0],
                                 _abi.as_ptr(index, C.c_uint32), _abi.as_ptr(local, C.c_uint32), n,
                                 _abi.as_ptr(rows, C.c_double), _abi.as_ptr(times, C.c_double))
    if status != 0:
        raise RuntimeError(f"oracle generation failed: {lib.oracle_last_error().decode()}")
    return rows, times


class OracleOutput:
    def __init__(self, detections, event_statistics, statistics, total_bounces, fates, times, coincident):
        self.detections = detections
        self.event_statistics = event_statistics
        self.statistics = statistics
        self.total_bounce_count = total_bounces
        self.photon_fate = fates
        self.photon_time_ns = times
        self.coincident = coincident


def transport(scene, batch, config, threads: int = 0, photon_range: tuple[int, int] | None = None,
              record_fates: bool = False) -> OracleOutput:
    """Runs the oracle on a batch (a g4go_b200 PhotonTransportBatch) under a PhotonTransportConfig."""
    lib = load()
    c_scene = scene.to_c()
    c_config = config.to_c()
    begin, end = photon_range if photon_range is not None else (0, 0)
    total = batch.photon_count
    span = (end if end else total) - begin
    events = batch.event_ids.shape[0]
    event_stats = (_abi.EventStatistics * max(events, 1))()
    result = OracleResult()
    result.event_statistics = C.cast(event_stats, C.POINTER(_abi.EventStatistics))
    result.event_capacity = events
    fates = times = None
    if record_fates:
        fates = np.zeros(span, dtype=np.uint32)
        times = np.zeros(span, dtype=np.float64)
        result.photon_fate = _abi.as_ptr(fates, C.c_uint32)
        result.photon_time_ns = _abi.as_ptr(times, C.c_double)
        result.photon_capacity = span
    args = (
        C.byref(c_scene.struct), C.byref(c_config), batch.emissions.ctypes.data_as(C.c_void_p),
        batch.emissions.shape[0], _abi.as_ptr(batch.event_ids, C.c_uint32), events,
        _abi.as_ptr(batch.emission_event_indices, C.c_uint32), threads, begin, end, C.byref(result),
    )
    # one run: without a detection buffer the oracle keeps the detections on
    # this thread, and oracle_take_detections copies them out afterwards
    status = lib.oracle_transport(*args)
    if status != _abi.OK:
        raise RuntimeError(f"oracle failed ({status}): {lib.oracle_last_error().decode()}")
    detections = np.empty(result.detection_count, dtype=_abi.DETECTION_DTYPE)
    taken = lib.oracle_take_detections(detections.ctypes.data_as(C.c_void_p), detections.shape[0])
    if taken != detections.shape[0]:
        raise RuntimeError(f"oracle kept {taken} detections, reported {detections.shape[0]}")
    stats = {name: getattr(result.statistics, name) for name, _ in _abi.Statistics._fields_ if name != "reserved"}
    # the per-event records stay one numpy array until first read (the same
    # list view the engine's binding returns), so a large batch's slice pays
    # nothing per event
    from g4go_b200.transport import EventStatisticsList

    per_event = EventStatisticsList(np.ctypeslib.as_array(event_stats)[:events].copy())
    return OracleOutput(detections, per_event, stats, int(result.total_bounce_count), fates, times,
                        (int(result.coincident_candidate_trace_count), int(result.coincident_candidate_hit_count)))
