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

_lock = threading.Lock()
_lib = None
_ref = None


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
        lib.oracle_uniform_f.restype = C.c_float
        lib.oracle_uniform_f.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
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
    status = lib.oracle_transport(*args)
    if status not in (_abi.OK, _abi.ERR_CAPACITY):
        raise RuntimeError(f"oracle failed ({status}): {lib.oracle_last_error().decode()}")
    detections = np.empty(result.detection_count, dtype=_abi.DETECTION_DTYPE)
    if result.detection_count:
        result.detections = detections.ctypes.data
        result.detection_capacity = result.detection_count
        status = lib.oracle_transport(*args)
        if status != _abi.OK:
            raise RuntimeError(f"oracle failed ({status}): {lib.oracle_last_error().decode()}")
    stats = {name: getattr(result.statistics, name) for name, _ in _abi.Statistics._fields_ if name != "reserved"}
    per_event = []
    for i in range(events):
        s = event_stats[i].statistics
        per_event.append((int(event_stats[i].event_id),
                          {name: getattr(s, name) for name, _ in _abi.Statistics._fields_ if name != "reserved"}))
    return OracleOutput(detections, per_event, stats, int(result.total_bounce_count), fates, times,
                        (int(result.coincident_candidate_trace_count), int(result.coincident_candidate_hit_count)))
