"""OpticalBatchScheduler over the engine's streaming batch scheduler (include/g4b_scheduler.h).

Mirrors include/g4go/optical/geant4/OpticalBatchScheduler.hpp:32-93: producer
threads submit one event's gensteps at a time and get a future for that
event's detections and statistics; the native scheduler's transport thread
batches the submissions and keeps up to batches_in_flight batches (eight by
default) on the GPU, one per engine handle. The ctypes calls release the GIL, so Python producer threads run
concurrently with one another and with the transport thread.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _abi
from .transport import (
    DETECTION_DTYPE,
    EMISSION_DTYPE,
    PERF_FIELDS,
    PhotonTransportConfig,
    PhotonTransportOutput,
    Scene,
    _stats_dict,
    raise_for_status,
)

BATCH_FIELDS = tuple(name for name, _ in _abi.BatchStatistics._fields_ if name != "performance")


@dataclass
class BatchSchedulerConfig:
    """The batching fields of PhotonTransportConfig (PhotonTransportConfig.hpp:31-37)."""

    target_photons_per_batch: int = 1_000_000
    max_events_per_batch: int = 10_000
    max_queued_photons: int = 2_000_000
    max_queued_submissions: int = 1_024
    batch_collection_timeout_ms: int = 10
    enable_performance_diagnostics: bool = False
    serial: bool = False  # the reference's order: retire a batch before collecting the next
    batches_in_flight: int = 8  # pipelined: engine handles and batches on the GPU at once (at most 8)

    def to_c(self) -> _abi.SchedulerConfig:
        config = _abi.SchedulerConfig()
        config.abi_version = _abi.ABI_VERSION
        config.target_photons_per_batch = int(self.target_photons_per_batch)
        config.max_events_per_batch = int(self.max_events_per_batch)
        config.max_queued_photons = int(self.max_queued_photons)
        config.max_queued_submissions = int(self.max_queued_submissions)
        config.batch_collection_timeout_ms = int(self.batch_collection_timeout_ms)
        config.enable_performance_diagnostics = int(bool(self.enable_performance_diagnostics))
        config.serial = int(bool(self.serial))
        config.batches_in_flight = int(self.batches_in_flight)
        return config


@dataclass
class OpticalSubmission:
    """OpticalSubmission (PhotonTransport.hpp:165-171): one event's gensteps."""

    event_id: int
    emissions: np.ndarray
    photon_count: int | None = None  # None: the sum over the emissions
    source_statistics: dict | None = None

    def __post_init__(self) -> None:
        self.emissions = np.ascontiguousarray(self.emissions, dtype=EMISSION_DTYPE)
        if self.photon_count is None:
            self.photon_count = int(self.emissions["photon_count"].sum(dtype=np.uint64))


def _statistics_struct(values: dict | None) -> _abi.Statistics:
    stats = _abi.Statistics()
    for name, value in (values or {}).items():
        setattr(stats, name, value)
    return stats


class PhotonTransportFuture:
    """std::shared_future<PhotonTransportOutput> of one submission."""

    def __init__(self, scheduler: "OpticalBatchScheduler", ticket: int) -> None:
        self._scheduler = scheduler
        self._ticket = ticket
        self._result: PhotonTransportOutput | None = None
        self._error: BaseException | None = None

    def done(self) -> bool:
        if self._result is not None or self._error is not None:
            return True
        return self._fetch(0)

    def result(self, timeout: float | None = None) -> PhotonTransportOutput:
        if self._result is None and self._error is None:
            if not self._fetch(-1 if timeout is None else int(timeout * 1000)):
                raise TimeoutError("optical submission not transported yet")
        if self._error is not None:
            raise self._error
        return self._result

    def _fetch(self, timeout_ms: int) -> bool:
        lib = self._scheduler._lib
        capacity = 4096
        while True:
            detections = np.empty(capacity, dtype=DETECTION_DTYPE)
            event = (_abi.EventStatistics * 1)()
            output = _abi.Output()
            output.detections = detections.ctypes.data_as(C.c_void_p)
            output.detection_capacity = capacity
            output.event_statistics = C.cast(event, C.POINTER(_abi.EventStatistics))
            output.event_capacity = 1
            status = lib.g4b_scheduler_wait(self._scheduler._handle, self._ticket, timeout_ms, C.byref(output))
            if status == _abi.ERR_TIMEOUT:
                return False
            if status == _abi.ERR_CAPACITY:
                capacity = int(output.detection_count)
                continue
            if status != _abi.OK:
                try:
                    raise_for_status(status, lib.g4b_scheduler_last_error().decode())
                except Exception as error:  # the future keeps the failure, as std::future does
                    self._error = error
                return True
            self._result = PhotonTransportOutput(
                detections=detections[: output.detection_count].copy(),
                statistics=_stats_dict(output.statistics),
                performance={name: getattr(output.performance, name) for name in PERF_FIELDS},
                event_statistics=[(int(event[0].event_id), _stats_dict(event[0].statistics))],
            )
            return True


class OpticalBatchScheduler:
    """OpticalBatchScheduler: BeginRun / Submit / EndRun over the native scheduler.

    transports: objects with enqueue(emissions, event_ids, emission_event_indices),
    poll() -> bool, query() -> (detections, events) and complete(output) driven
    instead of engine handles (one to eight; see g4b_scheduler_create_with_transport)."""

    def __init__(self, config: PhotonTransportConfig | None = None, scene: Scene | None = None,
                 batching: BatchSchedulerConfig | None = None, transports: Sequence | None = None) -> None:
        self._lib = _abi.load()
        self.config = config or PhotonTransportConfig()
        self.scene = scene
        self.batching = batching or BatchSchedulerConfig()
        self._transports = list(transports) if transports is not None else None
        self._ops_keepalive: list = []
        self._handle: C.c_void_p | None = None

    # -- lifetime ---------------------------------------------------------
    def begin_run(self) -> None:
        if self._handle is not None:
            return
        handle = C.c_void_p()
        batching = self.batching.to_c()
        if self._transports is None:
            if self.scene is None:
                raise ValueError("a scene is required to run the engine")
            c_scene = self.scene.to_c()
            status = self._lib.g4b_scheduler_create(C.byref(self.config.to_c()), C.byref(c_scene.struct),
                                                    C.byref(batching), C.byref(handle))
        else:
            ops = (_abi.TransportOps * len(self._transports))()
            for i, transport in enumerate(self._transports):
                ops[i] = _transport_ops(transport, self._ops_keepalive)
            status = self._lib.g4b_scheduler_create_with_transport(ops, len(self._transports), C.byref(batching),
                                                                   C.byref(handle))
        if status != _abi.OK:
            raise_for_status(status, self._lib.g4b_scheduler_last_error().decode())
        self._handle = handle

    def end_run(self) -> None:
        if self._handle is not None:
            self._check(self._lib.g4b_scheduler_end_run(self._handle))

    def close(self) -> None:
        if self._handle is not None:
            self._lib.g4b_scheduler_destroy(self._handle)
            self._handle = None

    def __enter__(self) -> "OpticalBatchScheduler":
        self.begin_run()
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int) -> None:
        if status != _abi.OK:
            raise_for_status(status, self._lib.g4b_scheduler_last_error().decode())

    # -- the reference interface -------------------------------------------
    def submit(self, submission: OpticalSubmission) -> PhotonTransportFuture:
        """Submit (OpticalBatchScheduler.cpp:144-218)."""
        if self._handle is None:
            from .transport import LogicError
            raise LogicError("optical submission queue is not ready")
        ticket = C.c_uint64()
        source = _statistics_struct(submission.source_statistics)
        emissions = submission.emissions
        self._check(self._lib.g4b_scheduler_submit(
            self._handle, int(submission.event_id), emissions.ctypes.data_as(C.c_void_p), emissions.shape[0],
            int(submission.photon_count), C.byref(source), C.byref(ticket)))
        return PhotonTransportFuture(self, int(ticket.value))

    def replay(self, submissions: Sequence[OpticalSubmission], producers: int = 4, window: int = 32) -> tuple[int, float]:
        """Streams the submissions through the scheduler from `producers` native
        threads (g4b_scheduler_replay); returns (detections, wall seconds)."""
        emissions = np.concatenate([sub.emissions for sub in submissions]) if submissions else \
            np.zeros(0, dtype=EMISSION_DTYPE)
        offsets = np.zeros(len(submissions) + 1, dtype=np.uint64)
        offsets[1:] = np.cumsum([sub.emissions.shape[0] for sub in submissions])
        event_ids = np.array([sub.event_id for sub in submissions], dtype=np.uint32)
        detections = C.c_uint64()
        seconds = C.c_double()
        self._check(self._lib.g4b_scheduler_replay(
            self._handle, emissions.ctypes.data_as(C.c_void_p), _abi.as_ptr(offsets, C.c_uint64),
            _abi.as_ptr(event_ids, C.c_uint32), len(submissions), producers, window, C.byref(detections),
            C.byref(seconds)))
        return int(detections.value), float(seconds.value)

    def run_statistics(self) -> dict:
        run = _abi.Statistics()
        self._check(self._lib.g4b_scheduler_statistics(self._handle, C.byref(run), None))
        return _stats_dict(run)

    def batch_statistics(self) -> dict:
        batch = _abi.BatchStatistics()
        self._check(self._lib.g4b_scheduler_statistics(self._handle, None, C.byref(batch)))
        values = {name: getattr(batch, name) for name in BATCH_FIELDS}
        values["performance"] = {name: getattr(batch.performance, name) for name in PERF_FIELDS}
        return values


def _transport_ops(transport, keepalive: list) -> _abi.TransportOps:
    """g4b_transport_ops calling a Python transport; exceptions become statuses."""
    state = {"error": C.create_string_buffer(b"no error")}

    def guarded(body):
        try:
            return body()
        except Exception as error:  # reported through last_error
            state["error"] = C.create_string_buffer(str(error).encode())
            return getattr(error, "status", _abi.ERR_LOGIC)

    def enqueue(_, emissions, emission_count, event_ids, event_count, indices):
        def body():
            size = emission_count * EMISSION_DTYPE.itemsize
            raw = C.string_at(emissions, size) if emission_count else b""
            batch = np.frombuffer(raw, dtype=EMISSION_DTYPE).copy()
            ids = np.ctypeslib.as_array(event_ids, shape=(event_count,)).copy() if event_count else np.empty(0, np.uint32)
            idx = np.ctypeslib.as_array(indices, shape=(emission_count,)).copy() if emission_count else np.empty(0, np.uint32)
            transport.enqueue(batch, ids, idx)
            return _abi.OK
        return guarded(body)

    def poll(_, ready):
        def body():
            ready[0] = 1 if transport.poll() else 0
            return _abi.OK
        return guarded(body)

    def query(_, detections, events):
        def body():
            d, e = transport.query()
            detections[0] = d
            events[0] = e
            return _abi.OK
        return guarded(body)

    def complete(_, output):
        return guarded(lambda: transport.complete(output.contents) or _abi.OK)

    def last_error(_):
        return C.addressof(state["error"])

    ops = _abi.TransportOps()
    ops.context = None
    callbacks = (_abi.TRANSPORT_ENQUEUE(enqueue), _abi.TRANSPORT_POLL(poll), _abi.TRANSPORT_QUERY(query),
                 _abi.TRANSPORT_COMPLETE(complete), _abi.TRANSPORT_LAST_ERROR(last_error))
    ops.enqueue, ops.poll, ops.query, ops.complete, ops.last_error = callbacks
    keepalive.append((callbacks, state))
    return ops
