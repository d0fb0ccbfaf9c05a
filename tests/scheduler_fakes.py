"""A CPU stand-in for the engine behind the batch scheduler's transport interface.

It keeps the engine's contract (one pending batch, per-event statistics with
the captured and terminal fields, batch sums) and derives detections from the
gensteps by a fixed rule, so the scheduler's batching, routing and checks can
be tested without a GPU: emission j of a batch yields photon_count // 10
detections, photon IDs first_photon_id + k, time_ns = the emission's time + k.
"""
from __future__ import annotations

import ctypes as C
import threading
import time

import numpy as np

from g4go_b200 import DETECTION_DTYPE, _abi

TERMINAL = sum(1 << f for f in (_abi.FIELD_DETECTED, _abi.FIELD_ABSORBED, _abi.FIELD_ESCAPED, _abi.FIELD_TRUNCATED,
                                _abi.FIELD_MAX_BOUNCE, _abi.FIELD_INVALID_STATE, _abi.FIELD_ZERO_STEP))
CAPTURED = 1 << _abi.FIELD_CAPTURED


class TransportFailure(RuntimeError):
    def __init__(self, message: str, status: int = _abi.ERR_CUDA) -> None:
        super().__init__(message)
        self.status = status


def expected_detections(emissions: np.ndarray) -> np.ndarray:
    rows = []
    for e in emissions:
        for k in range(int(e["photon_count"]) // 10):
            rows.append((e["event_id"], e["first_photon_id"] + k, e["time_ns"] + k))
    out = np.zeros(len(rows), dtype=DETECTION_DTYPE)
    if rows:
        out["event_id"] = [r[0] for r in rows]
        out["photon_id"] = [r[1] for r in rows]
        out["time_ns"] = [r[2] for r in rows]
    return out


class FakeTransport:
    """Engine stand-in; `latency_s` is how long a batch 'runs' after enqueue."""

    def __init__(self, latency_s: float = 0.0, corrupt_batch_sum: bool = False, fail_enqueue_at: int = -1,
                 shuffle_detections: bool = False) -> None:
        self.latency_s = latency_s
        self.shuffle_detections = shuffle_detections
        self.corrupt_batch_sum = corrupt_batch_sum
        self.fail_enqueue_at = fail_enqueue_at
        self.batches: list[tuple[np.ndarray, np.ndarray, np.ndarray]] = []
        self.pending = None
        self.started = 0.0
        self.release = threading.Event()
        self.release.set()
        self.max_in_flight_seen = 0
        self.lock = threading.Lock()

    def enqueue(self, emissions, event_ids, indices) -> None:
        if self.pending is not None:
            raise TransportFailure("transport queue is full", _abi.ERR_LOGIC)
        if len(self.batches) == self.fail_enqueue_at:
            raise TransportFailure("injected enqueue failure")
        self.batches.append((emissions, event_ids, indices))
        self.pending = (emissions, event_ids, indices)
        self.started = time.monotonic()

    def poll(self) -> bool:
        if self.pending is None:
            raise TransportFailure("transport queue is empty", _abi.ERR_LOGIC)
        return self.release.is_set() and time.monotonic() - self.started >= self.latency_s

    def _wait(self) -> None:
        self.release.wait()
        remaining = self.latency_s - (time.monotonic() - self.started)
        if remaining > 0:
            time.sleep(remaining)

    def query(self):
        self._wait()
        emissions, event_ids, _ = self.pending
        return int((emissions["photon_count"] // 10).sum()), len(event_ids)

    def complete(self, output) -> None:
        self._wait()
        emissions, event_ids, indices = self.pending
        detections = expected_detections(emissions)
        if self.shuffle_detections:  # as the engine returns them without ordered_detections
            detections = detections[np.random.default_rng(len(self.batches)).permutation(len(detections))]
        if output.detection_capacity < len(detections) or output.event_capacity < len(event_ids):
            raise TransportFailure("capacity", _abi.ERR_CAPACITY)
        if len(detections):
            C.memmove(output.detections, detections.ctypes.data, detections.nbytes)
        output.detection_count = len(detections)
        output.event_count = len(event_ids)
        total = _abi.Statistics()
        total.valid_fields = CAPTURED | TERMINAL
        for i, event_id in enumerate(event_ids):
            mine = emissions[indices == i]
            photons = int(mine["photon_count"].sum())
            detected = int((mine["photon_count"] // 10).sum())
            record = output.event_statistics[i]
            record.event_id = int(event_id)
            s = record.statistics
            s.valid_fields = CAPTURED | TERMINAL
            s.captured_count = photons
            s.detected_count = detected
            s.absorbed_count = photons - detected
            s.max_bounce_count = 7
            total.captured_count += photons
            total.detected_count += detected
            total.absorbed_count += photons - detected
            total.max_bounce_count = 7
        if self.corrupt_batch_sum:
            total.detected_count += 1
        output.statistics = total
        self.pending = None
