"""The batch scheduler over the engine on the GPU.

Every photon's history depends only on its RNG counters (seed, event ID,
photon ID), so an event's detections and statistics must not depend on which
batch it lands in: events submitted one at a time from several threads, and
batched by the scheduler however the timing falls, must come back bit for bit
as the CPU oracle transports the same gensteps in one batch, and as one
direct engine batch of them.
"""
import threading

import numpy as np
import pytest

from g4go_b200 import PhotonTransportConfig, TransportHost, scenes
from g4go_b200.scheduler import BatchSchedulerConfig, OpticalBatchScheduler, OpticalSubmission

pytestmark = pytest.mark.gpu

SEED = 2024
# the transport's terminal counters; the captured count comes from the
# submission's source statistics (CompleteBatch keeps only terminal fields of
# the transport's per-event record, OpticalBatchScheduler.cpp:309)
COUNTERS = ("detected_count", "absorbed_count", "escaped_count", "truncated_count", "max_bounce_count",
            "invalid_state_count", "zero_step_count")


def split_by_event(out):
    return {event_id: (out.detections[out.detections["event_id"] == event_id], stats)
            for event_id, stats in out.event_statistics}


@pytest.fixture(scope="module")
def direct(oracle):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=300, seed=3)
    with TransportHost(PhotonTransportConfig(seed=SEED)) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch()
    reference = oracle.transport(scene, batch, PhotonTransportConfig(seed=SEED, precision="fp32"))
    per_event = split_by_event(reference)
    engine = split_by_event(out)
    for event_id, (detections, stats) in per_event.items():  # the direct batch is the oracle's too
        assert engine[event_id][0].tobytes() == detections.tobytes(), event_id
        assert all(engine[event_id][1][name] == stats[name] for name in COUNTERS), event_id
    submissions = [OpticalSubmission(int(event_id), batch.emissions[batch.emission_event_indices == i])
                   for i, event_id in enumerate(batch.event_ids)]
    return scene, submissions, per_event


@pytest.mark.parametrize("serial", [False, True])
def test_scheduled_events_match_the_oracle(direct, serial):
    scene, submissions, per_event = direct
    batching = BatchSchedulerConfig(target_photons_per_batch=1_500_000, batch_collection_timeout_ms=2, serial=serial)
    with OpticalBatchScheduler(PhotonTransportConfig(seed=SEED), scene, batching) as scheduler:
        futures = {}
        lock = threading.Lock()

        def produce(k):
            for submission in submissions[k::4]:
                future = scheduler.submit(submission)
                with lock:
                    futures[submission.event_id] = future

        threads = [threading.Thread(target=produce, args=(k,)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for event_id, future in futures.items():
            out = future.result(timeout=120)
            want_detections, want_stats = per_event[event_id]
            assert out.detections.tobytes() == want_detections.tobytes(), event_id
            for name in COUNTERS:
                assert out.statistics[name] == want_stats[name], (event_id, name)
        scheduler.end_run()
        stats = scheduler.batch_statistics()
        assert stats["event_count"] == len(submissions)
        assert stats["batch_count"] >= 2
        if not serial:
            assert stats["overlapped_batch_count"] >= 1
        run = scheduler.run_statistics()
        assert run["detected_count"] == sum(len(d) for d, _ in per_event.values())
