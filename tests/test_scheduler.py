"""The batch scheduler (include/g4b_scheduler.h) on the CPU, over a stand-in transport.

Follows OpticalBatchScheduler (src/optical/geant4/OpticalBatchScheduler.cpp):
Submit's checks (:152-164), zero-photon submissions (:169-193), the queue
limits (:195-202), batch collection (:462-509), the per-event split and its
consistency checks (:230-446), EndRun draining the queue (:122-142) and a
transport failure failing the run (:595-634).
"""
import threading
import time

import numpy as np
import pytest

from g4go_b200 import EMISSION_DTYPE, LogicError, _abi
from g4go_b200.scheduler import BatchSchedulerConfig, OpticalBatchScheduler, OpticalSubmission
from scheduler_fakes import CAPTURED, TERMINAL, FakeTransport, expected_detections


def event(event_id: int, photons_per_emission=(30, 45, 12)) -> OpticalSubmission:
    emissions = np.zeros(len(photons_per_emission), dtype=EMISSION_DTYPE)
    emissions["event_id"] = event_id
    emissions["photon_count"] = photons_per_emission
    emissions["first_photon_id"] = np.concatenate([[0], np.cumsum(photons_per_emission)[:-1]])
    emissions["time_ns"] = np.arange(len(photons_per_emission), dtype=np.float32) * 100 + event_id
    return OpticalSubmission(event_id, emissions, source_statistics={"generated_count": 5, "valid_fields": 1})


def scheduler(transports, **batching) -> OpticalBatchScheduler:
    s = OpticalBatchScheduler(batching=BatchSchedulerConfig(**batching), transports=transports)
    s.begin_run()
    return s


@pytest.mark.parametrize("transports,serial", [(1, True), (1, False), (2, False)])
def test_events_from_many_threads_get_their_own_detections(transports, serial):
    fakes = [FakeTransport(latency_s=0.002) for _ in range(transports)]
    s = scheduler(fakes, target_photons_per_batch=400, batch_collection_timeout_ms=2, serial=serial)
    futures = {}
    lock = threading.Lock()

    def produce(first):
        for event_id in range(first, 120, 4):
            f = s.submit(event(event_id, (10 + event_id, 25, 40)))
            with lock:
                futures[event_id] = f

    threads = [threading.Thread(target=produce, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for event_id, f in futures.items():
        out = f.result(timeout=30)
        want = expected_detections(event(event_id, (10 + event_id, 25, 40)).emissions)
        assert np.array_equal(out.detections["photon_id"], want["photon_id"])
        assert np.array_equal(out.detections["event_id"], want["event_id"])
        assert out.statistics["detected_count"] == len(want)
        assert out.statistics["generated_count"] == 5
        assert out.statistics["valid_fields"] == 1 | TERMINAL  # source fields without captured + terminal fields
        assert out.event_statistics[0][0] == event_id
    s.end_run()
    run = s.run_statistics()
    batch = s.batch_statistics()
    assert batch["event_count"] == 120
    assert batch["photon_count"] == sum(10 + e + 65 for e in range(120))
    assert run["detected_count"] == sum(len(expected_detections(event(e, (10 + e, 25, 40)).emissions))
                                        for e in range(120))
    assert run["generated_count"] == 5 * 120
    assert batch["max_batch_photon_count"] >= 400 or batch["batch_count"] == 1
    if serial or transports == 1:
        assert batch["overlapped_batch_count"] == 0
    s.close()


@pytest.mark.parametrize("cap,expected", [(10, [1, 3, 3, 1]), (2, [1, 2, 2, 2, 1])])
def test_target_photon_count_and_event_cap_close_batches(cap, expected):
    """Events of 100 photons, target 250: a batch closes at 300 photons (three
    events) or at the event cap, whichever comes first (:482)."""
    fake = FakeTransport()
    fake.release.clear()  # hold the first batch so the rest queue up behind it
    s = scheduler([fake], target_photons_per_batch=250, max_events_per_batch=cap, batch_collection_timeout_ms=1,
                  serial=True)
    futures = [s.submit(event(0, (100,)))]
    time.sleep(0.1)  # event 0 alone is on the transport (its collection deadline passed)
    futures += [s.submit(event(e, (100,))) for e in range(1, 8)]
    fake.release.set()
    for f in futures:
        f.result(timeout=30)
    s.close()
    assert [len(ids) for _, ids, _ in fake.batches] == expected


def test_submission_checks():
    s = scheduler([FakeTransport()])
    good = event(1)
    with pytest.raises(ValueError, match="photon count does not match"):
        s.submit(OpticalSubmission(1, good.emissions, photon_count=good.photon_count + 1))
    with pytest.raises(ValueError, match="empty optical submissions cannot contain emissions"):
        empty = good.emissions.copy()
        empty["photon_count"] = 0
        s.submit(OpticalSubmission(1, empty, photon_count=0))
    with pytest.raises(ValueError, match="photon count does not match"):  # checked first, as in Submit
        s.submit(OpticalSubmission(1, np.zeros(0, dtype=EMISSION_DTYPE), photon_count=10))
    with pytest.raises(ValueError, match="event ID does not match"):
        s.submit(OpticalSubmission(2, good.emissions))
    s.close()


def test_zero_photon_submission_completes_at_once():
    fake = FakeTransport()
    s = scheduler([fake])
    f = s.submit(OpticalSubmission(9, np.zeros(0, dtype=EMISSION_DTYPE), photon_count=0,
                                   source_statistics={"generated_count": 3, "captured_count": 0,
                                                      "valid_fields": 1 | CAPTURED}))
    assert f.done()
    out = f.result()
    assert len(out.detections) == 0
    assert out.statistics["generated_count"] == 3
    assert out.statistics["valid_fields"] == 1 | CAPTURED | TERMINAL
    assert s.run_statistics()["valid_fields"] & TERMINAL == TERMINAL
    assert fake.batches == []
    s.close()


def test_queue_limit_blocks_producers_until_a_batch_is_taken():
    fake = FakeTransport()
    fake.release.clear()
    s = scheduler([fake], max_queued_submissions=2, target_photons_per_batch=10**6, batch_collection_timeout_ms=1,
                  serial=True)
    first = s.submit(event(0))
    time.sleep(0.1)  # event 0 is on the held transport; the queue is empty again
    s.submit(event(1))
    s.submit(event(2))
    done = threading.Event()

    def third():
        s.submit(event(3))
        done.set()

    t = threading.Thread(target=third)
    t.start()
    assert not done.wait(0.3)  # two queued submissions: the third waits
    fake.release.set()
    assert done.wait(10)
    t.join()
    first.result(timeout=10)
    s.end_run()
    assert s.batch_statistics()["event_count"] == 4
    s.close()


def test_end_run_transports_everything_queued():
    fake = FakeTransport(latency_s=0.001)
    s = scheduler([fake], target_photons_per_batch=200, batch_collection_timeout_ms=50)
    futures = [s.submit(event(e)) for e in range(40)]
    s.end_run()
    assert all(f.done() for f in futures)
    assert sum(len(ids) for _, ids, _ in fake.batches) == 40
    with pytest.raises(LogicError):
        s.submit(event(99))
    s.close()


def test_inconsistent_transport_statistics_fail_the_run():
    s = scheduler([FakeTransport(corrupt_batch_sum=True)], batch_collection_timeout_ms=1)
    f = s.submit(event(1))
    with pytest.raises(LogicError, match="batch/event statistics mismatch in detected count"):
        f.result(timeout=10)
    time.sleep(0.05)
    with pytest.raises(LogicError, match="mismatch"):
        s.submit(event(2))
    s.close()


def test_transport_failure_fails_every_pending_request():
    fake = FakeTransport(latency_s=0.05, fail_enqueue_at=1)
    s = scheduler([fake], target_photons_per_batch=50, max_events_per_batch=1, batch_collection_timeout_ms=1)
    futures = [s.submit(event(e)) for e in range(6)]
    results = []
    for f in futures:
        try:
            f.result(timeout=10)
            results.append("ok")
        except RuntimeError as error:
            assert "injected enqueue failure" in str(error)
            results.append("failed")
    assert results.count("failed") >= 5  # everything not handed out before the failure
    s.close()


def test_duplicate_event_ids_in_one_batch_fail_the_run():
    fake = FakeTransport()
    fake.release.clear()
    s = scheduler([fake], batch_collection_timeout_ms=200, serial=True)
    s.submit(event(0))
    time.sleep(0.1)
    a = s.submit(event(5))
    b = s.submit(event(5))
    fake.release.set()
    for f in (a, b):
        with pytest.raises(ValueError, match="duplicate event IDs"):
            f.result(timeout=10)
    s.close()


def test_two_transports_keep_two_batches_in_flight():
    fakes = [FakeTransport(latency_s=0.02), FakeTransport(latency_s=0.02)]
    s = scheduler(fakes, target_photons_per_batch=100, max_events_per_batch=1, batch_collection_timeout_ms=1)
    futures = [s.submit(event(e)) for e in range(12)]
    for f in futures:
        f.result(timeout=30)
    s.end_run()
    stats = s.batch_statistics()
    assert stats["batch_count"] == 12
    assert stats["overlapped_batch_count"] >= 6
    assert len(fakes[0].batches) >= 4 and len(fakes[1].batches) >= 4
    s.close()


def test_scheduler_symbols_are_exported():
    lib = _abi.load()
    for name in ("g4b_scheduler_create", "g4b_scheduler_create_with_transport", "g4b_scheduler_submit",
                 "g4b_scheduler_wait", "g4b_scheduler_end_run", "g4b_scheduler_statistics", "g4b_scheduler_destroy",
                 "g4b_scheduler_last_error", "g4b_poll_oldest"):
        assert hasattr(lib, name)


def test_native_replay_streams_every_event():
    fakes = [FakeTransport(latency_s=0.001), FakeTransport(latency_s=0.001)]
    s = scheduler(fakes, target_photons_per_batch=500, batch_collection_timeout_ms=1)
    submissions = [event(e, (10 + e, 25, 40)) for e in range(200)]
    detections, seconds = s.replay(submissions, producers=3, window=8)
    assert detections == sum(len(expected_detections(sub.emissions)) for sub in submissions)
    assert seconds > 0
    s.end_run()
    assert s.batch_statistics()["event_count"] == 200
    s.close()


def test_detections_out_of_photon_order_are_still_routed_per_event():
    fake = FakeTransport(shuffle_detections=True)
    s = scheduler([fake], target_photons_per_batch=2000, batch_collection_timeout_ms=5)
    futures = {e: s.submit(event(e, (10 + e, 25, 40))) for e in range(30)}
    for e, f in futures.items():
        got = f.result(timeout=10).detections
        want = expected_detections(event(e, (10 + e, 25, 40)).emissions)
        assert sorted(got["photon_id"].tolist()) == sorted(want["photon_id"].tolist())
        assert set(got["event_id"].tolist()) <= {e}
    s.close()


def test_four_transports_rotate_in_order():
    fakes = [FakeTransport(latency_s=0.01) for _ in range(4)]
    s = scheduler(fakes, target_photons_per_batch=100, max_events_per_batch=1, batch_collection_timeout_ms=1)
    futures = [s.submit(event(e)) for e in range(16)]
    for e, f in enumerate(futures):
        assert f.result(timeout=30).event_statistics[0][0] == e
    s.end_run()
    assert all(len(f.batches) >= 2 for f in fakes)
    assert s.batch_statistics()["overlapped_batch_count"] >= 8
    s.close()
