"""Behaviour of the drop-in boundary on the GPU: the reference's error cases
(src/optical/optix/OptiXTransportHost.cpp:511-605,779-807), empty and
zero-photon batches, replay determinism, hit-buffer overflow and ordering."""
import numpy as np
import pytest

from g4go_b200 import (
    INVALID_ID,
    LogicError,
    PhotonTransportBatch,
    PhotonTransportConfig,
    TransportHost,
    scenes,
)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene():
    return scenes.crystal_sipm_scene()


@pytest.fixture(scope="module")
def batch():
    return scenes.workload("batched", event_count=30, seed=13)


def test_queue_discipline(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=1)) as host:
        with pytest.raises(LogicError):  # "transport queue is empty" (:780-782)
            host.complete_oldest_batch()
        with pytest.raises(LogicError):  # relaunch without a staged batch
            host.relaunch()
        host.enqueue_emissions(scene, batch)
        with pytest.raises(LogicError):  # "transport queue is full" (:523-525)
            host.enqueue_emissions(scene, batch)
        with pytest.raises(LogicError):  # scene rebuild with a pending batch (:514-516)
            host.prepare_scene(scenes.crystal_sipm_scene())
        out = host.complete_oldest_batch()
        assert out.statistics["captured_count"] == batch.photon_count


def test_enqueue_before_scene_is_a_logic_error(batch):
    from g4go_b200 import _abi
    import ctypes as C

    with TransportHost(PhotonTransportConfig(seed=1)) as host:
        status = host._lib.g4b_enqueue(host._handle, batch.emissions.ctypes.data_as(C.c_void_p),
                                       batch.emissions.shape[0], _abi.as_ptr(batch.event_ids, C.c_uint32),
                                       batch.event_ids.shape[0], _abi.as_ptr(batch.emission_event_indices, C.c_uint32))
        assert status == _abi.ERR_NO_SCENE


def _mutated(batch, **changes):
    emissions = batch.emissions.copy()
    event_ids = batch.event_ids.copy()
    indices = batch.emission_event_indices.copy()
    if "event_ids" in changes:
        event_ids = changes["event_ids"]
    if "indices" in changes:
        indices = changes["indices"]
    for field, value in changes.get("emission", {}).items():
        emissions[field][0] = value
    return PhotonTransportBatch(emissions, event_ids, indices)


def test_invalid_batches_raise_value_error(scene, batch):
    bad = [
        _mutated(batch, event_ids=np.concatenate([batch.event_ids[:1], batch.event_ids[:-1]])),  # duplicate IDs
        _mutated(batch, indices=np.full_like(batch.emission_event_indices, batch.event_ids.shape[0])),  # bad index
        _mutated(batch, emission={"event_id": 987654}),  # index does not match event ID
        _mutated(batch, emission={"volume_id": 77}),  # unknown volume
        _mutated(batch, emission={"material_id": 9}),  # unknown material
    ]
    with TransportHost(PhotonTransportConfig(seed=1)) as host:
        for b in bad:
            with pytest.raises(ValueError):
                host.enqueue_emissions(scene, b)
        host.enqueue_emissions(scene, batch)  # the handle still works
        host.complete_oldest_batch()


def test_invalid_scenes_raise(scene):
    with TransportHost(PhotonTransportConfig(seed=1)) as host:
        broken = scenes.crystal_sipm_scene()
        broken.volumes[2].parent_volume_id = 55
        with pytest.raises(ValueError):
            host.prepare_scene(broken)
        duplicate = scenes.crystal_sipm_scene()
        duplicate.volumes[2].volume_id = duplicate.volumes[1].volume_id
        with pytest.raises(ValueError):
            host.prepare_scene(duplicate)
        no_world = scenes.crystal_sipm_scene()
        no_world.world_volume_id = INVALID_ID
        with pytest.raises(ValueError):
            host.prepare_scene(no_world)
        unsorted = scenes.crystal_sipm_scene()
        e, v = unsorted.materials[1].abs_length_mm
        unsorted.materials[1].abs_length_mm = (e[::-1].copy(), v)
        with pytest.raises(ValueError):
            host.prepare_scene(unsorted)


def test_empty_and_zero_photon_batches(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=1)) as host:
        empty = PhotonTransportBatch(batch.emissions[:0], batch.event_ids[:3], batch.emission_event_indices[:0])
        host.enqueue_emissions(scene, empty)
        out = host.complete_oldest_batch()
        assert out.detections.shape[0] == 0
        assert [eid for eid, _ in out.event_statistics] == list(batch.event_ids[:3])
        assert all(s["valid_fields"] == 0 for _, s in out.event_statistics)  # :597-602
        zero = batch.emissions[:4].copy()
        zero["photon_count"] = 0
        zb = PhotonTransportBatch(zero, batch.event_ids, batch.emission_event_indices[:4])
        host.enqueue_emissions(scene, zb)
        out = host.complete_oldest_batch()
        terminal = sum(1 << f for f in (2, 3, 4, 5, 6, 7, 8))
        for _, s in out.event_statistics:  # :612-626
            assert s["valid_fields"] & terminal == terminal


def test_relaunch_and_replay_are_deterministic(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=3)) as host:
        host.enqueue_emissions(scene, batch)
        first = host.complete_oldest_batch()
        host.relaunch()
        second = host.complete_oldest_batch()
        host.enqueue_emissions(scene, batch)
        third = host.complete_oldest_batch()
    assert first.detections.tobytes() == second.detections.tobytes() == third.detections.tobytes()
    assert first.event_statistics == second.event_statistics


def test_hit_buffer_overflow_reruns_identically(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=3)) as host:
        host.enqueue_emissions(scene, batch)
        full = host.complete_oldest_batch()
    with TransportHost(PhotonTransportConfig(seed=3, hit_capacity=17)) as host:
        host.enqueue_emissions(scene, batch)
        small = host.complete_oldest_batch()
    assert full.detections.shape[0] > 17
    assert small.detections.tobytes() == full.detections.tobytes()


def test_unordered_detections_are_the_same_set(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=3)) as host:
        host.enqueue_emissions(scene, batch)
        ordered = host.complete_oldest_batch().detections
    with TransportHost(PhotonTransportConfig(seed=3, ordered_detections=False)) as host:
        host.enqueue_emissions(scene, batch)
        unordered = host.complete_oldest_batch().detections
    key = lambda d: np.lexsort((d["photon_id"], d["event_id"]))  # noqa: E731
    assert ordered[key(ordered)].tobytes() == unordered[key(unordered)].tobytes()
    # the reference's order: events in batch order, photons by flattened index
    assert np.all(np.diff(ordered["event_id"].astype(np.int64)) >= 0)


def test_counts_only_completion_and_statistics_invariants(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=9)) as host:
        host.enqueue_emissions(scene, batch)
        counts = host.complete_oldest_batch(counts_only=True)
        host.relaunch()
        full = host.complete_oldest_batch()
    assert counts.detections.shape[0] == 0
    assert counts.statistics == {**full.statistics, "transport_time_ms": counts.statistics["transport_time_ms"]}
    s = full.statistics
    terminal = (s["detected_count"] + s["absorbed_count"] + s["escaped_count"] + s["truncated_count"]
                + s["invalid_state_count"])
    assert terminal == s["captured_count"] == batch.photon_count
    per_event = np.bincount(full.detections["event_id"] - batch.event_ids.min(),
                            minlength=batch.event_ids.shape[0])
    for i, (event_id, es) in enumerate(full.event_statistics):
        assert es["detected_count"] == per_event[event_id - batch.event_ids.min()]


def test_plain_form_groups_interleaved_events(oracle, scene, batch):
    """Emissions of different events interleaved in the batch: the plain form
    groups them per launch and still returns the reference's order."""
    order = np.argsort(np.arange(batch.emissions.shape[0]) % 3, kind="stable")
    shuffled = PhotonTransportBatch(batch.emissions[order], batch.event_ids, batch.emission_event_indices[order])
    config = PhotonTransportConfig(seed=4, launch_form="plain", precision="fp32")
    with TransportHost(config) as host:
        host.enqueue_emissions(scene, shuffled)
        out = host.complete_oldest_batch()
    reference = oracle.transport(scene, shuffled, config)
    assert out.detections.tobytes() == reference.detections.tobytes()


def test_autotune_picks_a_valid_shape(scene, batch):
    with TransportHost(PhotonTransportConfig(seed=2)) as host:
        host.enqueue_emissions(scene, batch)
        before = host.complete_oldest_batch()
        result = host.autotune(block_sizes=[128, 256], chunk_sizes=[64, 512], repeats=1)
        assert result["block_size"] in (128, 256) and result["chunk_photons"] in (64, 512)
        assert result["candidates_tried"] >= 4 and result["best_ms"] <= result["worst_ms"]
        host.relaunch()
        after = host.complete_oldest_batch()
    assert before.detections.tobytes() == after.detections.tobytes()


def _events_slice(batch, first, last):
    """The batch's events [first, last) with their gensteps (contiguous per event)."""
    keep = (batch.emission_event_indices >= first) & (batch.emission_event_indices < last)
    return PhotonTransportBatch(batch.emissions[keep], batch.event_ids[first:last],
                                batch.emission_event_indices[keep] - first)


def _without_time(statistics):
    return {k: v for k, v in statistics.items() if k != "transport_time_ms"}


def test_large_batches_are_staged_in_parallel_parts(scene):
    """g4b_enqueue stages a batch of 2^17 gensteps or more with several host
    threads: errors still name the first bad genstep in batch order, and the
    staged batch (offsets summed across the parts) gives exactly the results of
    its events enqueued in parts small enough for one thread."""
    batch = scenes.workload("batched", event_count=7300, seed=21)
    count = batch.emissions.shape[0]
    assert count >= 2 ** 18  # four parts where the host has the threads
    assert np.all(np.diff(batch.emission_event_indices.astype(np.int64)) >= 0)
    early, late = count // 9, count - 3

    def planted(fields):
        emissions = batch.emissions.copy()
        for (field, row), value in fields.items():
            emissions[field][row] = value
        return PhotonTransportBatch(emissions, batch.event_ids, batch.emission_event_indices)

    with TransportHost(PhotonTransportConfig(seed=5)) as host:
        with pytest.raises(ValueError, match="material"):
            host.enqueue_emissions(scene, planted({("material_id", early): 9, ("volume_id", late): 77}))
        with pytest.raises(ValueError, match="volume"):
            host.enqueue_emissions(scene, planted({("volume_id", early): 77, ("material_id", late): 9}))
        with pytest.raises(ValueError, match="volume"):
            host.enqueue_emissions(scene, planted({("volume_id", late): 77}))
        with pytest.raises(ValueError, match="does not match"):
            host.enqueue_emissions(scene, planted({("event_id", late): 987654}))
        host.enqueue_emissions(scene, batch)
        whole = host.complete_oldest_batch()
        whole.detections = whole.detections.copy()
        parts = []
        events = batch.event_ids.shape[0]
        for first, last in ((0, events // 3), (events // 3, 2 * events // 3), (2 * events // 3, events)):
            part = _events_slice(batch, first, last)
            assert part.emissions.shape[0] < 2 ** 17  # one staging thread
            host.enqueue_emissions(scene, part)
            out = host.complete_oldest_batch()
            parts.append((out.detections.copy(), out.event_statistics))
    assert whole.statistics["detected_count"] > 0
    assert whole.detections.tobytes() == np.concatenate([d for d, _ in parts]).tobytes()
    assert [(e, _without_time(s)) for e, s in whole.event_statistics] == \
        [(e, _without_time(s)) for _, stats in parts for e, s in stats]
