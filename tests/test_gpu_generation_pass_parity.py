"""The kernels the benchmark times, held byte for byte against the CPU oracle.

A batched FP32 batch of at least 2^24 photons (the benchmark's workload among
them) is not transported by the loop that generates inside itself: its photons
are made by GeneratePhotons into photon stores, wave by wave, and transported
by TransportBatched<float, 0, 1>, which reads the stores; each wave's hits are
ordered by MarkWaveSlots / ScatterWaveDetections. `generation_pass = 3` takes
that path for a batch of any size, and `wave_photons` cuts a small batch into
many waves, so the whole parity matrix runs through the benchmarked kernels at
sizes the oracle finishes in seconds. The last test runs the default
configuration on a real multi-wave batch (more than 2^28 photons, the largest
wave) and compares slices of whole events with the oracle run on the same
photon slots.
"""
import functools

import numpy as np
import pytest

from g4go_b200 import DETECTION_DTYPE, PhotonTransportConfig, TransportHost, scenes
from test_gpu_generation_pass import PinnedDetections
from test_gpu_parity import STAT_KEYS, assert_detections_equal, assert_statistics_equal

pytestmark = pytest.mark.gpu

CASES = {
    "scintillation_1mev": ("plain_cpu", 12),
    "cerenkov_1_10mev": ("plain_fp64", 3),
    "uneven_log_uniform": ("batched", 40),
}
SEED = 20250101


@functools.lru_cache(maxsize=None)
def case_batch(case):
    name, events = CASES[case]
    return scenes.workload(name, event_count=events, seed=7)


@functools.lru_cache(maxsize=None)
def oracle_output(case):
    from oracle import binding

    return binding.transport(scenes.crystal_sipm_scene(), case_batch(case),
                             PhotonTransportConfig(seed=SEED, precision="fp32"))


def run_pass(scene, batch, pinned=None, **config):
    with TransportHost(PhotonTransportConfig(seed=SEED, precision="fp32", generation_pass=3, **config)) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch(detections_out=pinned)
        out.detections = out.detections.copy()
    return out


def waves_of(batch, wave_photons):
    if wave_photons == 0:
        return 1
    wave = (wave_photons + 31) // 32 * 32
    count = -(-batch.photon_count // wave)
    return count


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("wave_photons", [0, 4096])
@pytest.mark.parametrize("graph", [True, False])
def test_generation_pass_matches_oracle_bit_for_bit(oracle, case, wave_photons, graph):
    scene = scenes.crystal_sipm_scene()
    batch = case_batch(case)
    engine = run_pass(scene, batch, wave_photons=wave_photons, use_cuda_graph=graph,
                      enable_performance_diagnostics=True)
    reference = oracle_output(case)
    assert engine.statistics["captured_count"] == batch.photon_count
    assert_detections_equal(engine.detections, reference.detections)
    assert_statistics_equal(engine, reference)
    assert engine.performance["total_bounce_count"] == reference.total_bounce_count
    assert engine.performance["coincident_candidate_trace_count"] == reference.coincident[0]
    assert engine.performance["coincident_candidate_hit_count"] == reference.coincident[1]
    # zero + per wave one generation, one transport and the wave's ordering
    assert engine.performance["kernel_launch_count"] >= 1 + 2 * waves_of(batch, wave_photons)


@pytest.mark.parametrize("case", sorted(CASES))
def test_generation_pass_unordered_and_pinned_match_oracle(oracle, case):
    """Unordered detections (rows in the order warps appended them) hold the
    oracle's records as a set; ordered ones streamed wave by wave into a
    page-locked buffer are the oracle's in its order."""
    scene = scenes.crystal_sipm_scene()
    batch = case_batch(case)
    reference = oracle_output(case)
    unordered = run_pass(scene, batch, wave_photons=4096, ordered_detections=False)
    key = lambda d: d[np.lexsort((d["photon_id"], d["event_id"]))]  # noqa: E731
    assert key(unordered.detections).tobytes() == key(reference.detections).tobytes()
    assert_statistics_equal(unordered, reference)
    buffer = PinnedDetections(max(batch.photon_count // 4, 1024))
    try:
        pinned = run_pass(scene, batch, pinned=buffer.array, wave_photons=4096)
    finally:
        buffer.free()
    assert_detections_equal(pinned.detections, reference.detections)
    assert_statistics_equal(pinned, reference)


def test_generation_pass_fates_match_oracle(oracle):
    """Per-photon fate, bounce count and end time of single isotropic photons,
    generated by GeneratePhotons in waves of 4096."""
    scene = scenes.crystal_sipm_scene()
    batch = scenes.isotropic_photons(20000, photons_per_event=500, seed=3)
    config = dict(seed=99, precision="fp32", record_photon_fates=True)
    with TransportHost(PhotonTransportConfig(generation_pass=3, wave_photons=4096, **config)) as host:
        host.enqueue_emissions(scene, batch)
        engine = host.complete_oldest_batch()
        fates, times = host.photon_fates()
    reference = oracle.transport(scene, batch, PhotonTransportConfig(**config), record_fates=True)
    assert_detections_equal(engine.detections, reference.detections)
    assert_statistics_equal(engine, reference)
    np.testing.assert_array_equal(fates, reference.photon_fate)
    np.testing.assert_array_equal(times.view(np.uint64), reference.photon_time_ns.view(np.uint64))


def test_generation_pass_rough_surfaces_and_rayleigh_match_oracle(oracle):
    from g4go_b200 import Surface, SurfaceBinding, _abi

    scene = scenes.crystal_sipm_scene(scenes.DetectorParameters(crystal_rayleigh_length_mm=30.0))
    wide = (np.array([2.0, 4.0], np.float32), np.array([0.9, 0.9], np.float32))
    ground = scene.add_surface(Surface(
        name="ground_wrapper", type=_abi.SURFACE_DIELECTRIC_METAL, model=_abi.MODEL_UNIFIED,
        finish=_abi.FINISH_GROUND, model_value=0.2, reflectivity=wide,
        specular_lobe=(wide[0], np.array([0.3, 0.3], np.float32)),
        specular_spike=(wide[0], np.array([0.2, 0.2], np.float32)),
        backscatter=(wide[0], np.array([0.1, 0.1], np.float32)),
    ))
    glisur = scene.add_surface(Surface(
        name="glisur_face", type=_abi.SURFACE_DIELECTRIC_DIELECTRIC, model=_abi.MODEL_GLISUR,
        finish=_abi.FINISH_GROUND, model_value=0.7,
    ))
    scene.surface_bindings = [
        SurfaceBinding(scenes.CRYSTAL, scenes.WORLD, ground),
        SurfaceBinding(scenes.WORLD, scenes.CRYSTAL, 1),
        SurfaceBinding(scenes.CRYSTAL, scenes.GREASE, glisur),
    ]
    batch = scenes.workload("plain_cpu", event_count=6, seed=11)
    engine = run_pass(scene, batch, wave_photons=2048)
    reference = oracle.transport(scene, batch, PhotonTransportConfig(seed=SEED, precision="fp32"))
    assert_detections_equal(engine.detections, reference.detections)
    assert_statistics_equal(engine, reference)


def event_slot_starts(batch):
    """Flattened photon slot where each event begins (emissions come grouped by
    event, in event order), plus the total at the end."""
    index = batch.emission_event_indices.astype(np.int64)
    assert np.all(np.diff(index) >= 0)
    per_event = np.bincount(index, weights=batch.emissions["photon_count"].astype(np.float64),
                            minlength=batch.event_ids.shape[0]).astype(np.int64)
    return np.concatenate([[0], np.cumsum(per_event)])


def test_default_configuration_two_wave_batch_matches_oracle_on_event_slices(oracle):
    """The benchmark's own configuration on more than 2^28 photons: two waves
    (or more, where the free device memory sizes them smaller), generation
    pass, captured graph, ordered detections. The oracle transports three
    slices of whole events (the first events, the events around the middle of
    the batch, where two waves meet, the last events) on the same photon slots;
    the engine's detections and counters for those events must be the
    oracle's."""
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=13000, seed=11)
    assert batch.photon_count > 2 ** 28
    config = PhotonTransportConfig(seed=SEED)
    with TransportHost(config) as host:
        host.enqueue_emissions(scene, batch)
        engine = host.complete_oldest_batch()
    assert engine.performance["kernel_launch_count"] >= 5  # zero, 2 x (generation, transport)
    starts = event_slot_starts(batch)
    events = batch.event_ids.shape[0]
    wave = (-(-batch.photon_count // 2) + 31) // 32 * 32
    boundary_event = int(np.searchsorted(starts, wave, side="right") - 1)
    slices = [(0, 8), (boundary_event - 4, boundary_event + 4), (events - 8, events)]
    engine_stats = dict(engine.event_statistics)
    checked = 0
    for first, last in slices:
        ids = batch.event_ids[first:last]
        reference = oracle.transport(scene, batch, config, photon_range=(int(starts[first]), int(starts[last])))
        mask = np.isin(engine.detections["event_id"], ids)
        assert_detections_equal(engine.detections[mask], reference.detections)
        oracle_stats = dict(reference.event_statistics)
        for event_id in ids.tolist():
            for key in STAT_KEYS:
                assert engine_stats[event_id][key] == oracle_stats[event_id][key], (event_id, key)
        checked += reference.detections.shape[0]
    assert checked > 1000
    assert engine.detections.dtype == DETECTION_DTYPE


@pytest.mark.parametrize("graph", [True, False])
def test_generation_pass_hit_region_overflow_reruns_identically(oracle, graph):
    """Each wave writes its hits to its own equal share of the hit buffer; a
    share too small for a wave's hits makes the batch rerun with larger ones
    (the counter RNG makes the rerun identical), whether the detections come
    back into a caller's pinned buffer wave by wave or after the rerun."""
    scene = scenes.crystal_sipm_scene()
    batch = case_batch("uneven_log_uniform")
    reference = oracle_output("uneven_log_uniform")
    small = run_pass(scene, batch, wave_photons=8192, hit_capacity=100, use_cuda_graph=graph)
    assert_detections_equal(small.detections, reference.detections)
    assert_statistics_equal(small, reference)
    buffer = PinnedDetections(batch.photon_count // 4)
    try:
        pinned = run_pass(scene, batch, pinned=buffer.array, wave_photons=8192, hit_capacity=100,
                          use_cuda_graph=graph)
    finally:
        buffer.free()
    assert_detections_equal(pinned.detections, reference.detections)
