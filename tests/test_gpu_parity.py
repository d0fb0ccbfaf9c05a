"""Parity of the CUDA engine with the CPU oracle, through the C ABI.

Both sides run the same gensteps under the same seed. With the shared
floating-point discipline (no contraction, the engine's own log/exp/sincos)
the detections must be identical byte for byte, in the reference's
flattened-photon order, and every per-event counter must match.
"""
import numpy as np
import pytest

from g4go_b200 import DETECTION_DTYPE, PhotonTransportConfig, TransportHost, scenes

pytestmark = pytest.mark.gpu

STAT_KEYS = ("captured_count", "detected_count", "absorbed_count", "escaped_count", "truncated_count",
             "max_bounce_count", "invalid_state_count", "zero_step_count")


def run_engine(scene, batch, **config):
    with TransportHost(PhotonTransportConfig(**config)) as host:
        host.enqueue_emissions(scene, batch)
        return host.complete_oldest_batch()


def assert_detections_equal(engine, reference):
    assert engine.dtype == DETECTION_DTYPE and reference.dtype == DETECTION_DTYPE
    assert engine.shape == reference.shape, f"{engine.shape[0]} engine hits vs {reference.shape[0]} oracle hits"
    a = engine.view(np.uint32).reshape(-1, 12)
    b = reference.view(np.uint32).reshape(-1, 12)
    rows = np.nonzero((a != b).any(axis=1))[0]
    assert rows.size == 0, (
        f"{rows.size} of {a.shape[0]} detections differ; first at {rows[0]}: "
        f"engine {engine[rows[0]]} oracle {reference[rows[0]]}"
    )


def assert_statistics_equal(engine_output, oracle_output):
    assert len(engine_output.event_statistics) == len(oracle_output.event_statistics)
    for (eid, es), (oid, os_) in zip(engine_output.event_statistics, oracle_output.event_statistics):
        assert eid == oid
        for key in STAT_KEYS:
            assert es[key] == os_[key], f"event {eid} {key}: engine {es[key]} oracle {os_[key]}"
    for key in STAT_KEYS:
        assert engine_output.statistics[key] == oracle_output.statistics[key], key


CASES = {
    "scintillation_1mev": ("plain_cpu", 12),
    "cerenkov_1_10mev": ("plain_fp64", 3),
    "uneven_log_uniform": ("batched", 40),
}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("form", ["batched", "plain"])
def test_engine_matches_oracle_bit_for_bit(oracle, case, precision, form):
    name, events = CASES[case]
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload(name, event_count=events, seed=7)
    config = dict(seed=20250101, precision=precision, launch_form=form)
    engine = run_engine(scene, batch, enable_performance_diagnostics=True, **config)
    reference = oracle.transport(scene, batch, PhotonTransportConfig(**config))
    assert engine.statistics["captured_count"] == batch.photon_count
    assert_detections_equal(engine.detections, reference.detections)
    assert_statistics_equal(engine, reference)
    assert engine.performance["total_bounce_count"] == reference.total_bounce_count
    assert engine.performance["coincident_candidate_trace_count"] == reference.coincident[0]
    assert engine.performance["coincident_candidate_hit_count"] == reference.coincident[1]
    # without diagnostics the kernel leaves the coincidence counters out and
    # transports identically
    quiet = run_engine(scene, batch, **config)
    assert quiet.detections.tobytes() == engine.detections.tobytes()
    assert quiet.performance["total_bounce_count"] == engine.performance["total_bounce_count"]
    assert quiet.performance["coincident_candidate_trace_count"] == 0


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_isotropic_single_photons_match_oracle_with_fates(oracle, precision):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.isotropic_photons(20000, photons_per_event=500, seed=3)
    config = dict(seed=99, precision=precision, record_photon_fates=True)
    with TransportHost(PhotonTransportConfig(**config)) as host:
        host.enqueue_emissions(scene, batch)
        engine = host.complete_oldest_batch()
        fates, times = host.photon_fates()
    reference = oracle.transport(scene, batch, PhotonTransportConfig(**config), record_fates=True)
    assert_detections_equal(engine.detections, reference.detections)
    assert_statistics_equal(engine, reference)
    np.testing.assert_array_equal(fates, reference.photon_fate)
    np.testing.assert_array_equal(times.view(np.uint64), reference.photon_time_ns.view(np.uint64))


def test_rayleigh_and_rough_surfaces_match_oracle(oracle):
    """Rayleigh scattering, a ground unified wrapper and a glisur grease face:
    paths the baseline scene does not reach, still bit-exact with the oracle."""
    from g4go_b200 import Surface, SurfaceBinding
    from g4go_b200 import _abi

    params = scenes.DetectorParameters(crystal_rayleigh_length_mm=30.0)
    scene = scenes.crystal_sipm_scene(params)
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
    for precision in ("fp32", "fp64"):
        config = dict(seed=5, precision=precision)
        engine = run_engine(scene, batch, **config)
        reference = oracle.transport(scene, batch, PhotonTransportConfig(**config))
        assert_detections_equal(engine.detections, reference.detections)
        assert_statistics_equal(engine, reference)
