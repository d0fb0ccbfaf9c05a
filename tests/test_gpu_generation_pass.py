"""The batched FP32 form's generation pass against generation inside the loop.

A batch of at least 2^24 photons has its photons made by GeneratePhotons into
photon stores, in equal waves of at most 2^26 photons (two here), overlapped
on a second stream, and captured into one CUDA graph or launched directly;
`generation_pass = 2` makes them inside the transport loop instead, the form
the parity tests hold byte-exact against the oracle. Every photon comes from
its own genstep and RNG counters either way, so the detections (in the
reference's flattened-photon order) and every counter must be identical.
"""
import pytest

from g4go_b200 import PhotonTransportConfig, TransportHost, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large_batch():
    batch = scenes.workload("batched", event_count=3300, seed=11)
    assert batch.photon_count > 2 ** 26  # two waves
    return scenes.crystal_sipm_scene(), batch


def run(scene, batch, **config):
    with TransportHost(PhotonTransportConfig(seed=99, **config)) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch()
        host.relaunch()  # a replay of the same batch (the captured graph, updated in place)
        again = host.complete_oldest_batch()
    return out, again


@pytest.mark.parametrize("graph", [True, False])
def test_generation_pass_matches_generation_in_the_loop(large_batch, graph):
    scene, batch = large_batch
    inline, _ = run(scene, batch, generation_pass=2, use_cuda_graph=graph)
    passed, replayed = run(scene, batch, generation_pass=0, use_cuda_graph=graph)
    assert inline.statistics["detected_count"] > 0
    for out in (passed, replayed):
        assert out.detections.tobytes() == inline.detections.tobytes()
        assert counters(out.statistics) == counters(inline.statistics)
        assert [(e, counters(s)) for e, s in out.event_statistics] == \
            [(e, counters(s)) for e, s in inline.event_statistics]
        assert out.performance["total_bounce_count"] == inline.performance["total_bounce_count"]
    # two waves: zero, two generations, two transports
    assert passed.performance["kernel_launch_count"] >= 5


def counters(statistics):
    """Everything but the wall-clock transport time."""
    return {k: v for k, v in statistics.items() if k != "transport_time_ms"}
