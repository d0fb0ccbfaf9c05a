"""The batched FP32 form's generation pass against generation inside the loop.

A batch of at least 2^24 photons has its photons made by GeneratePhotons into
photon stores, in equal waves (here of at most 2^26 photons: two), overlapped
on streams of their own, and captured into one CUDA graph or launched directly;
`generation_pass = 2` makes them inside the transport loop instead, the form
the parity tests hold byte-exact against the oracle. Every photon comes from
its own genstep and RNG counters either way, so the detections (in the
reference's flattened-photon order) and every counter must be identical.
"""
import ctypes as C

import numpy as np
import pytest

from g4go_b200 import DETECTION_DTYPE, PhotonTransportConfig, TransportHost, _abi, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large_batch():
    batch = scenes.workload("batched", event_count=3300, seed=11)
    assert batch.photon_count > 2 ** 26  # two waves of at most 2^26
    return scenes.crystal_sipm_scene(), batch


def run(scene, batch, pinned=None, **config):
    with TransportHost(PhotonTransportConfig(seed=99, **config)) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch(detections_out=pinned)
        out.detections = out.detections.copy()
        host.relaunch()  # a replay of the same batch (the captured graph, updated in place)
        again = host.complete_oldest_batch(detections_out=pinned)
        again.detections = again.detections.copy()
    return out, again


class PinnedDetections:
    """A page-locked detection buffer (g4b_host_alloc): g4b_complete copies
    the ordered detections straight into it."""

    def __init__(self, rows):
        self.lib = _abi.load()
        self.pointer = C.c_void_p()
        assert self.lib.g4b_host_alloc(rows * DETECTION_DTYPE.itemsize, C.byref(self.pointer)) == 0
        raw = (C.c_ubyte * (rows * DETECTION_DTYPE.itemsize)).from_address(self.pointer.value)
        self.array = np.frombuffer(raw, dtype=DETECTION_DTYPE)

    def free(self):
        self.array = None
        self.lib.g4b_host_free(self.pointer)


@pytest.mark.parametrize("graph,pinned,ordered", [(True, False, True), (False, False, True), (True, True, True),
                                                  (False, True, True), (True, True, False)])
def test_generation_pass_matches_generation_in_the_loop(large_batch, graph, pinned, ordered):
    scene, batch = large_batch
    buffer = PinnedDetections(batch.photon_count // 4) if pinned else None
    try:
        inline, _ = run(scene, batch, generation_pass=2, use_cuda_graph=graph, ordered_detections=ordered)
        passed, replayed = run(scene, batch, pinned=buffer.array if pinned else None, generation_pass=0,
                               wave_photons=1 << 26, use_cuda_graph=graph, ordered_detections=ordered)
    finally:
        if buffer is not None:
            buffer.free()
    assert inline.statistics["detected_count"] > 0
    for out in (passed, replayed):
        assert same_detections(out.detections, inline.detections, ordered)
        assert counters(out.statistics) == counters(inline.statistics)
        assert [(e, counters(s)) for e, s in out.event_statistics] == \
            [(e, counters(s)) for e, s in inline.event_statistics]
        assert out.performance["total_bounce_count"] == inline.performance["total_bounce_count"]
    # two waves: zero, two generations, two transports
    assert passed.performance["kernel_launch_count"] >= 5


def same_detections(a, b, ordered):
    """Byte for byte; without the flattened-photon order, the rows come in the
    order warps appended them, so they are compared sorted by event and photon."""
    if not ordered:
        a = a[np.lexsort((a["photon_id"], a["event_id"]))]
        b = b[np.lexsort((b["photon_id"], b["event_id"]))]
    return a.tobytes() == b.tobytes()


def counters(statistics):
    """Everything but the wall-clock transport time."""
    return {k: v for k, v in statistics.items() if k != "transport_time_ms"}
