"""A photon slice transported on its own gensteps is the same as that slice
of the whole batch (PhotonTransportBatch.photon_slice): each photon keeps its
event and photon ID, so it draws the same random numbers. The benchmark's CPU
sample relies on this to time slices of a large batch without the whole
batch's per-call checks."""
import numpy as np

from g4go_b200 import PhotonTransportConfig, scenes


def test_photon_slice_transports_like_the_whole_batch(oracle):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=60, seed=3)
    config = PhotonTransportConfig(seed=5, precision="fp64")
    total = batch.photon_count
    for begin, end in ((0, 5000), (total // 3, total // 3 + 7001), (total - 4000, total)):
        whole = oracle.transport(scene, batch, config, photon_range=(begin, end))
        part, inside = batch.photon_slice(begin, end)
        assert inside[1] - inside[0] == end - begin
        alone = oracle.transport(scene, part, config, photon_range=inside)
        assert alone.detections.tobytes() == whole.detections.tobytes()
        assert alone.total_bounce_count == whole.total_bounce_count
        counted = {e: s for e, s in whole.event_statistics if s["detected_count"] + s["absorbed_count"]
                   + s["escaped_count"] + s["truncated_count"] + s["invalid_state_count"] > 0}
        mine = {e: s for e, s in alone.event_statistics}
        for event_id, statistics in counted.items():
            for key in ("detected_count", "absorbed_count", "escaped_count", "truncated_count", "max_bounce_count"):
                assert mine[event_id][key] == statistics[key]


def test_photon_slice_rejects_ranges_outside_the_batch():
    import pytest

    batch = scenes.workload("batched", event_count=5, seed=3)
    with pytest.raises(ValueError):
        batch.photon_slice(0, batch.photon_count + 1)
    with pytest.raises(ValueError):
        batch.photon_slice(10, 10)
    part, inside = batch.photon_slice(0, batch.photon_count)
    assert inside == (0, batch.photon_count) and np.array_equal(part.emissions, batch.emissions)
