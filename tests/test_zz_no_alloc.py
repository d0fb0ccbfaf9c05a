"""g4b_order_detections_static, the ordering entry point that allocates no
device memory, against the ordered completion of g4b_complete (the order of
the reference's flagged compaction, src/optical/optix/OptiXHitCompaction.cu:23-30).

The file is collected last so that the entry point also runs after every
other test in the session has used the device."""
import ctypes as C

import numpy as np
import pytest

from g4go_b200 import PhotonTransportConfig, TransportHost, _abi, scenes
from g4go_b200.transport import raise_for_status

pytestmark = pytest.mark.gpu

MAX_SLOTS = 1 << 24


def _order_static(lib, unordered, slots, count, slot_limit, ordered, stream=0):
    status = lib.g4b_order_detections_static(unordered, slots, count, slot_limit, ordered, stream)
    return status, lib.g4b_last_error(None).decode()


def _slot_keys(batch, detections):
    """Flattened photon index of each detection: the photon offset of its
    emission in enqueue order plus its index within that emission."""
    emissions = batch.emissions
    counts = emissions["photon_count"].astype(np.int64)
    offsets = np.concatenate(([0], np.cumsum(counts)[:-1]))
    order = np.lexsort((emissions["first_photon_id"], emissions["event_id"]))
    starts = (emissions["event_id"][order].astype(np.int64) << 32) | emissions["first_photon_id"][order]
    query = (detections["event_id"].astype(np.int64) << 32) | detections["photon_id"]
    emission = order[np.searchsorted(starts, query, side="right") - 1]
    local = detections["photon_id"].astype(np.int64) - emissions["first_photon_id"][emission]
    assert np.all(emissions["event_id"][emission] == detections["event_id"])
    assert np.all((local >= 0) & (local < counts[emission]))
    return (offsets[emission] + local).astype(np.uint32)


@pytest.fixture(scope="module")
def transported():
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=30, seed=21)
    with TransportHost(PhotonTransportConfig(seed=5)) as host:
        host.enqueue_emissions(scene, batch)
        ordered = host.complete_oldest_batch().detections
    with TransportHost(PhotonTransportConfig(seed=5, ordered_detections=False)) as host:
        host.enqueue_emissions(scene, batch)
        unordered = host.complete_oldest_batch().detections
    return batch, ordered, unordered


def test_matches_the_ordered_completion_on_two_calls_in_a_row(engine_lib, transported):
    torch = pytest.importorskip("torch")
    batch, ordered, unordered = transported
    count = unordered.shape[0]
    assert count > 1000
    # the unordered completion really is out of order, so the check has teeth
    assert unordered.tobytes() != ordered.tobytes()
    keys = _slot_keys(batch, unordered)
    device_records = torch.from_numpy(unordered.view(np.uint8).reshape(-1).copy()).cuda()
    device_keys = torch.from_numpy(keys.view(np.int32)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        device_out = torch.zeros_like(device_records)
        status, message = _order_static(engine_lib, device_records.data_ptr(), device_keys.data_ptr(), count,
                                        batch.photon_count, device_out.data_ptr(), stream)
        raise_for_status(status, message)
        result = device_out.cpu().numpy().view(_abi.DETECTION_DTYPE)
        assert result.tobytes() == ordered.tobytes()


def test_full_scratch_size_against_a_host_sort(engine_lib):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(8)
    count = 1_500_000
    keys = rng.choice(MAX_SLOTS, size=count, replace=False).astype(np.uint32)
    keys[0] = MAX_SLOTS - 1  # the last slot of the scratch bitmap
    records = rng.integers(0, 256, size=(count, 48), dtype=np.uint8)
    expected = records[np.argsort(keys, kind="stable")]
    device_records = torch.from_numpy(records.reshape(-1)).cuda()
    device_keys = torch.from_numpy(keys.view(np.int32)).cuda()
    for _ in range(2):
        device_out = torch.zeros_like(device_records)
        status, message = _order_static(engine_lib, device_records.data_ptr(), device_keys.data_ptr(), count,
                                        MAX_SLOTS, device_out.data_ptr())
        raise_for_status(status, message)
        assert np.array_equal(device_out.cpu().numpy().reshape(count, 48), expected)


def test_rejects_what_does_not_fit_the_scratch(engine_lib):
    torch = pytest.importorskip("torch")
    records = torch.zeros(48 * 4, dtype=torch.uint8, device="cuda")
    out = torch.zeros_like(records)
    keys = torch.tensor([3, 1, 0, 2], dtype=torch.int32, device="cuda")
    status, message = _order_static(engine_lib, records.data_ptr(), keys.data_ptr(), 4, MAX_SLOTS + 1,
                                    out.data_ptr())
    assert status == _abi.ERR_OVERFLOW and "G4B_ORDER_STATIC_MAX_SLOTS" in message
    status, _ = _order_static(engine_lib, records.data_ptr(), keys.data_ptr(), 4, 3, out.data_ptr())
    assert status == _abi.ERR_INVALID_ARGUMENT
    status, _ = _order_static(engine_lib, records.data_ptr() + 4, keys.data_ptr(), 3, 4, out.data_ptr())
    assert status == _abi.ERR_INVALID_ARGUMENT
    status, _ = _order_static(engine_lib, records.data_ptr(), keys.data_ptr(), 4, 4, records.data_ptr() + 48)
    assert status == _abi.ERR_INVALID_ARGUMENT
    assert _order_static(engine_lib, None, None, 0, 4, None)[0] == _abi.OK


def test_repeated_and_out_of_range_keys_are_errors_and_leave_the_scratch_clean(engine_lib):
    torch = pytest.importorskip("torch")
    rows = torch.arange(4 * 48, dtype=torch.int32, device="cuda").to(torch.uint8)
    out = torch.zeros_like(rows)
    for bad in ([3, 1, 1, 2], [3, 1, 9, 2]):
        keys = torch.tensor(bad, dtype=torch.int32, device="cuda")
        status, message = _order_static(engine_lib, rows.data_ptr(), keys.data_ptr(), 4, 8, out.data_ptr())
        assert status == _abi.ERR_INVALID_ARGUMENT and "repeated" in message
    keys = torch.tensor([3, 1, 0, 2], dtype=torch.int32, device="cuda")
    status, message = _order_static(engine_lib, rows.data_ptr(), keys.data_ptr(), 4, 8, out.data_ptr())
    raise_for_status(status, message)
    expected = rows.view(4, 48)[torch.tensor([2, 1, 3, 0], device="cuda")].reshape(-1)
    assert torch.equal(out, expected)
