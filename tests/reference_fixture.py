"""The reference's own transport outputs (tests/golden/transport_reference.npz,
written by tests/golden/make_golden_transport.py from the reference's device
program compiled for the host) and the gates that hold an implementation of
the path to them. Shared by the oracle's CPU test and the engine's GPU test.

The reference computes with the CUDA library's logf/expf/sinf/cosf (the
host's, in the fixture) and OptiX's triangle intersection; this path computes
with its own series and a slab test. The counter RNG, the property and
spectrum tables and the order of every decision are the reference's, so the
histories agree photon by photon and the numbers to a few ulp, carried
through the bounces. Over thousands of bounces (photons the reference lets
leave their volume, some then reflecting totally for the rest of their
history) those ulps eventually flip a decision, so histories of LONG_HISTORY
bounces or more in the reference have looser gates:
  - photon outcome (detected / absorbed / escaped / truncated / invalid):
    at least 0.9999 of the short histories equal, 0.98 of the long ones;
    outcome and bounce count: 0.9995 of the short, 0.97 of the long;
  - detections: the same photons (matched by event and photon ID), the count
    within 0.05 % plus 2 % of the long histories; matched records: the same
    sensor, energy bit for bit, arrival time within 2e-5 relative, direction
    within 1e-5, position within 1e-3 mm for 99 % of them (5e-3 mm on rough
    surfaces, facet sampling) and within 0.1 mm for all;
  - run counters: detected / absorbed / escaped within the same allowance,
    truncated within one plus 2 % of the long histories, the rest equal.
"""
from pathlib import Path

import numpy as np

from g4go_b200 import DETECTION_DTYPE, EMISSION_DTYPE, PhotonTransportBatch, scenes

GOLDEN = Path(__file__).resolve().parent / "golden" / "transport_reference.npz"
SEED = 42
CASES = {
    "one_mev": "crystal_sipm_scene",
    "one_to_ten_mev": "crystal_sipm_scene",
    "uneven": "crystal_sipm_scene",
    "isotropic": "crystal_sipm_scene",
    "rough": "rough_surface_scene",
    "long_histories": "crystal_sipm_scene",
}
STAT_KEYS = ("detected_count", "absorbed_count", "escaped_count", "truncated_count", "max_bounce_count",
             "invalid_state_count", "zero_step_count")


def load():
    return np.load(GOLDEN)


def case(golden, name):
    """(scene, batch) of a fixture case."""
    batch = PhotonTransportBatch(golden[f"{name}_emissions"].view(EMISSION_DTYPE), golden[f"{name}_event_ids"],
                                 golden[f"{name}_event_indices"])
    return getattr(scenes, CASES[name])(), batch


LONG_HISTORY = 200  # bounces


def detection_slots(golden, name, detections):
    """Flattened photon slot of each detection record of a fixture case: the
    genstep holding its event and photon ID, plus the photon's place in it."""
    emissions = golden[f"{name}_emissions"].view(EMISSION_DTYPE)
    offsets = np.concatenate([[0], np.cumsum(emissions["photon_count"].astype(np.int64))])
    slots = np.empty(detections.shape[0], np.int64)
    for i, record in enumerate(detections):
        local = np.int64(record["photon_id"]) - emissions["first_photon_id"].astype(np.int64)
        e = np.nonzero((emissions["event_id"] == record["event_id"]) & (local >= 0)
                       & (local < emissions["photon_count"].astype(np.int64)))[0][0]
        slots[i] = offsets[e] + local[e]
    return slots


def assert_matches_reference(golden, name, fates, detections, statistics):
    """The gates of the module docstring for one case: `fates` is outcome |
    bounces << 3 per photon, `detections` in flattened order, `statistics` the
    run counters (dict)."""
    reference_fates = golden[f"{name}_fate"]
    reference = golden[f"{name}_detections"].view(DETECTION_DTYPE)
    assert fates.shape == reference_fates.shape
    short = (reference_fates >> 3) < LONG_HISTORY
    for part, outcome_bar, history_bar in ((short, 0.9999, 0.9995), (~short, 0.98, 0.97)):
        if part.any():
            outcome = np.mean((fates[part] & 7) == (reference_fates[part] & 7))
            history = np.mean(fates[part] == reference_fates[part])
            assert outcome >= outcome_bar, f"{name}: outcome agreement {outcome} ({part.sum()} histories)"
            assert history >= history_bar, f"{name}: history agreement {history} ({part.sum()} histories)"
    long_allowance = int(np.ceil(0.02 * np.count_nonzero(~short)))
    n = reference.shape[0]
    allowance = max(1, int(5e-4 * n)) + long_allowance
    assert abs(detections.shape[0] - n) <= allowance, f"{name}: {detections.shape[0]} vs {n} detections"
    key = lambda d: (d["event_id"].astype(np.uint64) << np.uint64(32)) | d["photon_id"]  # noqa: E731
    _, mine, theirs = np.intersect1d(key(detections), key(reference), return_indices=True)
    assert mine.size >= n - allowance, f"{name}: only {mine.size} of {n} detections matched"
    a, b = detections[mine], reference[theirs]
    assert np.array_equal(a["sensor_id"], b["sensor_id"])
    assert np.array_equal(a["energy_ev"].view(np.uint32), b["energy_ev"].view(np.uint32))
    assert np.max(np.abs(a["time_ns"] - b["time_ns"]) / b["time_ns"]) < 2e-5
    assert np.max(np.abs(a["direction"] - b["direction"])) < 1e-5
    position_error = np.max(np.abs(a["position_mm"] - b["position_mm"]), axis=1)
    long_detection = ~short[detection_slots(golden, name, b)]
    position_tolerance = 5e-3 if CASES[name] == "rough_surface_scene" else 1e-3
    if (~long_detection).any():
        assert np.quantile(position_error[~long_detection], 0.99) < position_tolerance
    assert np.max(position_error) < 0.1
    counters = golden[f"{name}_statistics"]
    for k, key_name in enumerate(STAT_KEYS):
        if key_name in ("detected_count", "absorbed_count", "escaped_count"):
            assert abs(int(statistics[key_name]) - int(counters[k])) <= allowance, key_name
        elif key_name == "truncated_count":
            assert abs(int(statistics[key_name]) - int(counters[k])) <= 1 + long_allowance, key_name
        elif key_name != "max_bounce_count":
            assert int(statistics[key_name]) == int(counters[k]), key_name
