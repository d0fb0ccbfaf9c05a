"""Precision and statistical agreement at full size.

- Precision study: 1e7 single photons uniform in the crystal, isotropic,
  380-500 nm, through the FP32 and FP64 engines with the same RNG counters:
  per-photon fate agreement and arrival-time error of the FP32 form against
  the FP64 one.
- Equal accuracy: the batched FP32 engine against the FP64 CPU
  oracle run with an independent seed on the same gensteps: mean detected
  count within 0.5 % and a two-sample KS test on arrival times with p > 0.01.
- Full-size invariants: photon conservation, per-event sums, hit counts,
  replay determinism.
"""
import hashlib

import numpy as np
import pytest
from scipy import stats

from g4go_b200 import PhotonTransportConfig, TransportHost, scenes

pytestmark = pytest.mark.gpu

DETECTED, ABSORBED, ESCAPED, TRUNCATED, INVALID = 1, 2, 3, 4, 5


def run(scene, batch, **config):
    with TransportHost(PhotonTransportConfig(**config)) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch()
        fates = host.photon_fates() if config.get("record_photon_fates") else None
    return out, fates


def test_precision_study_fp32_against_fp64():
    scene = scenes.crystal_sipm_scene()
    batch = scenes.isotropic_photons(10_000_000, photons_per_event=10_000, seed=17)
    out32, (fate32, time32) = run(scene, batch, seed=5, precision="fp32", record_photon_fates=True)
    out64, (fate64, time64) = run(scene, batch, seed=5, precision="fp64", record_photon_fates=True)
    outcome32, outcome64 = fate32 & 7, fate64 & 7
    same_fate = np.mean(outcome32 == outcome64)
    same_history = np.mean(fate32 == fate64)  # same outcome and bounce count
    both_detected = (outcome32 == DETECTED) & (fate32 == fate64)
    time_error = np.abs(time32[both_detected] - time64[both_detected]) / np.maximum(time64[both_detected], 1e-9)
    print(f"\nprecision study: fate agreement {same_fate:.6f}, same history {same_history:.6f}, "
          f"detected {out32.statistics['detected_count']} vs {out64.statistics['detected_count']}, "
          f"arrival-time relative error median {np.median(time_error):.2e} p99 {np.quantile(time_error, 0.99):.2e} "
          f"max {time_error.max():.2e}")
    assert same_fate > 0.995
    assert same_history > 0.99
    assert np.median(time_error) < 1e-6
    d32, d64 = out32.statistics["detected_count"], out64.statistics["detected_count"]
    assert abs(d32 - d64) / d64 < 0.005


def test_batched_fp32_matches_cpu_oracle_statistically(oracle):
    """Mean detected count within 0.5 % and arrival-time KS p > 0.01, independent RNG streams."""
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=600, seed=23)
    assert batch.photon_count > 1e7
    gpu, _ = run(scene, batch, seed=1001, precision="fp32", launch_form="batched")
    cpu = oracle.transport(scene, batch, PhotonTransportConfig(seed=2002, precision="fp64"))
    n_gpu = gpu.statistics["detected_count"]
    n_cpu = cpu.statistics["detected_count"]
    relative = abs(n_gpu - n_cpu) / n_cpu
    ks = stats.ks_2samp(gpu.detections["time_ns"], cpu.detections["time_ns"])
    # per-event mean detected count
    per_event_gpu = np.array([s["detected_count"] for _, s in gpu.event_statistics], dtype=np.float64)
    per_event_cpu = np.array([s["detected_count"] for _, s in cpu.event_statistics], dtype=np.float64)
    print(f"\nGPU FP32 {n_gpu} vs CPU FP64 {n_cpu} detected ({relative:.2e}); KS p = {ks.pvalue:.3f}; "
          f"per-event means {per_event_gpu.mean():.2f} vs {per_event_cpu.mean():.2f}")
    assert relative < 0.005
    assert ks.pvalue > 0.01
    assert abs(per_event_gpu.mean() - per_event_cpu.mean()) / per_event_cpu.mean() < 0.005


def test_plain_fp64_and_batched_fp32_have_equal_accuracy():
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=400, seed=29)
    fast, _ = run(scene, batch, seed=77, precision="fp32", launch_form="batched")
    plain, _ = run(scene, batch, seed=78, precision="fp64", launch_form="plain")
    relative = abs(fast.statistics["detected_count"] - plain.statistics["detected_count"]) / plain.statistics[
        "detected_count"]
    ks = stats.ks_2samp(fast.detections["time_ns"], plain.detections["time_ns"])
    print(f"\nbatched FP32 vs plain FP64: detected {relative:.2e} apart, KS p = {ks.pvalue:.3f}")
    assert relative < 0.005
    assert ks.pvalue > 0.01


def test_full_size_invariants_and_determinism():
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=20000, seed=31)
    with TransportHost(PhotonTransportConfig(seed=9)) as host:
        host.enqueue_emissions(scene, batch)
        first = host.complete_oldest_batch()
        host.relaunch()
        second = host.complete_oldest_batch()
    s = first.statistics
    assert s["captured_count"] == batch.photon_count > 3e8
    assert (s["detected_count"] + s["absorbed_count"] + s["escaped_count"] + s["truncated_count"]
            + s["invalid_state_count"]) == s["captured_count"]
    assert first.detections.shape[0] == s["detected_count"]
    for key in ("detected_count", "absorbed_count", "escaped_count", "truncated_count", "invalid_state_count",
                "zero_step_count"):
        assert sum(es[key] for _, es in first.event_statistics) == s[key], key
    assert max(es["max_bounce_count"] for _, es in first.event_statistics) == s["max_bounce_count"]
    digest = lambda out: hashlib.sha256(out.detections.tobytes()).hexdigest()  # noqa: E731
    assert digest(first) == digest(second)
    # detections in the reference's order: events ascending, photon IDs ascending within an event
    d = first.detections
    order = np.lexsort((d["photon_id"], d["event_id"]))
    assert np.array_equal(order, np.arange(d.shape[0]))
