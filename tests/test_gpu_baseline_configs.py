"""The plain-method workloads at their stated sizes against the CPU oracle.

- 1,000 events of 1 MeV electrons at the face centre (about 1e6 photons): the
  plain FP64 form, one event per launch, byte for byte against the FP64
  oracle; the batched FP32 form through the generation pass byte for byte
  against the FP32 oracle.
- 5,000 events of 1-10 MeV electrons with Cerenkov light (about 2.8e8
  photons): the plain FP64 GPU form byte for byte against the FP64 oracle on
  all host threads, and the batched FP32 form (independent seed) against that
  same CPU run with the reference's own regression gates
  (test/TestOpticalTransport.cxx:319-333: per-event detected count mean within
  5 % and RMS within 10 %, arrival-time mean within 1 % and RMS within 5 %,
  arrival-time shape test p >= 0.01) plus the tighter equal-accuracy bar of
  this path (mean detected count within 0.5 %, two-sample KS p > 0.01).
"""
import numpy as np
import pytest
from scipy import stats

from g4go_b200 import PhotonTransportConfig, TransportHost, scenes
from test_gpu_parity import assert_detections_equal, assert_statistics_equal

pytestmark = pytest.mark.gpu


def run(scene, batch, **config):
    with TransportHost(PhotonTransportConfig(**config)) as host:
        host.enqueue_emissions(scene, batch)
        return host.complete_oldest_batch()


def test_one_mev_workload_at_full_size_matches_oracle(oracle):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("plain_cpu", seed=1)
    assert batch.event_ids.shape[0] == 1000 and 0.8e6 < batch.photon_count < 1.3e6
    plain = run(scene, batch, seed=1, precision="fp64", launch_form="plain")
    reference64 = oracle.transport(scene, batch, PhotonTransportConfig(seed=1, precision="fp64"))
    assert_detections_equal(plain.detections, reference64.detections)
    assert_statistics_equal(plain, reference64)
    batched = run(scene, batch, seed=1, precision="fp32", generation_pass=3)
    reference32 = oracle.transport(scene, batch, PhotonTransportConfig(seed=1, precision="fp32"))
    assert_detections_equal(batched.detections, reference32.detections)
    assert_statistics_equal(batched, reference32)


def moments(values):
    values = np.asarray(values, dtype=np.float64)
    return values.mean(), values.std()


def relative(a, b):
    return abs(a - b) / max(abs(b), np.finfo(np.float64).eps)


def test_one_to_ten_mev_workload_at_full_size(oracle):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("plain_fp64", seed=2)
    assert batch.event_ids.shape[0] == 5000 and batch.photon_count > 2e8
    cpu = oracle.transport(scene, batch, PhotonTransportConfig(seed=11, precision="fp64"))
    plain = run(scene, batch, seed=11, precision="fp64", launch_form="plain")
    assert_detections_equal(plain.detections, cpu.detections)
    assert_statistics_equal(plain, cpu)
    del plain

    fast = run(scene, batch, seed=12, precision="fp32", launch_form="batched")
    n_fast, n_cpu = fast.statistics["detected_count"], cpu.statistics["detected_count"]
    per_event_fast = [s["detected_count"] for _, s in fast.event_statistics]
    per_event_cpu = [s["detected_count"] for _, s in cpu.event_statistics]
    mean_fast, rms_fast = moments(per_event_fast)
    mean_cpu, rms_cpu = moments(per_event_cpu)
    tof_mean_fast, tof_rms_fast = moments(fast.detections["time_ns"])
    tof_mean_cpu, tof_rms_cpu = moments(cpu.detections["time_ns"])
    ks = stats.ks_2samp(fast.detections["time_ns"], cpu.detections["time_ns"])
    print(f"\n5000 events, {batch.photon_count} photons: detected {n_fast} (batched FP32) vs {n_cpu} (CPU FP64), "
          f"{relative(n_fast, n_cpu):.2e} apart; per event mean {mean_fast:.1f}/{mean_cpu:.1f} "
          f"rms {rms_fast:.1f}/{rms_cpu:.1f}; ToF mean {tof_mean_fast:.4f}/{tof_mean_cpu:.4f} ns "
          f"rms {tof_rms_fast:.4f}/{tof_rms_cpu:.4f} ns; KS p {ks.pvalue:.3f}")
    # the reference's regression gates
    assert relative(mean_fast, mean_cpu) <= 0.05
    assert relative(rms_fast, rms_cpu) <= 0.10
    assert relative(tof_mean_fast, tof_mean_cpu) <= 0.01
    assert relative(tof_rms_fast, tof_rms_cpu) <= 0.05
    assert ks.pvalue >= 0.01
    # this path's equal-accuracy bar
    assert relative(n_fast, n_cpu) < 0.005
