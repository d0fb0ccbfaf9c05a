"""The CPU oracle against the reference's own device program.

The fixture (tests/golden/transport_reference.npz) holds outputs of
src/optical/optix/OptiXTransportDevice.cu compiled unmodified for the host
(oracle/_ref/libref_transport.so; recipe oracle/Makefile, generator
tests/golden/make_golden_transport.py). This pins the oracle's restatement
of the counter RNG, the property and spectrum sampling, photon generation
and the bounce loop to the reference's code:
  - Uniform, SampleProperty, SampleSpectrum and the spectrum CDF: bit for bit;
  - GeneratePhoton: positions and energies bit for bit, directions and
    polarisations within 1e-6 (sin/cos), times within 1e-6 relative (log);
  - the bounce loop: the gates of tests/reference_fixture.py.
Where the reference tree was there to build oracle/_ref, the live reference is
also run on inputs the fixture does not hold.
"""
import numpy as np
import pytest

import reference_fixture as rf
from g4go_b200 import EMISSION_DTYPE, PhotonTransportBatch, PhotonTransportConfig, scenes


@pytest.fixture(scope="module")
def golden():
    return rf.load()


def test_counter_rng_is_the_reference_bit_for_bit(oracle, golden):
    lib = oracle.load()
    for s, seed in enumerate(golden["uniform_seeds"]):
        mine = np.array([lib.oracle_uniform_f(int(seed), int(k), int(b), int(p), int(d))
                         for k, b, p, d in zip(golden["uniform_keys"], golden["uniform_bounce"],
                                               golden["uniform_process"], golden["uniform_draw"])], np.float32)
        assert np.array_equal(mine.view(np.uint32), golden["uniform"][s].view(np.uint32)), f"seed {seed}"


def test_property_and_spectrum_sampling_are_the_reference_bit_for_bit(oracle, golden):
    import ctypes as C

    lib = oracle.load()
    f = C.POINTER(C.c_float)
    energy, values = golden["property_energy"], golden["property_values"]
    mine = np.array([lib.oracle_sample_property_f(energy.ctypes.data_as(f), values.ctypes.data_as(f), energy.size,
                                                  float(x), -1.0) for x in golden["property_queries"]], np.float32)
    assert np.array_equal(mine.view(np.uint32), golden["property"].view(np.uint32))
    spectrum_energy = np.ascontiguousarray(golden["spectrum_energy"])
    spectrum_values = np.ascontiguousarray(golden["spectrum_values"])
    cdf = np.empty_like(spectrum_values)
    assert lib.oracle_spectrum_cdf(spectrum_energy.ctypes.data_as(f), spectrum_values.ctypes.data_as(f),
                                   spectrum_energy.size, cdf.ctypes.data_as(f)) == spectrum_energy.size
    assert np.array_equal(cdf.view(np.uint32), golden["spectrum_cdf"].view(np.uint32))
    mine = np.array([lib.oracle_sample_spectrum_f(spectrum_energy.ctypes.data_as(f), spectrum_values.ctypes.data_as(f),
                                                  spectrum_energy.size, float(u)) for u in golden["spectrum_queries"]],
                    np.float32)
    assert np.array_equal(mine.view(np.uint32), golden["spectrum"].view(np.uint32))


def test_photon_generation_matches_the_reference(oracle, golden):
    batch = PhotonTransportBatch(golden["generate_emissions"].view(EMISSION_DTYPE), golden["generate_event_ids"],
                                 golden["generate_event_indices"])
    rows, times = oracle.generate(scenes.crystal_sipm_scene(), batch, rf.SEED, golden["generate_index"],
                                  golden["generate_local"], precision="fp32")
    reference = golden["generate_rows"].astype(np.float64)
    assert np.array_equal(rows[:, :3], reference[:, :3])  # position along the step
    assert np.array_equal(rows[:, 9], reference[:, 9])  # energy
    assert np.max(np.abs(rows[:, 3:9] - reference[:, 3:9])) < 1e-6  # direction, polarisation
    assert np.max(np.abs(times - golden["generate_time"]) / np.abs(golden["generate_time"])) < 1e-6


@pytest.mark.parametrize("name", sorted(rf.CASES))
def test_bounce_loop_matches_the_reference(oracle, golden, name):
    scene, batch = rf.case(golden, name)
    config = PhotonTransportConfig(seed=rf.SEED, precision="fp32", enable_performance_diagnostics=True)
    out = oracle.transport(scene, batch, config, record_fates=True)
    rf.assert_matches_reference(golden, name, out.photon_fate, out.detections, out.statistics)


def test_oracle_matches_the_live_reference_on_fresh_inputs(oracle):
    """Inputs outside the fixture (another seed, other events), where the
    reference tree was present to build oracle/_ref."""
    if oracle.load_reference_transport() is None:
        pytest.skip("the reference's device program is not built here (no reference tree)")
    for scene, batch in ((scenes.crystal_sipm_scene(), scenes.workload("batched", event_count=4, seed=1234)),
                         (scenes.rough_surface_scene(), scenes.workload("plain_fp64", event_count=1, seed=99))):
        config = PhotonTransportConfig(seed=777, precision="fp32", enable_performance_diagnostics=True)
        reference = oracle.reference_transport(scene, batch, config)
        mine = oracle.transport(scene, batch, config, record_fates=True)
        assert np.mean((mine.photon_fate & 7) == (reference.photon_fate & 7)) >= 0.9999
        assert np.mean(mine.photon_fate == reference.photon_fate) >= 0.9995
        n = reference.detections.shape[0]
        assert abs(mine.detections.shape[0] - n) <= max(1, 5e-4 * n)
