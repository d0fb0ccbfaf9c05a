"""The CUDA engine against the reference's own device program, directly.

The fixture (tests/golden/transport_reference.npz) holds per-photon
outcomes, bounce counts and detections of src/optical/optix/OptiXTransportDevice.cu
compiled for the host. The engine runs the same gensteps under the same seed
in its default batched FP32 form and in the form that reads the photon store
(the generation pass, in waves), records every photon's fate, and must meet
the gates of tests/reference_fixture.py, as the oracle does on the CPU.
"""
import pytest

import reference_fixture as rf
from g4go_b200 import PhotonTransportConfig, TransportHost

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden():
    return rf.load()


@pytest.mark.parametrize("generation_pass", [2, 3])
@pytest.mark.parametrize("name", sorted(rf.CASES))
def test_engine_matches_the_reference(golden, name, generation_pass):
    scene, batch = rf.case(golden, name)
    config = PhotonTransportConfig(seed=rf.SEED, precision="fp32", record_photon_fates=True,
                                   generation_pass=generation_pass, wave_photons=8192)
    with TransportHost(config) as host:
        host.enqueue_emissions(scene, batch)
        out = host.complete_oldest_batch()
        fates, _ = host.photon_fates()
    rf.assert_matches_reference(golden, name, fates, out.detections, out.statistics)
