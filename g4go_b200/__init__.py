"""g4go_b200: B200-native optical-photon transport for G4GO's `--backend gpu` path.

Gensteps (Cerenkov / scintillation source records from Geant4) go in through
the C ABI in include/g4b.h; photon generation, the bounce loop and SiPM hit
compaction run in hand-written sm_100a CUDA (g4go_b200/csrc). This package is
the Python view of that ABI, mirroring the reference's transport interface.
"""
from .transport import (  # noqa: F401
    DETECTION_DTYPE,
    EMISSION_DTYPE,
    INVALID_ID,
    CapacityError,
    LogicError,
    Material,
    NoDeviceError,
    PhotonTransportBatch,
    PhotonTransportConfig,
    PhotonTransportOutput,
    Scene,
    Surface,
    SurfaceBinding,
    TransportHost,
    Volume,
    eval_fresnel,
    eval_lambertian,
    eval_math,
    eval_uniform,
)

__all__ = [
    "DETECTION_DTYPE", "EMISSION_DTYPE", "INVALID_ID", "CapacityError", "LogicError", "Material",
    "NoDeviceError", "PhotonTransportBatch", "PhotonTransportConfig", "PhotonTransportOutput", "Scene",
    "Surface", "SurfaceBinding", "TransportHost", "Volume", "eval_fresnel", "eval_lambertian", "eval_math",
    "eval_uniform",
]
