"""Generates tests/golden/transport_reference.npz from the reference itself.

Runs the reference's own device program (src/optical/optix/OptiXTransportDevice.cu,
compiled unmodified for the host by oracle/Makefile into
oracle/_ref/libref_transport.so, with oracle/ref_transport_shim.cpp standing
in for the OptiX pipeline) and records, for fixed seeded inputs:

- Uniform(seed, key, bounce, process, draw) over random counters;
- SampleProperty over an ascending table and SampleSpectrum over the
  detector's emission spectrum, with that spectrum's CDF;
- GeneratePhoton for random photons of Cerenkov and scintillation gensteps;
- the bounce loop (__raygen__rg) for every photon of six small batches:
  per-photon outcome and bounce count, the detections in flattened order,
  run and per-event counters. The batches: 1 MeV and 1-10 MeV electrons at
  the face centre, uneven log-uniform electrons, single isotropic photons,
  1 MeV electrons in the detector with rough (unified, ground) surfaces, and
  gensteps whose photons include histories of thousands of bounces.

The gensteps are stored with the outputs, so the fixture holds its inputs.
Needs the reference tree (G4GO_REFERENCE) to build oracle/_ref:

    G4GO_REFERENCE=<reference tree> python tests/golden/make_golden_transport.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from g4go_b200 import PhotonTransportConfig, scenes  # noqa: E402
from oracle import binding  # noqa: E402

OUT = Path(__file__).resolve().parent / "transport_reference.npz"
SEED = 42

# name -> (scene builder, batch builder)
CASES = {
    "one_mev": ("crystal_sipm_scene", lambda: scenes.workload("plain_cpu", event_count=40, seed=5)),
    "one_to_ten_mev": ("crystal_sipm_scene", lambda: scenes.workload("plain_fp64", event_count=1, seed=6)),
    "uneven": ("crystal_sipm_scene", lambda: scenes.workload("batched", event_count=3, seed=7)),
    "isotropic": ("crystal_sipm_scene", lambda: scenes.isotropic_photons(6000, photons_per_event=500, seed=3)),
    "rough": ("rough_surface_scene", lambda: scenes.workload("plain_cpu", event_count=30, seed=8)),
    "long_histories": ("crystal_sipm_scene", lambda: long_history_batch()),
}


def long_history_batch():
    """The five scintillation gensteps of the uneven workload (1,500 events,
    seed 1) that hold photons the reference keeps for thousands of bounces:
    photons that leave the crystal within the boundary tolerance of its face
    and then reflect totally inside the grease layer while counted in the
    crystal. 5,427 photons; eleven run to the 4,096-bounce limit."""
    from g4go_b200 import PhotonTransportBatch

    batch = scenes.workload("batched", event_count=200, seed=1)
    picks = np.array([866, 1888, 3038, 4101, 5370])
    return PhotonTransportBatch(batch.emissions[picks], batch.event_ids, batch.emission_event_indices[picks])
STAT_KEYS = ("detected_count", "absorbed_count", "escaped_count", "truncated_count", "max_bounce_count",
             "invalid_state_count", "zero_step_count")


def main() -> None:
    lib = binding.load_reference_transport()
    if lib is None:
        raise SystemExit("oracle/_ref/libref_transport.so is missing: set G4GO_REFERENCE and build oracle/")
    rng = np.random.default_rng(20260101)
    out: dict[str, np.ndarray] = {}

    # Uniform over random counters
    n = 4096
    seeds = np.array([0, SEED, (1 << 63) + 5, 0xDEADBEEFCAFEF00D], dtype=np.uint64)
    keys = rng.integers(0, 2**64, size=n, dtype=np.uint64)
    bounce = rng.integers(0, 4096, size=n).astype(np.uint32)
    process = rng.choice([0, 1, 2, 3, 4, 10, 20], size=n).astype(np.uint32)
    draw = rng.integers(0, 2048, size=n).astype(np.uint32)
    uniform = np.array([[lib.ref_uniform(int(s), int(k), int(b), int(p), int(d))
                         for k, b, p, d in zip(keys, bounce, process, draw)] for s in seeds], dtype=np.float32)
    out.update(uniform_seeds=seeds, uniform_keys=keys, uniform_bounce=bounce, uniform_process=process,
               uniform_draw=draw, uniform=uniform)

    # SampleProperty over an ascending table, SampleSpectrum over the emission spectrum
    import ctypes as C

    f = C.POINTER(C.c_float)
    table_e = np.array([1.8, 2.0, 2.3, 2.5, 2.9, 3.1, 3.3, 3.6, 4.0], np.float32)
    table_v = np.array([0.05, 0.12, 0.25, 0.31, 0.30, 0.22, 0.15, 0.07, 0.02], np.float32)
    queries = np.concatenate([rng.uniform(1.5, 4.3, 2000), table_e, [1.0, 5.0]]).astype(np.float32)
    prop = np.array([lib.ref_sample_property(table_e.ctypes.data_as(f), table_v.ctypes.data_as(f), table_e.size, 0,
                                             float(x), -1.0) for x in queries], np.float32)
    spec_e, spec_v = scenes.gaussian_spectrum()
    spec_e = np.ascontiguousarray(spec_e, np.float32)
    spec_v = np.ascontiguousarray(spec_v, np.float32)
    cdf = np.empty_like(spec_v)
    assert lib.ref_spectrum_cdf(spec_e.ctypes.data_as(f), spec_v.ctypes.data_as(f), spec_e.size,
                                cdf.ctypes.data_as(f)) == spec_e.size
    us = np.concatenate([rng.random(2000), [0.0, 1.0, cdf[0], cdf[5], cdf[-2]]]).astype(np.float32)
    spectrum = np.array([lib.ref_sample_spectrum(spec_e.ctypes.data_as(f), cdf.ctypes.data_as(f), spec_e.size,
                                                 float(u)) for u in us], np.float32)
    out.update(property_energy=table_e, property_values=table_v, property_queries=queries, property=prop,
               spectrum_energy=spec_e, spectrum_values=spec_v, spectrum_cdf=cdf, spectrum_queries=us,
               spectrum=spectrum)

    # GeneratePhoton on Cerenkov and scintillation gensteps
    scene = scenes.crystal_sipm_scene()
    gen_batch = scenes.workload("plain_fp64", event_count=2, seed=9)
    counts = gen_batch.emissions["photon_count"].astype(np.int64)
    picks = rng.choice(np.nonzero(counts > 0)[0], size=3000)
    local = (rng.random(3000) * counts[picks]).astype(np.uint32)
    rows, times = binding.generate(scene, gen_batch, SEED, picks, local, reference=True)
    out.update(generate_emissions=gen_batch.emissions.view(np.uint8), generate_event_ids=gen_batch.event_ids,
               generate_event_indices=gen_batch.emission_event_indices, generate_index=picks.astype(np.uint32),
               generate_local=local, generate_rows=rows.astype(np.float32), generate_time=times)

    # The bounce loop, photon by photon
    for name, (scene_name, make) in CASES.items():
        scene = getattr(scenes, scene_name)()
        batch = make()
        config = PhotonTransportConfig(seed=SEED, precision="fp32", enable_performance_diagnostics=True)
        ref = binding.reference_transport(scene, batch, config)
        per_event = np.array([[s[k] for k in STAT_KEYS] for _, s in ref.event_statistics], np.uint64)
        out.update({
            f"{name}_emissions": batch.emissions.view(np.uint8),
            f"{name}_event_ids": batch.event_ids,
            f"{name}_event_indices": batch.emission_event_indices,
            f"{name}_fate": ref.photon_fate,
            f"{name}_detections": ref.detections.view(np.uint8),
            f"{name}_statistics": np.array([ref.statistics[k] for k in STAT_KEYS], np.uint64),
            f"{name}_event_statistics": per_event,
            f"{name}_bounces": np.array([ref.total_bounce_count], np.uint64),
            f"{name}_coincident": np.array(ref.coincident, np.uint64),
        })
        print(f"{name}: {batch.photon_count} photons, {ref.detections.shape[0]} detections, "
              f"{ref.total_bounce_count} bounces")
    out["scenes"] = np.array([f"{k}:{v[0]}" for k, v in CASES.items()])
    out["seed"] = np.array([SEED], np.uint64)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
