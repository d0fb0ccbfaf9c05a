"""Analytic scenes and synthetic workloads for the crystal + grease + SiPM detector.

The detector follows the surface pattern of G4GO's DetectorConstruction
(src/detector/DetectorConstruction.cpp:50-169): a scintillating crystal in a
world of air, a specular reflective wrapper on the crystal's faces toward the
world (border surface crystal -> world), a black coating world -> crystal, an
optical-grease coupling layer on the +z end face and a SiPM behind it whose
skin surface absorbs everything and detects with a flat efficiency.

Workloads (all seeded, synthetic: there is no Geant4 here):
  plain_cpu    1,000 x 1 MeV e-, face centre, normal incidence, 1,000 ph/MeV
  plain_fp64   5,000 e-, 1-10 MeV uniform, 10,000 ph/MeV + Cerenkov
  batched      50,000 e-, 0.1-20 MeV log-uniform, entry uniform on the face,
               incidence uniform to 30 deg, 10,000 ph/MeV + Cerenkov
  precision    1e7 single photons, uniform in the crystal, isotropic,
               wavelength uniform in 380-500 nm
  gradients    2,000 x 5 MeV e-, 10,000 ph/MeV + Cerenkov
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from .transport import (
    INVALID_ID,
    Material,
    PhotonTransportBatch,
    Scene,
    Surface,
    SurfaceBinding,
    Volume,
    raise_for_status,
)

HC_EV_NM = 1239.84198
CERENKOV_EV = (HC_EV_NM / 500.0, HC_EV_NM / 380.0)  # RINDEX range, 380-500 nm


def gaussian_spectrum(mean_nm: float = 420.0, sigma_nm: float = 20.0, points: int = 64):
    """Emission spectrum Gaussian in wavelength, tabulated in ascending energy (relative intensity per eV)."""
    lo_ev = HC_EV_NM / (mean_nm + 4.0 * sigma_nm)
    hi_ev = HC_EV_NM / (mean_nm - 4.0 * sigma_nm)
    energy = np.linspace(lo_ev, hi_ev, points)
    wavelength = HC_EV_NM / energy
    intensity = np.exp(-0.5 * ((wavelength - mean_nm) / sigma_nm) ** 2) * wavelength**2 / HC_EV_NM
    return energy.astype(np.float32), (intensity / intensity.max()).astype(np.float32)


def _flat(value: float, energies=None):
    e = energies if energies is not None else CERENKOV_EV
    return (np.array([e[0], e[1]], dtype=np.float32), np.array([value, value], dtype=np.float32))


@dataclass
class DetectorParameters:
    crystal_half_mm: tuple = (1.5, 1.5, 5.0)  # 3 x 3 x 10 mm
    crystal_rindex: float = 1.82
    crystal_abs_length_mm: float = 400.0
    crystal_rayleigh_length_mm: float | None = None  # off
    grease_rindex: float = 1.41
    grease_thickness_mm: float = 0.1
    sipm_thickness_mm: float = 0.1
    wrapper_reflectivity: float = 0.95
    sipm_efficiency: float = 0.3
    world_half_mm: float = 50.0
    coupling_half_xy_mm: float | None = None  # grease and SiPM half width; None -> the crystal's
    emission_mean_nm: float = 420.0
    emission_sigma_nm: float = 20.0


# Volume, material and surface IDs of the detector scene.
WORLD, CRYSTAL, GREASE, SIPM = 0, 1, 2, 3
MAT_AIR, MAT_CRYSTAL, MAT_GREASE, MAT_SILICON = 0, 1, 2, 3
SURF_WRAPPER, SURF_COATING, SURF_CATHODE = 0, 1, 2


def crystal_sipm_scene(params: DetectorParameters | None = None) -> Scene:
    p = params or DetectorParameters()
    scene = Scene()
    spectrum_energy, spectrum_values = gaussian_spectrum(p.emission_mean_nm, p.emission_sigma_nm)
    wide = (min(CERENKOV_EV[0], float(spectrum_energy[0])), max(CERENKOV_EV[1], float(spectrum_energy[-1])))
    scene.add_material(Material(name="air", rindex=_flat(1.0)))
    scene.add_material(
        Material(
            name="crystal",
            rindex=_flat(p.crystal_rindex),
            abs_length_mm=_flat(p.crystal_abs_length_mm, wide),
            rayleigh_length_mm=None if p.crystal_rayleigh_length_mm is None else _flat(p.crystal_rayleigh_length_mm, wide),
            scintillation_spectrum=[(spectrum_energy, spectrum_values), None, None],
        )
    )
    scene.add_material(Material(name="grease", rindex=_flat(p.grease_rindex)))
    scene.add_material(Material(name="silicon"))
    wrapper = scene.add_surface(
        Surface(
            name="wrapper", type=_abi.SURFACE_DIELECTRIC_METAL, model=_abi.MODEL_UNIFIED,
            finish=_abi.FINISH_POLISHED, reflectivity=_flat(p.wrapper_reflectivity, wide),
        )
    )
    coating = scene.add_surface(
        Surface(
            name="coating", type=_abi.SURFACE_DIELECTRIC_METAL, model=_abi.MODEL_UNIFIED,
            finish=_abi.FINISH_POLISHED, reflectivity=_flat(0.0, wide),
        )
    )
    cathode = scene.add_surface(
        Surface(
            name="cathode", type=_abi.SURFACE_DIELECTRIC_METAL, model=_abi.MODEL_UNIFIED,
            finish=_abi.FINISH_POLISHED, reflectivity=_flat(0.0, wide), efficiency=_flat(p.sipm_efficiency, wide),
        )
    )
    hx, hy, hz = p.crystal_half_mm
    w = p.world_half_mm
    scene.add_volume(Volume("world", WORLD, MAT_AIR, INVALID_ID, INVALID_ID, INVALID_ID, (0.0, 0.0, 0.0), (w, w, w)))
    scene.add_volume(Volume("crystal", CRYSTAL, MAT_CRYSTAL, WORLD, INVALID_ID, INVALID_ID, (0.0, 0.0, 0.0), (hx, hy, hz)))
    g = p.grease_thickness_mm
    cx = hx if p.coupling_half_xy_mm is None else p.coupling_half_xy_mm
    cy = hy if p.coupling_half_xy_mm is None else p.coupling_half_xy_mm
    scene.add_volume(
        Volume("grease", GREASE, MAT_GREASE, WORLD, INVALID_ID, INVALID_ID, (0.0, 0.0, hz + g / 2), (cx, cy, g / 2))
    )
    s = p.sipm_thickness_mm
    scene.add_volume(
        Volume("sipm", SIPM, MAT_SILICON, WORLD, cathode, 0, (0.0, 0.0, hz + g + s / 2), (cx, cy, s / 2))
    )
    scene.add_surface_binding(SurfaceBinding(CRYSTAL, WORLD, wrapper))
    scene.add_surface_binding(SurfaceBinding(WORLD, CRYSTAL, coating))
    scene.world_volume_id = WORLD
    return scene


def rough_surface_scene(params: DetectorParameters | None = None) -> Scene:
    """The detector with rough surfaces on the reference's bounded paths: a
    ground unified wrapper (sigma_alpha 0.2 rad; specular lobe, spike,
    backscatter and Lambertian parts) and a ground unified crystal-grease face
    (sigma_alpha 0.1 rad, with a surface-roughness table so the roughness
    criterion of the reference's dielectric surfaces runs). No glisur ground
    surface: the reference's glisur facet loop never ends once a smear leaves
    the unit ball."""
    scene = crystal_sipm_scene(params)
    energies = np.array([1.5, 4.5], np.float32)

    def flat(value):
        return energies, np.array([value, value], np.float32)

    ground = scene.add_surface(Surface(
        name="ground_wrapper", type=_abi.SURFACE_DIELECTRIC_METAL, model=_abi.MODEL_UNIFIED,
        finish=_abi.FINISH_GROUND, model_value=0.2, reflectivity=flat(0.9),
        specular_lobe=flat(0.3), specular_spike=flat(0.2), backscatter=flat(0.1),
    ))
    face = scene.add_surface(Surface(
        name="ground_coupling", type=_abi.SURFACE_DIELECTRIC_DIELECTRIC, model=_abi.MODEL_UNIFIED,
        finish=_abi.FINISH_GROUND, model_value=0.1, surface_roughness=flat(2.0e-5),
        specular_lobe=flat(0.5), specular_spike=flat(0.3),
    ))
    scene.surface_bindings = [
        SurfaceBinding(CRYSTAL, WORLD, ground),
        SurfaceBinding(WORLD, CRYSTAL, SURF_COATING),
        SurfaceBinding(CRYSTAL, GREASE, face),
    ]
    return scene


# ---------------------------------------------------------------------------
# Synthetic gensteps (include/g4b_synth.h)
# ---------------------------------------------------------------------------

def _take(batch_ptr: C.c_void_p) -> PhotonTransportBatch:
    lib = _abi.load_synth()
    emissions = C.c_void_p()
    n = C.c_uint32()
    event_ids = C.c_void_p()
    n_events = C.c_uint32()
    indices = C.c_void_p()
    photons = C.c_uint64()
    try:
        raise_for_status(
            lib.g4b_synth_view(batch_ptr, C.byref(emissions), C.byref(n), C.byref(event_ids), C.byref(n_events),
                               C.byref(indices), C.byref(photons)),
            lib.g4b_synth_last_error().decode(),
        )
        count, events = int(n.value), int(n_events.value)
        em = np.empty(count, dtype=_abi.EMISSION_DTYPE)
        ev = np.empty(events, dtype=np.uint32)
        ix = np.empty(count, dtype=np.uint32)
        if count:
            C.memmove(em.ctypes.data, emissions.value, count * 128)
            C.memmove(ix.ctypes.data, indices.value, count * 4)
        if events:
            C.memmove(ev.ctypes.data, event_ids.value, events * 4)
    finally:
        lib.g4b_synth_free(batch_ptr)
    return PhotonTransportBatch(em, ev, ix)


def electron_gensteps(
    event_count: int,
    energy_mev: tuple = (1.0, 1.0),
    energy_mode: str = "fixed",
    entry: str = "center",
    max_incidence_deg: float = 0.0,
    yield_per_mev: float = 1000.0,
    cerenkov: bool = False,
    decay_time_ns: float = 40.0,
    rise_time_ns: float = 0.0,
    seed: int = 1,
    first_event_id: int = 0,
    params: DetectorParameters | None = None,
    threads: int = 0,
) -> PhotonTransportBatch:
    """Gensteps of `event_count` electrons entering the crystal's -z face."""
    p = params or DetectorParameters()
    lib = _abi.load_synth()
    sp = _abi.SynthParams()
    sp.event_count = event_count
    sp.first_event_id = first_event_id
    sp.seed = seed
    sp.energy_mode = {"fixed": 0, "uniform": 1, "log_uniform": 2}[energy_mode]
    sp.entry_mode = {"center": 0, "uniform": 1}[entry]
    sp.energy_min_mev, sp.energy_max_mev = float(energy_mev[0]), float(energy_mev[1])
    sp.max_incidence_deg = float(max_incidence_deg)
    for a in range(3):
        sp.crystal_center_mm[a] = 0.0
        sp.crystal_half_size_mm[a] = float(p.crystal_half_mm[a])
    sp.step_mm = 0.1
    sp.density_g_cm3 = 7.1
    sp.scintillation_yield_per_mev = float(yield_per_mev)
    sp.resolution_scale = 1.0
    sp.decay_time_ns = float(decay_time_ns)
    sp.rise_time_ns = float(rise_time_ns)
    sp.cerenkov = int(bool(cerenkov))
    sp.threads = threads
    sp.rindex = float(p.crystal_rindex)
    sp.cerenkov_energy_min_ev, sp.cerenkov_energy_max_ev = CERENKOV_EV
    sp.volume_id = CRYSTAL
    sp.material_id = MAT_CRYSTAL
    sp.spectrum_id = 0
    out = C.c_void_p()
    raise_for_status(lib.g4b_synth_electrons(C.byref(sp), C.byref(out)), lib.g4b_synth_last_error().decode())
    return _take(out)


def isotropic_photons(
    photon_count: int,
    photons_per_event: int = 1000,
    seed: int = 1,
    wavelength_nm: tuple = (380.0, 500.0),
    params: DetectorParameters | None = None,
) -> PhotonTransportBatch:
    """Single photons uniform in the crystal, isotropic, wavelength uniform in the range."""
    p = params or DetectorParameters()
    lib = _abi.load_synth()
    center = (C.c_float * 3)(0.0, 0.0, 0.0)
    half = (C.c_float * 3)(*p.crystal_half_mm)
    out = C.c_void_p()
    raise_for_status(
        lib.g4b_synth_isotropic_photons(
            photon_count, photons_per_event, seed, center, half, wavelength_nm[0], wavelength_nm[1], CRYSTAL,
            MAT_CRYSTAL, C.byref(out),
        ),
        lib.g4b_synth_last_error().decode(),
    )
    return _take(out)


WORKLOADS = {
    "plain_cpu": dict(event_count=1000, energy_mev=(1.0, 1.0), energy_mode="fixed", entry="center",
                      max_incidence_deg=0.0, yield_per_mev=1000.0, cerenkov=False),
    "plain_fp64": dict(event_count=5000, energy_mev=(1.0, 10.0), energy_mode="uniform", entry="center",
                       max_incidence_deg=0.0, yield_per_mev=10000.0, cerenkov=True),
    "batched": dict(event_count=50000, energy_mev=(0.1, 20.0), energy_mode="log_uniform", entry="uniform",
                    max_incidence_deg=30.0, yield_per_mev=10000.0, cerenkov=True),
    "gradients": dict(event_count=2000, energy_mev=(5.0, 5.0), energy_mode="fixed", entry="center",
                      max_incidence_deg=0.0, yield_per_mev=10000.0, cerenkov=True),
}


def workload(name: str, event_count: int | None = None, seed: int = 1, **overrides) -> PhotonTransportBatch:
    spec = dict(WORKLOADS[name])
    if event_count is not None:
        spec["event_count"] = event_count
    spec.update(overrides)
    return electron_gensteps(seed=seed, **spec)
