/*
 * g4b_synth.h - seeded synthetic genstep source.
 *
 * Geant4 is not available to this engine's test and benchmark harness, so
 * the Cerenkov and scintillation gensteps that Geant4EventAdapter would
 * capture (src/optical/geant4/Geant4EventAdapter.cpp:282-388, with yields
 * from G4GOQuasiScintillation.cpp:146-160,270-289) are produced here by a
 * stand-in electron track: straight steps along the incidence direction, a
 * continuous-slowing-down energy loss, scintillation yield x deposited energy
 * (Poisson below a mean of 10, Gaussian above), and a Frank-Tamm Cerenkov
 * mean per step with pre/post-step means. The records have the 128-byte
 * OpticalEmission layout and go straight into g4b_enqueue. This is input
 * synthesis for tests and benchmarks, not part of the transport.
 */
#ifndef G4B_SYNTH_H
#define G4B_SYNTH_H

#include <stdint.h>

#include "g4b.h"

#ifdef __cplusplus
extern "C" {
#endif

enum { G4B_SYNTH_ENERGY_FIXED = 0, G4B_SYNTH_ENERGY_UNIFORM = 1, G4B_SYNTH_ENERGY_LOG_UNIFORM = 2 };
enum { G4B_SYNTH_ENTRY_FACE_CENTER = 0, G4B_SYNTH_ENTRY_UNIFORM_ON_FACE = 1 };

typedef struct g4b_synth_params {
    uint32_t event_count;
    uint32_t first_event_id;
    uint64_t seed;
    uint32_t energy_mode;        /* G4B_SYNTH_ENERGY_* */
    uint32_t entry_mode;         /* G4B_SYNTH_ENTRY_*: on the crystal's -z face */
    double energy_min_mev;       /* the fixed energy for G4B_SYNTH_ENERGY_FIXED */
    double energy_max_mev;
    double max_incidence_deg;    /* polar angle uniform in [0, max] about +z, azimuth uniform */
    float crystal_center_mm[3];
    float crystal_half_size_mm[3];
    double step_mm;              /* 0 -> 0.1 */
    double density_g_cm3;        /* 0 -> 7.1 */
    double scintillation_yield_per_mev;
    double resolution_scale;     /* 0 -> 1 */
    float decay_time_ns;
    float rise_time_ns;
    uint32_t cerenkov;           /* 1: emit Cerenkov gensteps */
    uint32_t threads;            /* 0 -> all hardware threads */
    double rindex;               /* constant refractive index for the Cerenkov threshold and yield */
    double cerenkov_energy_min_ev;
    double cerenkov_energy_max_ev;
    uint32_t volume_id;
    uint32_t material_id;
    uint32_t spectrum_id;
    uint32_t reserved;
} g4b_synth_params;

typedef struct g4b_synth_batch g4b_synth_batch;

/* Generates the gensteps of params->event_count electron events. Event i has
 * event ID first_event_id + i; events are independent streams of the seed,
 * so the result does not depend on the thread count. */
int g4b_synth_electrons(const g4b_synth_params* params, g4b_synth_batch** out);

/* One direct photon (type 0, photon_count 1) per genstep: positions uniform
 * in the box, isotropic directions, random transverse polarisations,
 * wavelengths uniform in [wavelength_min_nm, wavelength_max_nm], grouped
 * photons_per_event to an event. */
int g4b_synth_isotropic_photons(uint64_t photon_count, uint32_t photons_per_event, uint64_t seed,
                                const float center_mm[3], const float half_size_mm[3], double wavelength_min_nm,
                                double wavelength_max_nm, uint32_t volume_id, uint32_t material_id,
                                g4b_synth_batch** out);

int g4b_synth_view(const g4b_synth_batch* batch, const g4b_optical_emission** emissions, uint32_t* emission_count,
                   const uint32_t** event_ids, uint32_t* event_count, const uint32_t** emission_event_indices,
                   uint64_t* photon_count);

void g4b_synth_free(g4b_synth_batch* batch);

const char* g4b_synth_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
