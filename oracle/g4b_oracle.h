/*
 * g4b_oracle.h - CPU oracle for the optical-photon transport path.
 *
 * TEST INFRASTRUCTURE ONLY. This library restates, on the CPU, the algorithm
 * of G4GO's GPU optical path (src/optical/optix/OptiXTransportDevice.cu and
 * OptiXBoundaryPhysics.cuh, host-side tables from OptiXTransportHost.cpp)
 * with the engine's analytic box intersection standing where optixTrace
 * stood. It is the checker for the CUDA engine: the tests, the smoke check
 * and the CPU-baseline leg of the benchmark may call it; the engine never
 * does. It shares no source with the engine.
 *
 * Pinning: its boundary functions are compared with the reference's own
 * OptiXBoundaryPhysics.cuh compiled from the reference tree (oracle/_ref) and
 * with the reference's known-answer tests (test/TestOpticalBoundaryPhysics.cxx:37-101).
 */
#ifndef G4B_ORACLE_H
#define G4B_ORACLE_H

#include <stdint.h>

#include "../include/g4b.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_result {
    /* detections in flattened-photon order (the reference's compacted order) */
    g4b_photon_detection* detections;
    uint64_t detection_capacity;
    uint64_t detection_count;
    /* per-event statistics, in event order of the batch */
    g4b_event_statistics* event_statistics;
    uint32_t event_capacity;
    uint32_t event_count;
    g4b_statistics statistics;
    uint64_t total_bounce_count;
    uint64_t coincident_candidate_trace_count;
    uint64_t coincident_candidate_hit_count;
    /* optional per-photon records (may be NULL): outcome | bounces << 3, end time */
    uint32_t* photon_fate;
    double* photon_time_ns;
    uint64_t photon_capacity;
    uint64_t photon_count;
} oracle_result;

/* Transports one batch. precision: G4B_PRECISION_FP32 or G4B_PRECISION_FP64.
 * threads: 0 -> all hardware threads. photon_begin/photon_end restrict the
 * run to a slice of the flattened photon range (photon_end 0 -> all), used
 * for bounded CPU-baseline samples. Returns 0 or a negative g4b_status.
 * With result->detections NULL the detections are kept (on the calling
 * thread) for oracle_take_detections, so a caller that does not know the
 * count in advance transports the photons once. */
int oracle_transport(const g4b_scene* scene, const g4b_config* config, const g4b_optical_emission* emissions,
                     uint32_t emission_count, const uint32_t* event_ids, uint32_t event_count,
                     const uint32_t* emission_event_indices, uint32_t threads, uint64_t photon_begin,
                     uint64_t photon_end, oracle_result* result);

const char* oracle_last_error(void);

/* Copies up to `capacity` detections kept by the calling thread's last
 * oracle_transport call without a detection buffer into `out`, releases them,
 * and returns how many there were. */
uint64_t oracle_take_detections(g4b_photon_detection* out, uint64_t capacity);

/* Restated boundary functions (OptiXBoundaryPhysics.cuh), FP32 and FP64. */
void oracle_fresnel_f(const float direction[3], const float polarization[3], const float normal[3], float index_from,
                      float index_to, float out[14]);
void oracle_fresnel_d(const double direction[3], const double polarization[3], const double normal[3],
                      double index_from, double index_to, double out[14]);
int oracle_classify_surface(float reflectivity, float transmittance, int has_reflectivity, int has_transmittance,
                            float sample);
int oracle_evaluate_absorption(float efficiency, int sensor, float sample);
void oracle_lambertian_f(const float normal[3], float radial, float azimuth, float out[3]);
void oracle_lambertian_d(const double normal[3], double radial, double azimuth, double out[3]);

/* The engine's own transcendental functions, restated (float and double). */
float oracle_log_f(float x);
float oracle_exp_f(float x);
void oracle_sincos_turn_f(float turns, float* s, float* c);
double oracle_log_d(double x);
double oracle_exp_d(double x);
void oracle_sincos_turn_d(double turns, double* s, double* c);

/* GeneratePhoton (OptiXTransportDevice.cu:346-481) for photon local[i] of
 * genstep emissionIndex[i], in FP32 or FP64. Each output row: position[3],
 * direction[3], polarization[3], energy; the global time separately. */
int oracle_generate(const g4b_scene* scene, uint64_t seed, uint32_t precision,
                    const g4b_optical_emission* emissions, uint32_t emission_count, const uint32_t* emission_index,
                    const uint32_t* local, uint32_t n, double* out, double* time_out);

/* SampleProperty (OptiXTransportDevice.cu:198-216) on a property table, and
 * SampleSpectrum (:322-344) on the CDF the oracle builds from a spectrum
 * table (OptiXTransportHost.cpp:371-410), in FP32. */
float oracle_sample_property_f(const float* energy, const float* values, uint32_t count, float x,
                               float default_value);
float oracle_sample_spectrum_f(const float* energy, const float* values, uint32_t count, float u);

/* Uniform(seed, key, bounce, process, draw) (OptiXTransportDevice.cu:254-286). */
float oracle_uniform_f(uint64_t seed, uint64_t photon_key, uint32_t bounce, uint32_t process, uint32_t draw);

/* Normalised trapezoid CDF of a scintillation spectrum
 * (OptiXTransportHost.cpp:371-410); returns count or 0 if rejected. */
uint32_t oracle_spectrum_cdf(const float* energy, const float* values, uint32_t count, float* cdf_out);

#ifdef __cplusplus
}
#endif

#endif
