/*
 * g4b.h - C ABI of the B200 optical-photon transport engine.
 *
 * This is the drop-in boundary for the `--backend gpu` optical path of G4GO.
 * Geant4 keeps the charged-particle tracking on the host and hands over
 * gensteps (one Cerenkov or scintillation source record per charged step);
 * everything after that (photon generation, the bounce loop, SiPM hit
 * compaction) runs in hand-written sm_100a CUDA behind this header.
 *
 * The entry points replace the C++ class OptiXTransportHost
 * (include/g4go/optical/optix/OptiXTransportHost.hpp:10-26):
 *
 *   OptiXTransportHost(PhotonTransportConfig)   -> g4b_create
 *   ~OptiXTransportHost()                        -> g4b_destroy
 *   PrepareScene(const Scene&)                   -> g4b_set_scene
 *   EnqueueEmissions(const Scene&, batch)        -> g4b_enqueue
 *   CompleteOldestBatch()                        -> g4b_query_oldest + g4b_complete
 *
 * Conventions:
 *   - every function returns an int status (G4B_OK == 0, negative on error);
 *     g4b_last_error(handle) gives the message of the last failure on that
 *     handle (g4b_last_error(NULL) for calls that take no handle);
 *   - no C++ exception crosses this boundary;
 *   - plain pointers and sizes only; the caller owns every buffer it passes,
 *     borrowed for the duration of the call (inputs are copied into the
 *     engine's pinned staging before the call returns);
 *   - units as in the reference: mm, ns, eV.
 *
 * A handle is used from one host thread at a time, like OptiXTransportHost,
 * which only OpticalBatchScheduler's GPU thread calls
 * (src/optical/geant4/OpticalBatchScheduler.cpp:556-618).
 */
#ifndef G4B_H
#define G4B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define G4B_ABI_VERSION 1u
#define G4B_INVALID_ID 0xffffffffu

/* Limits of the analytic scene held in shared memory by every CTA. */
#define G4B_MAX_VOLUMES 64u
#define G4B_MAX_MATERIALS 16u
#define G4B_MAX_SURFACES 16u
#define G4B_MAX_PROPERTY_FLOATS 6144u

/* Status codes. The C++ shim (g4b_transport_host.hpp) maps them back onto
 * the exception types OptiXTransportHost throws
 * (src/optical/optix/OptiXTransportHost.cpp:47-52,515,524,575-605,655-660,781). */
typedef enum g4b_status {
    G4B_OK = 0,
    G4B_ERR_INVALID_ARGUMENT = -1, /* std::invalid_argument */
    G4B_ERR_OVERFLOW = -2,         /* std::overflow_error */
    G4B_ERR_LOGIC = -3,            /* std::logic_error: queue full/empty, scene rebuild while busy */
    G4B_ERR_CUDA = -4,             /* std::runtime_error from a CUDA call */
    G4B_ERR_CAPACITY = -5,         /* caller's output buffer too small; the batch stays pending */
    G4B_ERR_TIMEOUT = -6,          /* a bounded device wait gave up */
    G4B_ERR_NO_SCENE = -7,         /* enqueue before any scene was set */
    G4B_ERR_UNSUPPORTED = -8,      /* scene feature outside the analytic-box engine */
    G4B_ERR_NO_DEVICE = -9         /* no CUDA device / the kernel image cannot run here */
} g4b_status;

/* OpticalEmissionType (include/g4go/optical/PhotonTransport.hpp:14-18). */
typedef enum g4b_emission_type {
    G4B_EMISSION_DIRECT = 0,
    G4B_EMISSION_CERENKOV = 1,
    G4B_EMISSION_SCINTILLATION = 2
} g4b_emission_type;

/* Genstep: byte-for-byte the 128-byte OpticalEmission record
 * (include/g4go/optical/PhotonTransport.hpp:40-69, static_assert :177), so a
 * std::span<const OpticalEmission> can be passed through unchanged. */
typedef struct g4b_optical_emission {
    float position_mm[3];
    float time_ns;
    float direction[3];
    float step_length_mm;
    float step_delta_mm[3];
    float pre_velocity_mm_per_ns;
    float polarization[3];
    float delta_velocity_mm_per_ns;
    float energy_ev;
    float pre_mean_photon_count;
    float post_mean_photon_count;
    float decay_time_ns;
    float rise_time_ns;
    float charge;
    uint32_t event_id;
    uint32_t first_photon_id;
    uint32_t photon_count;
    uint32_t volume_id;
    uint32_t material_id;
    uint32_t spectrum_id;
    uint8_t type; /* g4b_emission_type */
    uint8_t reserved[15];
} g4b_optical_emission;

/* Detection: byte-for-byte the 48-byte PhotonDetection record
 * (include/g4go/optical/PhotonTransport.hpp:71-81, static_assert :178). */
typedef struct g4b_photon_detection {
    float position_mm[3];
    float time_ns;
    float direction[3];
    float energy_ev;
    uint32_t event_id;
    uint32_t photon_id;
    uint32_t sensor_id;
    uint32_t reserved;
} g4b_photon_detection;

/* PhotonTransportStatisticField bit numbers (PhotonTransport.hpp:20-35). */
enum {
    G4B_FIELD_GENERATED = 0,
    G4B_FIELD_CAPTURED = 1,
    G4B_FIELD_DETECTED = 2,
    G4B_FIELD_ABSORBED = 3,
    G4B_FIELD_ESCAPED = 4,
    G4B_FIELD_TRUNCATED = 5,
    G4B_FIELD_MAX_BOUNCE = 6,
    G4B_FIELD_INVALID_STATE = 7,
    G4B_FIELD_ZERO_STEP = 8,
    G4B_FIELD_TRANSPORT_TIME = 9
};

/* PhotonTransportStatistics (PhotonTransport.hpp:83-95). */
typedef struct g4b_statistics {
    uint32_t valid_fields;
    uint32_t reserved;
    uint64_t generated_count;
    uint64_t captured_count;
    uint64_t detected_count;
    uint64_t absorbed_count;
    uint64_t escaped_count;
    uint64_t truncated_count;
    uint64_t max_bounce_count;
    uint64_t invalid_state_count;
    uint64_t zero_step_count;
    double transport_time_ms;
} g4b_statistics;

/* PhotonTransportEventStatistics (PhotonTransport.hpp:97-100). */
typedef struct g4b_event_statistics {
    uint32_t event_id;
    uint32_t reserved;
    g4b_statistics statistics;
} g4b_event_statistics;

/* The transport-side fields of PhotonTransportPerformance
 * (PhotonTransport.hpp:102-150); kernel_ms stands where optiXKernelMs stood.
 * Hit compaction is fused into the transport kernel, so
 * device_hit_compaction_ms is always 0. */
typedef struct g4b_performance {
    double host_to_device_ms;
    uint64_t host_to_device_bytes;
    double device_memset_ms;
    double kernel_ms;
    double device_hit_compaction_ms;
    double device_to_host_ms;
    double device_metadata_to_host_ms;
    uint64_t device_metadata_to_host_bytes;
    double device_hits_to_host_ms;
    uint64_t device_hits_to_host_bytes;
    double host_hit_compaction_ms;
    uint64_t total_bounce_count;
    uint64_t coincident_candidate_trace_count;
    uint64_t coincident_candidate_hit_count;
    uint64_t kernel_launch_count;
} g4b_performance;

/* Arithmetic of the transport (positions, directions, Fresnel, tables). */
typedef enum g4b_precision {
    G4B_PRECISION_FP32 = 0, /* FP32 transport, FP64 global time and near-grazing TIR test */
    G4B_PRECISION_FP64 = 1  /* everything in FP64 */
} g4b_precision;

/* How a batch is launched. */
typedef enum g4b_launch_form {
    /* one persistent launch per batch, warps refill lanes from a device work
     * queue, replayed from a captured CUDA graph */
    G4B_FORM_BATCHED = 0,
    /* one launch per event, one thread per photon (the reference's layout) */
    G4B_FORM_PLAIN = 1
} g4b_launch_form;

/* Engine configuration: the transport fields of PhotonTransportConfig
 * (include/g4go/optical/PhotonTransportConfig.hpp:26-40) plus the launch
 * knobs of this engine. Zero-initialise, set abi_version, then override. */
typedef struct g4b_config {
    uint32_t abi_version;            /* must be G4B_ABI_VERSION */
    int32_t device;                  /* CUDA device ordinal; -1 = current device */
    uint64_t seed;                   /* PhotonTransportConfig::seed */
    uint32_t max_bounces_per_photon; /* 0 -> 4096 (PhotonTransportConfig.hpp:30) */
    float boundary_tolerance_mm;     /* 0 -> 1e-4 (PhotonTransportConfig.hpp:31) */
    uint32_t precision;              /* g4b_precision */
    uint32_t launch_form;            /* g4b_launch_form */
    uint32_t enable_performance_diagnostics; /* 1: count coincident-face retraces and hits
                                                (g4b_performance), as the reference does only then */
    uint32_t ordered_detections;     /* 1: detections in flattened photon order, as the reference returns them */
    uint64_t hit_capacity;           /* device hit-buffer rows; 0 -> photons of the batch */
    uint32_t block_size;             /* 0 -> autotuned/default (256) */
    uint32_t blocks_per_sm;          /* 0 -> from occupancy */
    uint32_t chunk_photons;          /* photons a warp takes from the work queue at a time (rounded up to
                                        a multiple of 32); 0 -> 512, or less (down to 32) for a batch
                                        too small to give every warp eight chunks, until g4b_autotune
                                        picks one. Photons per thread per grab = chunk / 32. */
    uint32_t use_cuda_graph;         /* 1 -> batched launches replay a captured graph */
    uint32_t record_photon_fates;    /* 1 -> keep a per-photon fate/bounce/time record (diagnostics) */
    uint32_t generation_pass;        /* batched FP32 form: 0 or 1 -> the photons of a batch of at least 2^24
                                        photons are made by a separate generation kernel into a photon
                                        store, in waves of up to 2^28 photons, and read by the transport
                                        kernel (smaller batches generate inside the transport loop);
                                        2 -> always inside the transport loop;
                                        3 -> always the separate generation kernel, whatever the size */
    uint32_t wave_photons;           /* most photons in one generation-pass wave, rounded up to a multiple of
                                        32 (at most 2^28); 0 -> the largest of 2^28, 2^27, 2^26 whose photon
                                        stores (64 B per photon, one per wave in flight, up to four) fit in
                                        half of the free device memory, else 2^26. Smaller waves give a
                                        small batch several waves. */
    uint32_t reserved[5];
} g4b_config;

/* --- Scene (analytic boxes) ------------------------------------------------
 * The reference exports triangle meshes for OptiX (Scene.hpp:94-120,
 * OptiXTransportHost.cpp:1118-1336). B200 has no RT cores, so volumes are
 * axis-aligned boxes intersected analytically; materials, surfaces, skin and
 * border bindings keep the reference's meaning (Scene.hpp:61-126). */

/* PropertyTable (Scene.hpp:61-67): count == 0 means the property is absent. */
typedef struct g4b_property {
    const float* energy_ev;
    const float* values;
    uint32_t count;
    uint32_t reserved;
} g4b_property;

/* Material (Scene.hpp:69-76) plus an optional Rayleigh scattering length. */
typedef struct g4b_material {
    g4b_property rindex;
    float rindex_max; /* max of rindex values; 0 -> computed from the table */
    uint32_t reserved;
    g4b_property group_velocity_mm_per_ns;
    g4b_property abs_length_mm;
    g4b_property rayleigh_length_mm; /* not in the reference's GPU path; count == 0 -> off */
    g4b_property scintillation_spectrum[3];
} g4b_material;

/* SurfaceType / SurfaceModel / SurfaceFinish (Scene.hpp:15-28). */
enum { G4B_SURFACE_DIELECTRIC_DIELECTRIC = 0, G4B_SURFACE_DIELECTRIC_METAL = 1 };
enum { G4B_MODEL_GLISUR = 0, G4B_MODEL_UNIFIED = 1 };
enum { G4B_FINISH_POLISHED = 0, G4B_FINISH_GROUND = 1 };

/* Surface (Scene.hpp:78-92). */
typedef struct g4b_surface {
    uint8_t type;
    uint8_t model;
    uint8_t finish;
    uint8_t reserved0;
    float model_value; /* glisur polish or unified sigma_alpha */
    g4b_property reflectivity;
    g4b_property efficiency;
    g4b_property transmittance;
    g4b_property rindex;
    g4b_property specular_lobe;
    g4b_property specular_spike;
    g4b_property backscatter;
    g4b_property surface_roughness;
} g4b_surface;

/* Volume (Scene.hpp:107-120) with an axis-aligned box in world coordinates
 * in place of a mesh + transform. */
typedef struct g4b_volume {
    uint32_t volume_id;
    uint32_t material_id;
    uint32_t parent_volume_id; /* G4B_INVALID_ID for the world */
    uint32_t skin_surface_id;  /* G4B_INVALID_ID if none */
    uint32_t sensor_id;        /* G4B_INVALID_ID if not a sensor */
    uint32_t reserved;
    float center_mm[3];
    float half_size_mm[3];
} g4b_volume;

/* SurfaceBinding (Scene.hpp:122-126): a border surface from -> to. */
typedef struct g4b_surface_binding {
    uint32_t from_volume_id;
    uint32_t to_volume_id;
    uint32_t surface_id;
} g4b_surface_binding;

typedef struct g4b_scene {
    const g4b_material* materials;
    uint32_t material_count;
    uint32_t surface_count;
    const g4b_surface* surfaces;
    const g4b_volume* volumes;
    uint32_t volume_count;
    uint32_t binding_count;
    const g4b_surface_binding* bindings;
    uint32_t world_volume_id;
    uint32_t reserved;
} g4b_scene;

/* Output of g4b_complete (PhotonTransportOutput, PhotonTransport.hpp:152-157),
 * in caller-owned buffers. */
typedef struct g4b_output {
    g4b_photon_detection* detections; /* [detection_capacity] */
    uint64_t detection_capacity;
    uint64_t detection_count; /* out */
    g4b_event_statistics* event_statistics; /* [event_capacity] */
    uint32_t event_capacity;
    uint32_t event_count; /* out */
    g4b_statistics statistics;   /* out */
    g4b_performance performance; /* out */
} g4b_output;

typedef struct g4b_handle g4b_handle;

/* OptiXTransportHost::OptiXTransportHost(PhotonTransportConfig)
 * (OptiXTransportHost.hpp:12, OptiXTransportHost.cpp:440-478): binds the
 * device, creates the transport stream and pinned staging. */
int g4b_create(const g4b_config* config, g4b_handle** out_handle);

/* OptiXTransportHost::~OptiXTransportHost (OptiXTransportHost.cpp:480-509). */
int g4b_destroy(g4b_handle* handle);

/* Message of the last failure on this handle, or of the last handle-less
 * call on this thread when handle is NULL. Never NULL. */
const char* g4b_last_error(const g4b_handle* handle);

/* OptiXTransportHost::PrepareScene (OptiXTransportHost.cpp:511-519,
 * 1206-1339): validates and uploads the scene. Unlike the reference, which
 * keys the rebuild on the Scene's address, every call rebuilds; calling it
 * with a batch pending is G4B_ERR_LOGIC (:514-516). */
int g4b_set_scene(g4b_handle* handle, const g4b_scene* scene);

/* OptiXTransportHost::EnqueueEmissions (OptiXTransportHost.cpp:521-777):
 * validates the batch (:574-605,643-666), copies it into pinned staging and
 * onto the device, launches the transport, and queues the metadata copy
 * back. One batch may be pending at a time (:523-525). */
int g4b_enqueue(g4b_handle* handle, const g4b_optical_emission* emissions, uint32_t emission_count,
                const uint32_t* event_ids, uint32_t event_count, const uint32_t* emission_event_indices);

/* Re-runs the transport of the batch most recently passed to g4b_enqueue on
 * the copy already resident in device memory (no host-to-device copy) and
 * makes it the pending batch. Used to time the device path alone. */
int g4b_relaunch(g4b_handle* handle);

/* Sizes of the pending batch's output: waits for the device metadata, then
 * reports how many detections and events g4b_complete will return. */
int g4b_query_oldest(g4b_handle* handle, uint64_t* detection_count, uint32_t* event_count);

/* Without waiting: *ready = 1 once the pending batch's transport and metadata
 * copy have finished on the device (g4b_query_oldest and g4b_complete will then
 * not block on the GPU), else 0. No counterpart in the reference, whose
 * CompleteOldestBatch only blocks; the batch scheduler (g4b_scheduler.h) polls
 * it to keep collecting submissions while a batch runs. */
int g4b_poll_oldest(g4b_handle* handle, int* ready);

/* OptiXTransportHost::CompleteOldestBatch (OptiXTransportHost.cpp:779-883):
 * waits for the pending batch, copies the compacted hits back and fills
 * *output. If output->detection_capacity or event_capacity is too small it
 * returns G4B_ERR_CAPACITY with the needed counts and keeps the batch.
 * With output->detections == NULL and detection_capacity == 0 it returns the
 * counts and statistics only and leaves the hits in device memory. */
int g4b_complete(g4b_handle* handle, g4b_output* output);

/* The cudaStream_t the handle launches on (for CUDA-event timing). */
int g4b_get_stream(g4b_handle* handle, void** stream);

/* Per-photon record of the last completed batch when record_photon_fates was
 * set: fate[i] = outcome | (bounces << 3) for flattened photon i (outcome:
 * 1 detected, 2 absorbed, 3 escaped, 4 truncated, 5 invalid), time_ns[i] the
 * global time at the end of the history. Either pointer may be NULL. */
int g4b_photon_fates(g4b_handle* handle, uint32_t* fate, double* time_ns, uint64_t capacity, uint64_t* count);

/* Launch-shape autotuner: times the staged batch (the last one passed to
 * g4b_enqueue, which must have completed) under every candidate
 * block size x blocks per SM x queue chunk size, keeps the fastest in the
 * handle and reports it. Candidate lists may be NULL for the built-in sweep. */
typedef struct g4b_tune_result {
    uint32_t block_size;
    uint32_t blocks_per_sm;
    uint32_t chunk_photons;
    uint32_t candidates_tried;
    double best_ms;
    double worst_ms;
} g4b_tune_result;
int g4b_autotune(g4b_handle* handle, const uint32_t* block_sizes, uint32_t n_block_sizes,
                 const uint32_t* chunk_sizes, uint32_t n_chunk_sizes, uint32_t repeats,
                 g4b_tune_result* result);

/* --- Gradients (no counterpart in the reference) ---------------------------
 * Derivatives of the detected count N and of the mean arrival time of the
 * detected photons with respect to four parameters, for the batch last
 * completed on this handle (same gensteps, same seed): a refractive index
 * (of one material, constant RINDEX table), an absorption length (one
 * material), a reflectivity (one surface) and the scintillation decay time
 * (all scintillation gensteps). Every photon of the batch is regenerated and
 * re-transported from its RNG counters with forward-mode dual numbers
 * (pathwise derivatives through the step loop) while the score terms
 * d log p / d theta of its discrete choices (surface classification, survival
 * of bulk absorption, Fresnel choices at surfaces) accumulate. For the
 * refractive index, a Fresnel choice at a boundary without a surface uses the
 * measure-valued form instead of a score: the branch not taken is transported
 * to its end with draws of its own, and the difference of the two outcomes is
 * weighted by dT/dn (the score dT/T has unbounded variance near the critical
 * angle). The index derivative also carries the boundary term of the edges
 * of the volumes' boxes: where a change of n moves a ray across the edge
 * between two faces of the box it leaves (a ray refracted into a thin
 * coupling layer reaching the layer's side face instead of the sensor), the
 * photon's fate jumps. Steps that leave their box within a window h of such
 * an edge weight the difference of the outcomes through the two faces (the
 * other one transported as a branch with the photon's own draws) by the
 * edge's speed over 2h, with h = edge_band_mm: a bias of the order of the
 * window, a variance growing as it shrinks. edge_index_window > 0 widens the
 * window of fast edges (rays refracted close to the critical angle) to the
 * distance they move while n changes by +-edge_index_window: weights bounded
 * by 1 / (2 edge_index_window) and a lower variance, but a bias that grows
 * with it (about +1 % at 0.00025 on the detector of the benchmark, where the
 * band alone of 0.1 mm is within 1.4 % of a finite difference). Nothing of
 * the forward trajectories
 * is stored. FP32 replay for an FP32 handle with FP64 accumulation. Batches
 * the plain form regrouped by event are not supported. */
typedef struct g4b_gradient_request {
    uint32_t rindex_material_id;      /* G4B_INVALID_ID: no index derivative */
    uint32_t abs_length_material_id;  /* G4B_INVALID_ID: none */
    uint32_t reflectivity_surface_id; /* G4B_INVALID_ID: none */
    float edge_band_mm;               /* least half width of the edge-term window; 0: 0.1 mm; < 0: no edge term */
    float edge_index_window;          /* > 0: the window's half width in n for fast edges; else none */
    uint32_t reserved[3];
} g4b_gradient_request;

/* Parameter order in the arrays: 0 refractive index, 1 absorption length
 * (per mm), 2 reflectivity, 3 scintillation decay time (per ns). */
typedef struct g4b_gradient_result {
    uint64_t detected;
    uint64_t replay_mismatches; /* |replayed detections - the batch's detections|; 0 expected */
    double mean_time_ns;
    double d_detected[4];
    double d_mean_time_ns[4];
    double kernel_ms;
} g4b_gradient_result;

int g4b_gradients(g4b_handle* handle, const g4b_gradient_request* request, g4b_gradient_result* result);

/* --- Device-evaluated boundary and math kernels ---------------------------
 * Run the transport's own device functions on caller inputs, so the boundary
 * unit cases of test/TestOpticalBoundaryPhysics.cxx:37-101 can be checked on
 * the GPU path itself. Host buffers in and out; precision picks FP32/FP64. */

/* BoundaryPhysics::ComputeFresnel (src/optical/optix/OptiXBoundaryPhysics.cuh:130-186).
 * Inputs are n rows of direction[3], polarization[3], normal[3], n_from, n_to;
 * each output row is reflected_direction[3], transmitted_direction[3],
 * reflected_polarization[3], transmitted_polarization[3], transmittance, tir
 * (14 doubles). */
int g4b_eval_fresnel(int device, uint32_t precision, uint32_t n, const double* direction,
                     const double* polarization, const double* normal, const double* index_from,
                     const double* index_to, double* out);

/* BoundaryPhysics::SampleLambertian (OptiXBoundaryPhysics.cuh:111-128):
 * normal[3], radial sample, azimuth sample -> direction[3]. */
int g4b_eval_lambertian(int device, uint32_t precision, uint32_t n, const double* normal,
                        const double* radial_sample, const double* azimuth_sample, double* out);

/* The engine's own log / exp / sin+cos-of-turns (float), for bit-level
 * comparison with the CPU oracle. kind: 0 log, 1 exp, 2 sincos(2*pi*x)
 * (out holds sin then cos: 2n floats). */
int g4b_eval_math(int device, uint32_t kind, uint32_t n, const float* x, float* out);

/* The counter RNG draw Uniform(seed, key, bounce, process, draw)
 * (src/optical/optix/OptiXTransportDevice.cu:254-286), evaluated on the device. */
int g4b_eval_uniform(int device, uint32_t n, uint64_t seed, const uint64_t* photon_key,
                     const uint32_t* bounce, const uint32_t* process, const uint32_t* draw, float* out);

/* Page-locked host memory for output buffers: g4b_complete copies detections
 * straight into such a buffer instead of through the engine's staging. */
int g4b_host_alloc(size_t bytes, void** pointer);
int g4b_host_free(void* pointer);

/* Orders device-resident detection records by a unique per-record slot key
 * and allocates no device memory. No counterpart in the reference: it is the
 * ranking step of the ordered completion (the order the reference's
 * cub::DeviceSelect::Flagged compaction gives,
 * src/optical/optix/OptiXHitCompaction.cu:23-30), offered on its own for
 * callers that cannot allocate: a caller whose device memory is all held by
 * its own pool, or one on a path where cudaMalloc/cudaFree would stall other
 * streams by synchronizing the device.
 *
 * Record i of `unordered` is written to row r of `ordered`, r being the number
 * of keys smaller than slots[i]; with the flattened photon index of a launch
 * as key this restores the reference's order. All pointers are device
 * memory on the current device, the record pointers 16-byte aligned, and
 * `unordered` and `ordered` must not overlap. Keys must be unique and below
 * slot_limit, and slot_limit at most G4B_ORDER_STATIC_MAX_SLOTS
 * (G4B_ERR_OVERFLOW otherwise). A key out of range or repeated gives
 * G4B_ERR_INVALID_ARGUMENT and leaves `ordered` undefined.
 *
 * Scratch is one 4 MiB array compiled into the library (bitmap, prefix and
 * block sums); each call zeroes the bitmap and its status word on `stream`
 * before use. The first call on a device looks the array up with
 * cudaGetSymbolAddress, which may load the library's kernels there: make that
 * call before any stream capture starts on the device. The first call on a
 * host thread reserves a 256-byte host buffer for error messages; later calls
 * allocate nothing. The call returns once `stream` has finished the
 * ordering. Calls that overlap in time on one device share the scratch array
 * and race: callers on several host threads must serialize them. */
#define G4B_ORDER_STATIC_MAX_SLOTS 16777216u
int g4b_order_detections_static(const g4b_photon_detection* unordered, const uint32_t* slots, uint64_t count,
                                uint32_t slot_limit, g4b_photon_detection* ordered, void* stream);

/* Version of this library (G4B_ABI_VERSION). */
uint32_t g4b_abi_version(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* G4B_H */
