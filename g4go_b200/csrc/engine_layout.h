// engine_layout.h - data layout shared by the engine's host code and kernels.
//
// The analytic scene is packed on the host into one blob that every CTA
// copies into shared memory at launch: boxes, per-volume metadata, a dense
// (from, to) -> surface table, materials, surfaces, and one pool of property
// floats. Launch parameters travel by value in the kernel's constant bank.
#pragma once

#include <cstddef>
#include <cstdint>

namespace g4b {

constexpr std::uint32_t kInvalidID = 0xffffffffU;
constexpr std::uint32_t kMaxVolumes = 64;
constexpr std::uint32_t kMaxMaterials = 16;
constexpr std::uint32_t kMaxSurfaces = 16;
constexpr std::uint32_t kMaxPoolFloats = 6144;
constexpr std::uint8_t kNoSurface = 0xff;
constexpr std::uint8_t kNoVolume = 0xff;

// A property table in the pool: energies at [offset, offset + count), values
// at [offset + count, offset + 2 * count). count == 0: absent.
struct PackedProperty {
    std::uint16_t offset;
    std::uint16_t count;
    std::uint16_t constant;  // PropertyTable::Constant (src/optical/Scene.cpp:184-188)
    std::uint16_t reserved;
};

struct PackedMaterial {
    PackedProperty rindex;
    PackedProperty groupVelocity;
    PackedProperty absLength;
    PackedProperty rayleighLength;
    PackedProperty spectrum[3];  // energies + normalised CDF
    float rindexMax;
    std::uint32_t reserved;
};

struct PackedSurface {
    std::uint8_t type;
    std::uint8_t model;
    std::uint8_t finish;
    std::uint8_t reserved0;
    float modelValue;
    PackedProperty reflectivity;
    PackedProperty efficiency;
    PackedProperty transmittance;
    PackedProperty rindex;
    PackedProperty specularLobe;
    PackedProperty specularSpike;
    PackedProperty backscatter;
    PackedProperty roughness;
};

// Box as two float4 (lo.xyz, hi.xyz; w unused) for 16-byte shared loads.
struct PackedBox {
    float lo[4];
    float hi[4];
};

struct PackedVolume {
    std::uint8_t parent;          // dense index or kNoVolume
    std::uint8_t material;
    std::uint8_t coincidentFaces; // bit f: face f = 2*axis + side touches another volume
    std::uint8_t mayCoincide;     // Volume::mayHaveCoincidentBoundary
    std::uint32_t sensorID;       // kInvalidID if not a sensor
    // Boxes a ray starting inside this volume can cross first: itself and its
    // daughters (bit b = volume b), in ascending order.
    unsigned long long traceMask;
    // Boxes whose faces can coincide with this volume's: itself and every
    // volume it shares a coincident face with.
    unsigned long long neighbourMask;
};

struct PackedScene {
    std::uint32_t volumeCount;
    std::uint32_t materialCount;
    std::uint32_t surfaceCount;
    std::uint32_t poolFloats;
    std::uint32_t world;
    std::uint32_t hasRayleigh;
    std::uint32_t reserved[2];
    PackedBox boxes[kMaxVolumes];
    PackedVolume volumes[kMaxVolumes];
    PackedMaterial materials[kMaxMaterials];
    PackedSurface surfaces[kMaxSurfaces];
    std::uint8_t surfaceTable[kMaxVolumes * kMaxVolumes];  // FindSurfaceID(from, to) or kNoSurface
    // followed by poolFloats floats
};

static_assert(sizeof(PackedScene) % 16 == 0, "scene blob must stay 16-byte aligned");

// Per-warp photon queue in shared memory (batched form): 32 generated photons,
// structure of arrays so that lanes reading different entries hit different
// banks. Fields: position, direction, polarization (3 each), energy in the
// transport type; time in double; eventID, photonID, volume, event index, slot.
constexpr std::uint32_t kQueueBytesFP32 = 10U * 32U * 4U + 32U * 8U + 5U * 32U * 4U;  // 2176
constexpr std::uint32_t kQueueBytesFP64 = 10U * 32U * 8U + 32U * 8U + 5U * 32U * 4U;  // 3456
// Per-warp ring of photons stopped at a Fresnel boundary (pending) or done
// with it (ready): 12 real columns, FP64 time, 7 u32 columns, 40 entries (a
// batch of 32 plus room to keep parking while ready photons drain; with 40,
// three 256-thread blocks use at most 196 KB of shared memory per SM, which
// leaves the L1 data cache 60 KB instead of 28 KB).
constexpr std::uint32_t kFresnelRingEntries = 40;
constexpr std::uint32_t kRingBytesFP32 = kFresnelRingEntries * (12U * 4U + 8U + 7U * 4U);  // 3360
constexpr std::uint32_t kRingBytesFP64 = kFresnelRingEntries * (12U * 8U + 8U + 7U * 4U);  // 5280
// The ring of the form with a generation pass (no photon queue in shared
// memory): 64 entries, more than one step can ever need (at most 31 ready or
// pending entries between steps, plus 32 parking), so that form has no
// full-ring fallback; three blocks use 191 KB of shared memory per SM.
constexpr std::uint32_t kFresnelRingEntriesPass = 64;
constexpr std::uint32_t kRingBytesFP32Pass = kFresnelRingEntriesPass * (12U * 4U + 8U + 7U * 4U);  // 5376
// Per-thread event counters and bounce total of the batched form, kept in
// shared memory instead of registers (they change once per photon).
constexpr std::uint32_t kLaneTallyBytes = 40;

// Per-event counters (DeviceEventTransportStats, OptiXDeviceData.cuh:159-167),
// padded to 64 bytes.
struct EventCounters {
    unsigned long long detected;
    unsigned long long absorbed;
    unsigned long long escaped;
    unsigned long long truncated;
    unsigned long long maxBounce;
    unsigned long long invalid;
    unsigned long long zeroStep;
    unsigned long long reserved;
};

// Batch-wide counters that have no per-event breakdown, plus queue state.
// With a generation pass each wave counts its hit rows separately (its own
// region of the hit buffer); hitCount is then their sum, and maxWaveHits the
// largest, which tells whether a region overflowed.
struct RunCounters {
    unsigned long long totalBounces;
    unsigned long long coincidentTraces;
    unsigned long long coincidentHits;
    unsigned long long hitCount;
    unsigned int workTicket;
    unsigned int reserved0;
    unsigned long long maxWaveHits;
    unsigned long long reserved[2];
};

// Sums of the gradient replay over the detected photons, FP64. Parameter j:
// 0 refractive index, 1 absorption length, 2 reflectivity, 3 decay time.
struct GradientSums {
    double detected;       // N
    double time;           // sum of arrival times of the detected photons
    double score[4];       // dN/dtheta_j: score, pathwise and alternate-branch terms
    double timeScore[4];   // d(sum of arrival times)/dtheta_j
};

// Compacted hits, structure of arrays, `capacity` rows each.
struct HitColumns {
    float* positionX;
    float* positionY;
    float* positionZ;
    float* time;
    float* directionX;
    float* directionY;
    float* directionZ;
    float* energy;
    std::uint32_t* eventID;
    std::uint32_t* photonID;
    std::uint32_t* sensorID;
    std::uint32_t* slot;  // flattened photon index: restores the reference's order on the host
    unsigned long long capacity;
};

// Photons of one wave of the batched FP32 form, made by the generation pass
// and read by the transport: one column per field, row = slot - photonBegin.
// eventIndex == kInvalidID marks a photon that failed the validity test.
struct PhotonStore {
    float* position[3];
    float* direction[3];
    float* polarization[3];
    float* energy;
    double* time;
    std::uint32_t* eventID;
    std::uint32_t* photonID;
    std::uint32_t* volume;
    std::uint32_t* eventIndex;
};
constexpr std::uint32_t kPhotonStoreBytes{10U * 4U + 8U + 4U * 4U};  // per photon: 64
constexpr std::uint32_t kPhotonStoreWave{1U << 28};                  // most photons in one generation wave
constexpr std::uint32_t kPhotonStoreWaveMin{1U << 26};               // smallest wave the memory sizing picks
constexpr std::uint32_t kWaveSlots{4};                                // generation-pass waves in flight at once

// A photon of the generation pass's transport parked in the wave's queue,
// which the parked-photon form of the pass kernel transports: the state
// StepPhoton continues from. Parked are the
// photons that leave their volume the way the reference lets them (a trace
// that has to search the whole scene; some then reflect totally at every step
// for thousands of steps) and any history that reaches kDeferBounces bounces.
// In the transport kernel such a photon would advance one step per Fresnel
// ring completion and keep a whole block resident for one warp while the next
// wave waits for its SMs.
struct DeferredPhoton {
    float position[3];
    float direction[3];
    float polarization[3];
    float energy;
    double time;
    std::uint32_t volume;
    std::uint32_t bounce;
    std::uint32_t eventID;
    std::uint32_t photonID;
    std::uint32_t eventIndex;
    std::uint32_t slot;
};
static_assert(sizeof(DeferredPhoton) == 72, "deferred photon layout");

struct DeferredQueue {
    DeferredPhoton* photons;  // nullptr: no deferral
    unsigned int* count;      // photons parked; may exceed capacity (those beyond stay in their lane)
    std::uint32_t capacity;
    std::uint32_t reserved;
};
constexpr std::uint32_t kDeferBounces{256};
constexpr std::uint32_t kDeferredMinCapacity{1U << 19};  // per wave in flight (38 MB), or wave / 64 if more

struct LaunchParams {
    const float4* emissions;               // [emissionCount] 128-byte gensteps as 8 float4 each
    const std::uint32_t* emissionOffsets;  // [emissionCount + 1] exclusive prefix of photon counts
    const std::uint32_t* emissionEventIndices;
    const std::uint32_t* slotBase;         // optional [emissionCount]: flattened slot of each emission's first photon
                                           // when the launch order differs from the batch order (plain form)
    const PackedScene* scene;              // device copy of the blob
    std::uint32_t sceneBytes;
    std::uint32_t emissionCount;
    std::uint32_t eventCount;
    std::uint32_t photonBegin;             // first flattened photon of this launch
    std::uint32_t photonEnd;               // one past the last
    std::uint32_t emissionBegin;           // plain form: first emission of the event
    std::uint32_t emissionEnd;
    std::uint32_t chunk;                   // batched form: photons per queue take (multiple of 32)
    unsigned long long seed;
    std::uint32_t maxBounce;
    float epsilon;
    EventCounters* events;
    RunCounters* run;
    HitColumns hits;
    unsigned long long* hitCounter;        // allocator of hit rows: &run->hitCount, or a wave's own counter
    std::uint32_t* photonFate;             // optional [photons]
    double* photonTime;                    // optional [photons]
    PhotonStore store;                     // batched FP32 form with a generation pass
    unsigned int* workTicket;              // batched form: next unclaimed photon of the launch
    DeferredQueue deferred;                // generation pass: where long histories are parked
};

}  // namespace g4b
