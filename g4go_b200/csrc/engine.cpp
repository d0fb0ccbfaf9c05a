// engine.cpp - the C ABI of the B200 optical-photon engine (include/g4b.h).
//
// Host side of the transport: the counterpart of OptiXTransportHost
// (src/optical/optix/OptiXTransportHost.cpp). It validates and packs the
// analytic scene, validates and stages each batch in pinned memory, launches
// the transport (a replayed CUDA graph for the batched form, one launch per
// event for the plain form), orders the compacted hits back into the
// reference's flattened-photon order and assembles the per-event and batch
// statistics. Errors are C++ exceptions inside and status codes at the ABI.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/g4b.h"
#include "engine_layout.h"
#include "kernels.h"

static_assert(sizeof(g4b_optical_emission) == 128, "genstep record must match OpticalEmission (128 bytes)");
static_assert(sizeof(g4b_photon_detection) == 48, "detection record must match PhotonDetection (48 bytes)");

namespace {

using g4b::EventCounters;
using g4b::HitColumns;
using g4b::kInvalidID;
using g4b::LaunchParams;
using g4b::kWaveSlots;
using g4b::PackedProperty;
using g4b::PackedScene;
using g4b::RunCounters;

thread_local std::string gHandlelessError;

struct EngineError : std::runtime_error {
    int code;
    EngineError(int status, const std::string& message) : std::runtime_error(message), code(status) {}
};

[[noreturn]] void Throw(int status, const std::string& message) { throw EngineError(status, message); }

void Check(cudaError_t error, const char* operation) {
    if (error != cudaSuccess) {
        Throw(G4B_ERR_CUDA, std::string(operation) + " failed: " + cudaGetErrorString(error));
    }
}

// Device allocation that only grows.
struct DeviceBuffer {
    void* pointer{nullptr};
    std::size_t bytes{0};
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { Release(); }
    void Release() {
        if (pointer != nullptr) {
            cudaFree(pointer);
            pointer = nullptr;
            bytes = 0;
        }
    }
    void Ensure(std::size_t needed, const char* what) {
        needed = std::max<std::size_t>(needed, 256);
        if (needed <= bytes) {
            return;
        }
        Release();
        Check(cudaMalloc(&pointer, needed), what);
        bytes = needed;
    }
    template<class T>
    T* As() const {
        return static_cast<T*>(pointer);
    }
};

// Page-locked host allocation that only grows.
struct PinnedBuffer {
    void* pointer{nullptr};
    std::size_t bytes{0};
    PinnedBuffer() = default;
    PinnedBuffer(const PinnedBuffer&) = delete;
    PinnedBuffer& operator=(const PinnedBuffer&) = delete;
    ~PinnedBuffer() { Release(); }
    void Release() {
        if (pointer != nullptr) {
            cudaFreeHost(pointer);
            pointer = nullptr;
            bytes = 0;
        }
    }
    void Ensure(std::size_t needed, const char* what) {
        needed = std::max<std::size_t>(needed, 64);
        if (needed <= bytes) {
            return;
        }
        Release();
        Check(cudaMallocHost(&pointer, needed), what);
        bytes = needed;
    }
    template<class T>
    T* As() const {
        return static_cast<T*>(pointer);
    }
};

struct TimerPair {
    cudaEvent_t start{nullptr};
    cudaEvent_t stop{nullptr};
    void Create() {
        Check(cudaEventCreate(&start), "cudaEventCreate");
        Check(cudaEventCreate(&stop), "cudaEventCreate");
    }
    void Destroy() {
        if (start != nullptr) cudaEventDestroy(start);
        if (stop != nullptr) cudaEventDestroy(stop);
        start = stop = nullptr;
    }
    double Milliseconds() const {
        float ms{0.0F};
        if (cudaEventElapsedTime(&ms, start, stop) != cudaSuccess) {
            return 0.0;
        }
        return static_cast<double>(ms);
    }
};

constexpr int kHitColumns = 12;

std::uint32_t FieldBit(int field) { return 1U << static_cast<unsigned>(field); }

std::uint32_t TerminalFields() {
    return FieldBit(G4B_FIELD_DETECTED) | FieldBit(G4B_FIELD_ABSORBED) | FieldBit(G4B_FIELD_ESCAPED) |
           FieldBit(G4B_FIELD_TRUNCATED) | FieldBit(G4B_FIELD_MAX_BOUNCE) | FieldBit(G4B_FIELD_INVALID_STATE) |
           FieldBit(G4B_FIELD_ZERO_STEP);
}

}  // namespace

struct g4b_handle {
    g4b_config config{};
    int device{0};
    int smCount{0};
    cudaStream_t stream{nullptr};
    std::string error;

    // Scene.
    bool hasScene{false};
    std::vector<unsigned char> sceneBlob;
    DeviceBuffer dScene;
    std::uint32_t sceneBytes{0};
    std::unordered_map<std::uint32_t, std::uint32_t> volumeIndex;
    std::uint32_t materialCount{0};

    // Staging and device buffers.
    PinnedBuffer hEmissions, hOffsets, hEventIndices, hSlotBase, hEvents, hRun, hDetections;
    DeviceBuffer dEmissions, dOffsets, dEventIndices, dSlotBase, dEvents, dRun;
    DeviceBuffer dHits[kHitColumns];
    std::uint64_t hitCapacity{0};
    DeviceBuffer dBitmap, dPrefix, dBlockSums, dDetections, dFate, dFateTime, dGradient;
    // kWaveSlots photon stores and work tickets of the generation pass: wave k
    // uses slot k % kWaveSlots, and its transport and parked-photon launch run
    // on transport stream k % kWaveSlots (the handle's stream, then
    // waveStreams). Up to kWaveSlots waves are in flight, so a wave's longest
    // photon histories - serial chains of thousands of steps - overlap the
    // next waves' transports instead of holding up the GPU. The waves' hit
    // orderings and row copies run in wave order on orderStream, so that a
    // transport stream never waits for an ordering: those kernels get SMs
    // only when a transport's blocks leave, and a transport queued behind one
    // would start only after the previous wave's transport had drained.
    DeviceBuffer dStore;
    DeviceBuffer dTickets;
    DeviceBuffer dDeferred;        // per slot: deferredCapacity parked photons
    std::uint32_t deferredCapacity{0};
    std::uint64_t waveLimit{0};    // most photons per wave for the staged batch (set by SizeWaves)
    DeviceBuffer dDeferredCounts;  // per slot: how many were parked
    cudaStream_t generationStream{nullptr};
    cudaStream_t waveStreams[kWaveSlots - 1]{};
    cudaEvent_t zeroedEvent{nullptr};
    cudaEvent_t generatedEvent[kWaveSlots]{};
    cudaEvent_t storeFreeEvent[kWaveSlots]{};
    cudaEvent_t parkedEvent[kWaveSlots]{};  // a wave's parked photons transported: its hits can be ordered
    cudaStream_t orderStream{nullptr};
    cudaEvent_t orderJoinEvent{nullptr};  // the ordering stream's last work, joined into the handle's stream
    cudaEvent_t joinEvents[kWaveSlots - 1]{};  // each wave stream's last work, joined into the handle's stream
    cudaGraphExec_t wavesExec{nullptr};  // the generation-pass waves of the last batch, captured
    // Per-wave hits and ordering of the generation-pass form: wave k writes its
    // hits to rows [k * waveRegionRows, (k + 1) * waveRegionRows) of the hit
    // buffer, counting them in dWaveCounts[k]; after its transport they are
    // ordered into dDetections from row dWaveRows[k] on (the sum of the earlier
    // waves' counts, chained on the device), dWaveRows[k + 1] copied to
    // hWaveRows and an event recorded, so g4b_complete can copy each wave's
    // detections to the host while later waves run.
    DeviceBuffer dWaveCounts;
    DeviceBuffer dWaveRows;
    PinnedBuffer hWaveRows;
    std::uint64_t waveRegionRows{0};
    std::vector<cudaEvent_t> waveEvents;
    std::uint64_t pendingWaves{0};  // waves of the pending batch ordered that way (0: none)
    cudaStream_t copyStream{nullptr};

    // The staged batch (kept for g4b_relaunch) and the pending one.
    bool hasStaged{false};
    bool busy{false};
    bool metadataReady{false};
    std::uint32_t emissionCount{0};
    std::uint32_t eventCount{0};
    std::uint64_t photonCount{0};
    std::vector<std::uint32_t> eventIDs;
    std::vector<std::uint64_t> captured;
    std::vector<std::uint8_t> eventHasEmission;
    bool usesSlotBase{false};
    struct PlainEvent {
        std::uint32_t emissionBegin, emissionEnd, photonBegin, photonEnd;
    };
    std::vector<PlainEvent> plainEvents;
    std::uint64_t hostToDeviceBytes{0};
    bool fatesValid{false};

    // Launch shape.
    std::uint32_t blockSize{256};
    std::uint32_t blocksPerSM{0};
    std::uint32_t chunk{512};
    bool chunkAdaptive{false};  // chunk_photons left at 0 and no autotune: shrink the chunk for small batches

    // Graph for the batched form: [ZeroCounters] -> [TransportBatched].
    cudaGraph_t graph{nullptr};
    cudaGraphExec_t graphExec{nullptr};
    cudaGraphNode_t zeroNode{nullptr};
    cudaGraphNode_t transportNode{nullptr};
    int graphPrecision{-1};

    TimerPair hostToDeviceTimer, memsetTimer, kernelTimer, metadataTimer, hitsTimer;
    cudaEvent_t metadataReadyEvent{nullptr};
    std::chrono::steady_clock::time_point startedAt{};
    std::uint64_t launchCount{0};
    std::uint64_t batchLaunches{0};
};

namespace {

int Precision(const g4b_handle& h) { return h.config.precision == G4B_PRECISION_FP64 ? g4b::kFP64 : g4b::kFP32; }
int Form(const g4b_handle& h) { return h.config.launch_form == G4B_FORM_PLAIN ? g4b::kPlain : g4b::kBatched; }

// The batched FP32 form makes the photons of a large batch in a separate
// generation pass (config 0 or 1) unless the configuration asks for
// generation inside the transport loop (2). A batch below
// kGenerationPassMinPhotons keeps generation in the loop: a single wave has
// nothing to overlap its generation with, and the transport of a small batch
// is bound by its tail, so the pass only adds latency there. Config 3 takes
// the pass for a batch of any size (the same kernels as a large batch's).
constexpr std::uint64_t kGenerationPassMinPhotons{1ULL << 24};
// Blocks of a wave's launch over its parked photons.
constexpr unsigned kParkedBlocks{16U};
// Default half width of the window in which the gradient replay estimates the
// boundary term of box edges (edge_band_mm == 0).
constexpr float kDefaultEdgeBandMm{0.1F};
bool UsesGenerationPass(const g4b_handle& h) {
    if (Form(h) != g4b::kBatched || Precision(h) != g4b::kFP32 || h.photonCount == 0U) {
        return false;
    }
    if (h.config.generation_pass == 3U) {
        return true;
    }
    return h.config.generation_pass != 2U && h.photonCount >= kGenerationPassMinPhotons;
}

// The kernel variant of a form: with the coincidence counters only when
// performance diagnostics are enabled, as the reference counts them, and for
// the batched form with a generation pass the one that reads the photon store.
int KernelOf(const g4b_handle& h, int form) {
    return form | (h.config.enable_performance_diagnostics != 0 ? g4b::kWithDiagnostics : 0) |
           (form == g4b::kBatched && UsesGenerationPass(h) ? g4b::kPregenerated : 0);
}

std::size_t SceneSharedBytes(const g4b_handle& h) {
    return (static_cast<std::size_t>(h.sceneBytes) + 15U) & ~std::size_t{15};
}

// Dynamic shared memory of a launch: the scene blob, plus one photon queue
// (not with a generation pass) and one Fresnel ring per warp and one tally
// per lane for the batched form.
std::size_t SharedBytes(const g4b_handle& h, int form, std::uint32_t blockSize) {
    std::size_t bytes{SceneSharedBytes(h)};
    if (form == g4b::kBatched) {
        const bool fp64{h.config.precision == G4B_PRECISION_FP64};
        const std::size_t queue{UsesGenerationPass(h) ? 0U : (fp64 ? g4b::kQueueBytesFP64 : g4b::kQueueBytesFP32)};
        const std::size_t ring{fp64 ? g4b::kRingBytesFP64
                                    : (UsesGenerationPass(h) ? g4b::kRingBytesFP32Pass : g4b::kRingBytesFP32)};
        bytes += (queue + ring) * (blockSize / 32U) + g4b::kLaneTallyBytes * blockSize;
    }
    return bytes;
}

std::uint32_t RoundChunk(std::uint32_t chunk) { return std::max<std::uint32_t>((chunk + 31U) / 32U * 32U, 32U); }


// --- scene packing ---------------------------------------------------------

struct PoolBuilder {
    std::vector<float> floats;
    PackedProperty Add(const g4b_property& property, const char* what) {
        PackedProperty packed{};
        if (property.count == 0) {
            return packed;
        }
        if (property.energy_ev == nullptr || property.values == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, std::string("property table ") + what + " has null arrays");
        }
        for (std::uint32_t i{1}; i < property.count; ++i) {
            if (!(property.energy_ev[i] >= property.energy_ev[i - 1])) {
                Throw(G4B_ERR_INVALID_ARGUMENT, std::string("property table ") + what + " energies must ascend");
            }
        }
        for (std::uint32_t i{}; i < property.count; ++i) {
            if (!std::isfinite(property.energy_ev[i])) {
                Throw(G4B_ERR_INVALID_ARGUMENT, std::string("property table ") + what + " has a non-finite energy");
            }
        }
        bool constant{true};
        for (std::uint32_t i{1}; i < property.count; ++i) {
            if (property.values[i] != property.values[0]) {
                constant = false;
            }
        }
        return Append(property.energy_ev, property.values, property.count, constant, what);
    }
    // Scintillation spectrum: the normalised trapezoid CDF of
    // UploadSpectrumProperty (OptiXTransportHost.cpp:371-410); a rejected
    // spectrum is absent.
    PackedProperty AddSpectrum(const g4b_property& property, const char* what) {
        PackedProperty packed{};
        if (property.count == 0 || property.energy_ev == nullptr || property.values == nullptr) {
            return packed;
        }
        const std::uint32_t count{property.count};
        std::vector<float> cdf(count, 0.0F);
        if (count == 1) {
            cdf[0] = 1.0F;
            return Append(property.energy_ev, cdf.data(), 1, false, what);
        }
        for (std::uint32_t i{1}; i < count; ++i) {
            const float energyDelta{property.energy_ev[i] - property.energy_ev[i - 1]};
            const float value0{std::max(property.values[i - 1], 0.0F)};
            const float value1{std::max(property.values[i], 0.0F)};
            if (!(energyDelta >= 0.0F) || !std::isfinite(energyDelta) || !std::isfinite(value0) ||
                !std::isfinite(value1)) {
                return packed;
            }
            cdf[i] = cdf[i - 1] + 0.5F * energyDelta * (value0 + value1);
        }
        const float integral{cdf[count - 1]};
        if (!(integral > 0.0F) || !std::isfinite(integral)) {
            return packed;
        }
        for (auto& value : cdf) {
            value /= integral;
        }
        cdf[count - 1] = 1.0F;
        return Append(property.energy_ev, cdf.data(), count, false, what);
    }
    PackedProperty Append(const float* energy, const float* values, std::uint32_t count, bool constant,
                          const char* what) {
        if (floats.size() + 2U * count > g4b::kMaxPoolFloats) {
            Throw(G4B_ERR_UNSUPPORTED, std::string("property tables exceed the shared-memory pool at ") + what);
        }
        PackedProperty packed{};
        packed.offset = static_cast<std::uint16_t>(floats.size());
        packed.count = static_cast<std::uint16_t>(count);
        packed.constant = constant ? 1U : 0U;
        floats.insert(floats.end(), energy, energy + count);
        floats.insert(floats.end(), values, values + count);
        return packed;
    }
};

// FindSurfaceID (OptiXTransportDevice.cu:218-252) evaluated once per
// (from, to) pair on the host: border binding first, then skin surfaces with
// Geant4's precedence (Scene.cpp:286-316).
std::uint32_t ResolveSurface(const std::vector<g4b_volume>& volumes, const std::vector<std::uint32_t>& parents,
                             const std::vector<std::pair<std::uint64_t, std::uint32_t>>& bindings, std::uint32_t from,
                             std::uint32_t to) {
    const std::uint64_t key{(static_cast<std::uint64_t>(from) << 32U) | to};
    const auto it{std::lower_bound(bindings.begin(), bindings.end(), std::make_pair(key, 0U))};
    if (it != bindings.end() && it->first == key) {
        return it->second;
    }
    const auto& fromVolume{volumes[from]};
    const auto& toVolume{volumes[to]};
    if (parents[to] == from) {
        if (toVolume.skin_surface_id != kInvalidID) {
            return toVolume.skin_surface_id;
        }
        return fromVolume.skin_surface_id;
    }
    if (fromVolume.skin_surface_id != kInvalidID) {
        return fromVolume.skin_surface_id;
    }
    return toVolume.skin_surface_id;
}

void BuildScene(g4b_handle& h, const g4b_scene& scene) {
    if (scene.volume_count == 0 || scene.volumes == nullptr) {
        Throw(G4B_ERR_INVALID_ARGUMENT, "scene cannot be empty");
    }
    if (scene.volume_count > g4b::kMaxVolumes) {
        Throw(G4B_ERR_UNSUPPORTED, "scene has more than 64 volumes");
    }
    if (scene.material_count > g4b::kMaxMaterials || scene.surface_count > g4b::kMaxSurfaces) {
        Throw(G4B_ERR_UNSUPPORTED, "scene has more than 16 materials or 16 surfaces");
    }
    if ((scene.material_count != 0 && scene.materials == nullptr) ||
        (scene.surface_count != 0 && scene.surfaces == nullptr) ||
        (scene.binding_count != 0 && scene.bindings == nullptr)) {
        Throw(G4B_ERR_INVALID_ARGUMENT, "scene table pointer is null");
    }
    // CreateVolumeIndices (OptiXTransportHost.cpp:1002-1019).
    std::unordered_map<std::uint32_t, std::uint32_t> index;
    std::vector<g4b_volume> volumes(scene.volumes, scene.volumes + scene.volume_count);
    for (std::uint32_t i{}; i < scene.volume_count; ++i) {
        const auto id{volumes[i].volume_id};
        if (id == kInvalidID || !index.emplace(id, i).second) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "scene volume IDs must be unique and valid");
        }
    }
    const auto map{[&](std::uint32_t id, const char* what) -> std::uint32_t {
        if (id == kInvalidID) {
            return kInvalidID;
        }
        const auto it{index.find(id)};
        if (it == index.end()) {
            Throw(G4B_ERR_INVALID_ARGUMENT, std::string("scene references an unknown ") + what + " volume ID");
        }
        return it->second;
    }};
    std::vector<std::uint32_t> parents(scene.volume_count);
    for (std::uint32_t i{}; i < scene.volume_count; ++i) {
        parents[i] = map(volumes[i].parent_volume_id, "parent");
        if (volumes[i].material_id >= scene.material_count) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "volume references an unknown material");
        }
        for (int a{}; a < 3; ++a) {
            if (!(volumes[i].half_size_mm[a] > 0.0F) || !std::isfinite(volumes[i].half_size_mm[a]) ||
                !std::isfinite(volumes[i].center_mm[a])) {
                Throw(G4B_ERR_INVALID_ARGUMENT, "volume box must have finite centre and positive half sizes");
            }
        }
    }
    if (scene.world_volume_id == kInvalidID) {
        Throw(G4B_ERR_INVALID_ARGUMENT, "scene has no world volume ID");
    }
    const std::uint32_t world{map(scene.world_volume_id, "world")};
    std::vector<std::pair<std::uint64_t, std::uint32_t>> bindings;
    for (std::uint32_t b{}; b < scene.binding_count; ++b) {
        if (scene.bindings[b].from_volume_id == kInvalidID || scene.bindings[b].to_volume_id == kInvalidID) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "scene has no boundary source or target volume ID");
        }
        const auto from{map(scene.bindings[b].from_volume_id, "boundary source")};
        const auto to{map(scene.bindings[b].to_volume_id, "boundary target")};
        bindings.emplace_back((static_cast<std::uint64_t>(from) << 32U) | to, scene.bindings[b].surface_id);
    }
    std::stable_sort(bindings.begin(), bindings.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    for (std::size_t b{1}; b < bindings.size(); ++b) {
        if (bindings[b].first == bindings[b - 1].first) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "scene has two border surfaces for one ordered volume pair");
        }
    }

    auto packed{std::make_unique<PackedScene>()};
    std::memset(packed.get(), 0, sizeof(PackedScene));
    PoolBuilder pool;
    packed->volumeCount = scene.volume_count;
    packed->materialCount = scene.material_count;
    packed->surfaceCount = scene.surface_count;
    packed->world = world;
    for (std::uint32_t m{}; m < scene.material_count; ++m) {
        const auto& source{scene.materials[m]};
        auto& material{packed->materials[m]};
        material.rindex = pool.Add(source.rindex, "RINDEX");
        float rindexMax{source.rindex_max};
        if (rindexMax == 0.0F) {
            rindexMax = 1.0F;
            if (source.rindex.count != 0) {
                rindexMax = *std::max_element(source.rindex.values, source.rindex.values + source.rindex.count);
            }
        }
        material.rindexMax = rindexMax;
        material.groupVelocity = pool.Add(source.group_velocity_mm_per_ns, "GROUPVEL");
        material.absLength = pool.Add(source.abs_length_mm, "ABSLENGTH");
        material.rayleighLength = pool.Add(source.rayleigh_length_mm, "RAYLEIGH");
        if (material.rayleighLength.count != 0) {
            packed->hasRayleigh = 1;
        }
        for (int c{}; c < 3; ++c) {
            material.spectrum[c] = pool.AddSpectrum(source.scintillation_spectrum[c], "SCINTILLATIONCOMPONENT");
        }
    }
    for (std::uint32_t s{}; s < scene.surface_count; ++s) {
        const auto& source{scene.surfaces[s]};
        auto& surface{packed->surfaces[s]};
        if (source.type > 1 || source.model > 1 || source.finish > 1) {
            Throw(G4B_ERR_UNSUPPORTED, "surface type/model/finish outside dielectric_{dielectric,metal}, "
                                       "{glisur,unified}, {polished,ground}");
        }
        surface.type = source.type;
        surface.model = source.model;
        surface.finish = source.finish;
        surface.modelValue = source.model_value;
        surface.reflectivity = pool.Add(source.reflectivity, "REFLECTIVITY");
        surface.efficiency = pool.Add(source.efficiency, "EFFICIENCY");
        surface.transmittance = pool.Add(source.transmittance, "TRANSMITTANCE");
        surface.rindex = pool.Add(source.rindex, "surface RINDEX");
        surface.specularLobe = pool.Add(source.specular_lobe, "SPECULARLOBECONSTANT");
        surface.specularSpike = pool.Add(source.specular_spike, "SPECULARSPIKECONSTANT");
        surface.backscatter = pool.Add(source.backscatter, "BACKSCATTERCONSTANT");
        surface.roughness = pool.Add(source.surface_roughness, "SURFACEROUGHNESS");
    }
    for (std::uint32_t i{}; i < scene.volume_count; ++i) {
        auto& box{packed->boxes[i]};
        for (int a{}; a < 3; ++a) {
            box.lo[a] = static_cast<float>(static_cast<double>(volumes[i].center_mm[a]) -
                                           static_cast<double>(volumes[i].half_size_mm[a]));
            box.hi[a] = static_cast<float>(static_cast<double>(volumes[i].center_mm[a]) +
                                           static_cast<double>(volumes[i].half_size_mm[a]));
        }
        auto& volume{packed->volumes[i]};
        volume.parent = parents[i] == kInvalidID ? g4b::kNoVolume : static_cast<std::uint8_t>(parents[i]);
        volume.material = static_cast<std::uint8_t>(volumes[i].material_id);
        volume.sensorID = volumes[i].sensor_id;
    }
    // Coincident faces: the analytic counterpart of MarkCoincidentBoundaries
    // (Geant4SceneExporter.cpp:379-487). Siblings must touch with opposite
    // outward normals; parent and child may share either side.
    constexpr double tolerance{1.0e-5};
    std::vector<std::pair<std::uint32_t, std::uint32_t>> touching;
    for (std::uint32_t i{}; i < scene.volume_count; ++i) {
        for (std::uint32_t j{i + 1}; j < scene.volume_count; ++j) {
            const bool sameParent{parents[i] != kInvalidID && parents[i] == parents[j]};
            const bool parentChild{parents[i] == j || parents[j] == i};
            if (!sameParent && !parentChild) {
                continue;
            }
            auto& first{packed->boxes[i]};
            auto& second{packed->boxes[j]};
            for (int axis{}; axis < 3; ++axis) {
                const int u{(axis + 1) % 3};
                const int v{(axis + 2) % 3};
                const double overlapU{std::min<double>(first.hi[u], second.hi[u]) - std::max<double>(first.lo[u], second.lo[u])};
                const double overlapV{std::min<double>(first.hi[v], second.hi[v]) - std::max<double>(first.lo[v], second.lo[v])};
                if (!(overlapU > 0.0 && overlapV > 0.0 && overlapU * overlapV > tolerance * tolerance)) {
                    continue;
                }
                for (int sideFirst{}; sideFirst < 2; ++sideFirst) {
                    for (int sideSecond{}; sideSecond < 2; ++sideSecond) {
                        if (!parentChild && sideFirst == sideSecond) {
                            continue;
                        }
                        const double planeFirst{sideFirst == 0 ? first.lo[axis] : first.hi[axis]};
                        const double planeSecond{sideSecond == 0 ? second.lo[axis] : second.hi[axis]};
                        if (std::fabs(planeFirst - planeSecond) <= tolerance) {
                            // One plane for both faces. Centre +- half in float can leave
                            // touching faces an ulp apart, and along a grazing ray an ulp
                            // in z is far more than the coincidence window in distance.
                            (sideSecond == 0 ? second.lo[axis] : second.hi[axis]) = static_cast<float>(planeFirst);
                            packed->volumes[i].coincidentFaces |= static_cast<std::uint8_t>(1U << (2 * axis + sideFirst));
                            packed->volumes[j].coincidentFaces |= static_cast<std::uint8_t>(1U << (2 * axis + sideSecond));
                            packed->volumes[i].mayCoincide = 1;
                            packed->volumes[j].mayCoincide = 1;
                            touching.emplace_back(i, j);
                        }
                    }
                }
            }
        }
    }
    // Trace candidates: the volume itself and its daughters. Coincidence
    // candidates: the volume and every volume it shares a coincident face with.
    for (std::uint32_t i{}; i < scene.volume_count; ++i) {
        packed->volumes[i].traceMask |= 1ULL << i;
        packed->volumes[i].neighbourMask |= 1ULL << i;
        if (parents[i] != kInvalidID) {
            packed->volumes[parents[i]].traceMask |= 1ULL << i;
        }
    }
    for (const auto& [i, j] : touching) {
        packed->volumes[i].neighbourMask |= 1ULL << j;
        packed->volumes[j].neighbourMask |= 1ULL << i;
    }
    std::memset(packed->surfaceTable, g4b::kNoSurface, sizeof(packed->surfaceTable));
    for (std::uint32_t from{}; from < scene.volume_count; ++from) {
        for (std::uint32_t to{}; to < scene.volume_count; ++to) {
            const auto surface{ResolveSurface(volumes, parents, bindings, from, to)};
            packed->surfaceTable[from * g4b::kMaxVolumes + to] =
                surface < scene.surface_count ? static_cast<std::uint8_t>(surface) : g4b::kNoSurface;
        }
    }
    packed->poolFloats = static_cast<std::uint32_t>(pool.floats.size());

    const std::size_t poolBytes{(pool.floats.size() * sizeof(float) + 15U) & ~std::size_t{15}};
    std::vector<unsigned char> blob(sizeof(PackedScene) + poolBytes, 0);
    std::memcpy(blob.data(), packed.get(), sizeof(PackedScene));
    if (!pool.floats.empty()) {
        std::memcpy(blob.data() + sizeof(PackedScene), pool.floats.data(), pool.floats.size() * sizeof(float));
    }
    h.dScene.Ensure(blob.size(), "cudaMalloc scene");
    Check(cudaMemcpy(h.dScene.pointer, blob.data(), blob.size(), cudaMemcpyHostToDevice), "cudaMemcpy scene");
    Check(g4b::ConfigureTransportKernels(((blob.size() + 15U) & ~std::size_t{15}) +
                                         8U * (g4b::kQueueBytesFP64 + g4b::kRingBytesFP64) +
                                         256U * g4b::kLaneTallyBytes),
          "cudaFuncSetAttribute shared memory");
    h.sceneBlob = std::move(blob);
    h.sceneBytes = static_cast<std::uint32_t>(h.sceneBlob.size());
    h.volumeIndex = std::move(index);
    h.materialCount = scene.material_count;
    h.hasScene = true;
    h.hasStaged = false;
    if (h.graphExec != nullptr) {
        cudaGraphExecDestroy(h.graphExec);
        h.graphExec = nullptr;
    }
    if (h.graph != nullptr) {
        cudaGraphDestroy(h.graph);
        h.graph = nullptr;
    }
}

// --- launching -------------------------------------------------------------

LaunchParams BaseParams(const g4b_handle& h) {
    LaunchParams p{};
    p.emissions = h.dEmissions.As<const float4>();
    p.emissionOffsets = h.dOffsets.As<const std::uint32_t>();
    p.emissionEventIndices = h.dEventIndices.As<const std::uint32_t>();
    p.slotBase = h.usesSlotBase ? h.dSlotBase.As<const std::uint32_t>() : nullptr;
    p.scene = h.dScene.As<const PackedScene>();
    p.sceneBytes = h.sceneBytes;
    p.emissionCount = h.emissionCount;
    p.eventCount = h.eventCount;
    p.photonBegin = 0;
    p.photonEnd = static_cast<std::uint32_t>(h.photonCount);
    p.emissionBegin = 0;
    p.emissionEnd = h.emissionCount;
    p.chunk = h.chunk;
    p.seed = h.config.seed;
    p.maxBounce = h.config.max_bounces_per_photon;
    p.epsilon = h.config.boundary_tolerance_mm;
    p.events = h.dEvents.As<EventCounters>();
    p.run = h.dRun.As<RunCounters>();
    p.workTicket = &p.run->workTicket;
    HitColumns hits{};
    hits.positionX = h.dHits[0].As<float>();
    hits.positionY = h.dHits[1].As<float>();
    hits.positionZ = h.dHits[2].As<float>();
    hits.time = h.dHits[3].As<float>();
    hits.directionX = h.dHits[4].As<float>();
    hits.directionY = h.dHits[5].As<float>();
    hits.directionZ = h.dHits[6].As<float>();
    hits.energy = h.dHits[7].As<float>();
    hits.eventID = h.dHits[8].As<std::uint32_t>();
    hits.photonID = h.dHits[9].As<std::uint32_t>();
    hits.sensorID = h.dHits[10].As<std::uint32_t>();
    hits.slot = h.dHits[11].As<std::uint32_t>();
    hits.capacity = h.hitCapacity;
    p.hits = hits;
    p.hitCounter = &p.run->hitCount;
    p.photonFate = h.config.record_photon_fates != 0 ? h.dFate.As<std::uint32_t>() : nullptr;
    p.photonTime = h.config.record_photon_fates != 0 ? h.dFateTime.As<double>() : nullptr;
    return p;
}

void EnsureHitCapacity(g4b_handle& h, std::uint64_t rows) {
    rows = std::max<std::uint64_t>(rows, 1);
    if (rows <= h.hitCapacity) {
        return;
    }
    for (auto& column : h.dHits) {
        column.Ensure(rows * 4U, "cudaMalloc hit column");
    }
    h.hitCapacity = rows;
}

unsigned BatchedGrid(g4b_handle& h) {
    if (h.blocksPerSM == 0) {
        int blocks{0};
        Check(g4b::TransportOccupancy(Precision(h), KernelOf(h, g4b::kBatched), static_cast<int>(h.blockSize),
                                      SharedBytes(h, g4b::kBatched, h.blockSize), &blocks),
              "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        h.blocksPerSM = static_cast<std::uint32_t>(std::max(blocks, 1));
    }
    return static_cast<unsigned>(h.smCount) * h.blocksPerSM;
}

void DestroyGraph(g4b_handle& h) {
    if (h.graphExec != nullptr) {
        cudaGraphExecDestroy(h.graphExec);
        h.graphExec = nullptr;
    }
    if (h.graph != nullptr) {
        cudaGraphDestroy(h.graph);
        h.graph = nullptr;
    }
}

// Builds (once) or updates the two-node graph and launches it.
void LaunchBatchedGraph(g4b_handle& h, const LaunchParams& params, unsigned grid) {
    EventCounters* events{params.events};
    std::uint32_t eventCount{params.eventCount};
    RunCounters* run{params.run};
    void* zeroArgs[]{&events, &eventCount, &run};
    void* transportArgs[]{const_cast<LaunchParams*>(&params)};
    const unsigned long long zeroWords{static_cast<unsigned long long>(eventCount) * (sizeof(EventCounters) / 16U)};
    const unsigned zeroBlocks{static_cast<unsigned>(std::min<unsigned long long>(
        std::max<unsigned long long>((zeroWords + 255ULL) / 256ULL, 1ULL), 1048576ULL))};

    cudaKernelNodeParams zero{};
    zero.func = const_cast<void*>(g4b::ZeroCountersKernel());
    zero.gridDim = dim3(zeroBlocks);
    zero.blockDim = dim3(256);
    zero.sharedMemBytes = 0;
    zero.kernelParams = zeroArgs;
    cudaKernelNodeParams transport{};
    transport.func = const_cast<void*>(g4b::TransportKernel(Precision(h), KernelOf(h, g4b::kBatched)));
    transport.gridDim = dim3(grid);
    transport.blockDim = dim3(h.blockSize);
    transport.sharedMemBytes = static_cast<unsigned>(SharedBytes(h, g4b::kBatched, h.blockSize));
    transport.kernelParams = transportArgs;

    if (h.graphExec == nullptr || h.graphPrecision != Precision(h)) {
        DestroyGraph(h);
        Check(cudaGraphCreate(&h.graph, 0), "cudaGraphCreate");
        Check(cudaGraphAddKernelNode(&h.zeroNode, h.graph, nullptr, 0, &zero), "cudaGraphAddKernelNode zero");
        Check(cudaGraphAddKernelNode(&h.transportNode, h.graph, &h.zeroNode, 1, &transport),
              "cudaGraphAddKernelNode transport");
        Check(cudaGraphInstantiate(&h.graphExec, h.graph, 0), "cudaGraphInstantiate");
        h.graphPrecision = Precision(h);
    } else {
        Check(cudaGraphExecKernelNodeSetParams(h.graphExec, h.zeroNode, &zero), "cudaGraphExecKernelNodeSetParams");
        Check(cudaGraphExecKernelNodeSetParams(h.graphExec, h.transportNode, &transport),
              "cudaGraphExecKernelNodeSetParams");
    }
    Check(cudaGraphLaunch(h.graphExec, h.stream), "cudaGraphLaunch");
}

// Photons per wave of the generation pass: the batch cut into equal waves
// of at most `limit` photons.
std::uint64_t EqualWaves(std::uint64_t photons, std::uint64_t limit) {
    const std::uint64_t waves{(photons + limit - 1U) / limit};
    // a multiple of 32, so every wave starts on a word of the slot bitmap
    return waves == 0U ? 0U : ((photons + waves - 1U) / waves + 31U) / 32U * 32U;
}

std::uint64_t WavePhotons(const g4b_handle& h) {
    return EqualWaves(h.photonCount, h.waveLimit != 0U ? h.waveLimit : g4b::kPhotonStoreWaveMin);
}

// Bytes of one photon store for `rows` photons: 256-byte aligned columns.
std::size_t StoreBytes(std::uint64_t rows) {
    const auto rounded{[](std::size_t bytes) { return (bytes + 255U) & ~std::size_t{255}; }};
    return 10U * rounded(rows * sizeof(float)) + rounded(rows * sizeof(double)) +
           4U * rounded(rows * sizeof(std::uint32_t));
}

// Wave size of the staged batch. The configured wave_photons, else the
// largest limit from kPhotonStoreWave down to kPhotonStoreWaveMin (halving)
// whose stores - one per wave in flight - fit in half of the device memory
// that is free or already held by this handle's stores: fewer, larger waves
// pay fewer wave changes (each a transport's drain and a generation not
// hidden behind it), and the stores of the benchmark's 1.1e9-photon batch
// take 58 GB at 2^28 photons per wave. The parked-photon queues hold 1/64 of
// a wave each, at least kDeferredMinCapacity.
void SizeWaves(g4b_handle& h) {
    if (h.config.wave_photons != 0U) {
        h.waveLimit = std::min<std::uint64_t>((h.config.wave_photons + 31ULL) / 32ULL * 32ULL, g4b::kPhotonStoreWave);
    } else {
        std::size_t free{0};
        std::size_t total{0};
        Check(cudaMemGetInfo(&free, &total), "cudaMemGetInfo");
        const std::size_t budget{(free + h.dStore.bytes) / 2U};
        std::uint64_t limit{g4b::kPhotonStoreWave};
        while (limit > g4b::kPhotonStoreWaveMin) {
            const std::uint64_t wave{EqualWaves(h.photonCount, limit)};
            const std::uint64_t waves{wave == 0U ? 0U : (h.photonCount + wave - 1U) / wave};
            if (std::min<std::uint64_t>(waves, kWaveSlots) * StoreBytes(wave) <= budget) {
                break;
            }
            limit /= 2U;
        }
        h.waveLimit = limit;
    }
    h.deferredCapacity = static_cast<std::uint32_t>(
        std::max<std::uint64_t>(g4b::kDeferredMinCapacity, WavePhotons(h) / 64U));
}

// Column views of photon store `which` (0 or 1) of the handle's allocation,
// each store sized for `rows` photons.
g4b::PhotonStore StoreView(g4b_handle& h, std::uint64_t rows, int which) {
    const auto rounded{[](std::size_t bytes) { return (bytes + 255U) & ~std::size_t{255}; }};
    const std::size_t floatColumn{rounded(rows * sizeof(float))};
    const std::size_t doubleColumn{rounded(rows * sizeof(double))};
    const std::size_t wordColumn{rounded(rows * sizeof(std::uint32_t))};
    char* next{h.dStore.As<char>() + static_cast<std::size_t>(which) * StoreBytes(rows)};
    const auto column{[&](std::size_t bytes) {
        char* start{next};
        next += bytes;
        return start;
    }};
    g4b::PhotonStore store{};
    for (int axis{}; axis < 3; ++axis) {
        store.position[axis] = reinterpret_cast<float*>(column(floatColumn));
        store.direction[axis] = reinterpret_cast<float*>(column(floatColumn));
        store.polarization[axis] = reinterpret_cast<float*>(column(floatColumn));
    }
    store.energy = reinterpret_cast<float*>(column(floatColumn));
    store.time = reinterpret_cast<double*>(column(doubleColumn));
    store.eventID = reinterpret_cast<std::uint32_t*>(column(wordColumn));
    store.photonID = reinterpret_cast<std::uint32_t*>(column(wordColumn));
    store.volume = reinterpret_cast<std::uint32_t*>(column(wordColumn));
    store.eventIndex = reinterpret_cast<std::uint32_t*>(column(wordColumn));
    return store;
}

void EnsureGenerationStream(g4b_handle& h) {
    if (h.generationStream != nullptr) {
        return;
    }
    Check(cudaStreamCreateWithFlags(&h.generationStream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    Check(cudaEventCreateWithFlags(&h.zeroedEvent, cudaEventDisableTiming), "cudaEventCreate");
    for (std::uint32_t k{}; k < kWaveSlots; ++k) {
        Check(cudaEventCreateWithFlags(&h.generatedEvent[k], cudaEventDisableTiming), "cudaEventCreate");
        Check(cudaEventCreateWithFlags(&h.storeFreeEvent[k], cudaEventDisableTiming), "cudaEventCreate");
    }
    for (std::uint32_t k{}; k + 1U < kWaveSlots; ++k) {
        Check(cudaStreamCreateWithFlags(&h.waveStreams[k], cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
        Check(cudaEventCreateWithFlags(&h.joinEvents[k], cudaEventDisableTiming), "cudaEventCreate");
    }
    for (auto& event : h.parkedEvent) {
        Check(cudaEventCreateWithFlags(&event, cudaEventDisableTiming), "cudaEventCreate");
    }
    Check(cudaStreamCreateWithFlags(&h.orderStream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    Check(cudaEventCreateWithFlags(&h.orderJoinEvent, cudaEventDisableTiming), "cudaEventCreate");
}

// Batched FP32 form with a generation pass. The batch is cut into equal waves
// of at most kPhotonStoreWave photons. GeneratePhotons fills a wave's store
// on the generation stream, and the transport kernel then takes the wave's
// photons from it. Up to kWaveSlots stores and work tickets rotate, so wave
// k+1 is generated while wave k is transported: its blocks fill the SMs that
// wave k's finished warps leave. The transports rotate over kWaveSlots
// streams as well, so wave k+1's transport also starts while wave k's last
// warps still run their longest photon histories; each wave has its own
// region of the hit buffer and its own row counter for that. A wave's parked
// photons follow its transport on its stream. The waves' orderings run in
// wave order on a stream of their own. Counters are zeroed once per batch.
// LaunchBatchedWaves returns the number of kernels launched.
void PrepareWaves(g4b_handle& h) {
    EnsureGenerationStream(h);
    const std::uint64_t wave{WavePhotons(h)};
    const std::uint64_t waves{(h.photonCount + wave - 1U) / wave};
    // a store per wave in flight: fewer for a batch of fewer waves
    h.dStore.Ensure(std::min<std::uint64_t>(waves, kWaveSlots) * StoreBytes(wave), "cudaMalloc photon stores");
    h.dTickets.Ensure(2U * kWaveSlots * sizeof(unsigned int), "cudaMalloc work tickets");  // waves, parked photons
    h.dDeferred.Ensure(std::size_t{kWaveSlots} * h.deferredCapacity * sizeof(g4b::DeferredPhoton),
                       "cudaMalloc deferred photons");
    h.dDeferredCounts.Ensure(kWaveSlots * sizeof(unsigned int), "cudaMalloc deferred counts");
    h.dWaveCounts.Ensure(waves * sizeof(unsigned long long), "cudaMalloc wave counts");
    h.dWaveRows.Ensure((waves + 1U) * sizeof(unsigned long long), "cudaMalloc wave rows");
    h.hWaveRows.Ensure((waves + 1U) * sizeof(unsigned long long), "cudaMallocHost wave rows");
    while (h.waveEvents.size() < waves) {
        cudaEvent_t event{nullptr};
        Check(cudaEventCreateWithFlags(&event, cudaEventDisableTiming), "cudaEventCreate");
        h.waveEvents.push_back(event);
    }
    // every wave gets an equal share of the hit rows
    h.waveRegionRows = h.hitCapacity / waves;
    const std::uint32_t words{static_cast<std::uint32_t>((h.photonCount + 31U) / 32U)};
    h.dBitmap.Ensure(sizeof(std::uint32_t) * words, "cudaMalloc slot bitmap");
    h.dPrefix.Ensure(sizeof(std::uint32_t) * words, "cudaMalloc slot prefix");
    h.dBlockSums.Ensure(sizeof(std::uint32_t) * ((words + 1023U) / 1024U + 1U), "cudaMalloc block sums");
    h.dDetections.Ensure(sizeof(g4b_photon_detection) * h.hitCapacity, "cudaMalloc detections");
}

// Rows [first, first + rows) of the hit buffer as columns of their own.
HitColumns HitRegion(const HitColumns& hits, std::uint64_t first, std::uint64_t rows) {
    HitColumns region{hits};
    region.positionX += first;
    region.positionY += first;
    region.positionZ += first;
    region.time += first;
    region.directionX += first;
    region.directionY += first;
    region.directionZ += first;
    region.energy += first;
    region.eventID += first;
    region.photonID += first;
    region.sensorID += first;
    region.slot += first;
    region.capacity = rows;
    return region;
}

std::uint64_t LaunchBatchedWaves(g4b_handle& h, const LaunchParams& base, unsigned grid, std::uint32_t block,
                                 bool capturing = false) {
    PrepareWaves(h);
    const std::uint64_t wave{WavePhotons(h)};
    const std::uint64_t waves{(h.photonCount + wave - 1U) / wave};
    auto* waveCounts{h.dWaveCounts.As<unsigned long long>()};
    auto* waveRows{h.dWaveRows.As<unsigned long long>()};
    const auto waveParams{[&](std::uint64_t k) {
        LaunchParams p{base};
        p.photonBegin = static_cast<std::uint32_t>(k * wave);
        p.photonEnd = static_cast<std::uint32_t>(std::min<std::uint64_t>((k + 1U) * wave, h.photonCount));
        p.store = StoreView(h, wave, static_cast<int>(k % kWaveSlots));
        p.workTicket = h.dTickets.As<unsigned int>() + k % kWaveSlots;
        p.hits = HitRegion(base.hits, k * h.waveRegionRows, h.waveRegionRows);
        p.hitCounter = waveCounts + k;
        p.deferred.photons = h.dDeferred.As<g4b::DeferredPhoton>() + (k % kWaveSlots) * h.deferredCapacity;
        p.deferred.count = h.dDeferredCounts.As<unsigned int>() + k % kWaveSlots;
        p.deferred.capacity = h.deferredCapacity;
        return p;
    }};
    cudaStream_t streams[kWaveSlots]{h.stream};
    for (std::uint32_t k{1}; k < kWaveSlots; ++k) {
        streams[k] = h.waveStreams[k - 1U];
    }
    const unsigned generateGrid{static_cast<unsigned>(h.smCount) * 8U};
    Check(g4b::LaunchZeroCounters(base.events, base.eventCount, base.run, h.stream), "zero counters");
    Check(cudaMemsetAsync(waveCounts, 0, waves * sizeof(unsigned long long), h.stream), "zero wave counts");
    Check(cudaMemsetAsync(waveRows, 0, sizeof(unsigned long long), h.stream), "zero wave rows");
    Check(cudaEventRecord(h.zeroedEvent, h.stream), "cudaEventRecord");
    Check(cudaStreamWaitEvent(h.generationStream, h.zeroedEvent, 0), "cudaStreamWaitEvent");
    for (cudaStream_t stream : h.waveStreams) {
        Check(cudaStreamWaitEvent(stream, h.zeroedEvent, 0), "cudaStreamWaitEvent");
    }
    Check(cudaStreamWaitEvent(h.orderStream, h.zeroedEvent, 0), "cudaStreamWaitEvent");
    Check(g4b::LaunchGenerate(waveParams(0), generateGrid, SceneSharedBytes(h), h.generationStream),
          "generation launch");
    Check(cudaEventRecord(h.generatedEvent[0], h.generationStream), "cudaEventRecord");
    std::uint64_t launches{2};
    const bool ordered{h.config.ordered_detections != 0};
    for (std::uint64_t k{0}; k < waves; ++k) {
        const LaunchParams p{waveParams(k)};
        const std::uint32_t slot{static_cast<std::uint32_t>(k % kWaveSlots)};
        const cudaStream_t stream{streams[slot]};
        Check(cudaStreamWaitEvent(stream, h.generatedEvent[slot], 0), "cudaStreamWaitEvent");
        Check(cudaMemsetAsync(p.workTicket, 0, sizeof(unsigned int), stream), "reset work ticket");
        Check(cudaMemsetAsync(p.deferred.count, 0, sizeof(unsigned int), stream), "reset deferred count");
        Check(g4b::LaunchTransport(p, g4b::kFP32, KernelOf(h, g4b::kBatched) | g4b::kPregenerated, grid, block,
                                   SharedBytes(h, g4b::kBatched, block), stream),
              "transport launch");
        Check(cudaEventRecord(h.storeFreeEvent[slot], stream), "cudaEventRecord");
        // the photons the wave parked (they left their volume, or their
        // history grew long), transported by the kernel's parked-photon form
        // from the queue, with small queue grabs; the wave's ordering waits
        // for it. A few blocks, but for the last wave: the queue holds little
        // work, but its longest histories (thousands of steps) keep their
        // blocks resident long after the rest, and every block slot they hold
        // is one the next wave's transport cannot use meanwhile.
        const unsigned parkedGrid{k + 1U == waves ? grid : std::min(grid, kParkedBlocks)};
        LaunchParams parked{p};
        parked.photonBegin = 0U;
        parked.photonEnd = 0U;
        parked.chunk = 32U;
        parked.workTicket = h.dTickets.As<unsigned int>() + kWaveSlots + slot;
        Check(cudaMemsetAsync(parked.workTicket, 0, sizeof(unsigned int), stream), "reset work ticket");
        Check(g4b::LaunchTransport(parked, g4b::kFP32,
                                   KernelOf(h, g4b::kBatched) | g4b::kPregenerated | g4b::kParkedQueue, parkedGrid,
                                   block, SharedBytes(h, g4b::kBatched, block), stream),
              "parked photons launch");
        Check(cudaEventRecord(h.parkedEvent[slot], stream), "cudaEventRecord");
        launches += 2;
        if (k + 1U < waves) {
            const std::uint32_t next{static_cast<std::uint32_t>((k + 1U) % kWaveSlots)};
            if (k + 1U >= kWaveSlots) {  // the next wave's store and ticket were last used kWaveSlots waves ago
                Check(cudaStreamWaitEvent(h.generationStream, h.storeFreeEvent[next], 0), "cudaStreamWaitEvent");
            }
            Check(g4b::LaunchGenerate(waveParams(k + 1U), generateGrid, SceneSharedBytes(h), h.generationStream),
                  "generation launch");
            Check(cudaEventRecord(h.generatedEvent[next], h.generationStream), "cudaEventRecord");
            ++launches;
        }
        // order this wave's hits after the previous wave's, on the ordering
        // stream, while the next waves are generated and transported
        Check(cudaStreamWaitEvent(h.orderStream, h.parkedEvent[slot], 0), "cudaStreamWaitEvent");
        Check(g4b::LaunchOrderWaveHits(p.hits, waveCounts + k, waveRows + k, base.run, p.photonBegin, p.photonEnd,
                                       h.dBitmap.As<std::uint32_t>(), h.dPrefix.As<std::uint32_t>(),
                                       h.dBlockSums.As<std::uint32_t>(), h.dDetections.pointer, ordered,
                                       static_cast<unsigned>(h.smCount) * 4U, h.orderStream),
              "wave hit ordering");
        launches += ordered ? 6U : 2U;
        Check(cudaMemcpyAsync(h.hWaveRows.As<unsigned long long>() + k + 1U, waveRows + k + 1U,
                              sizeof(unsigned long long), cudaMemcpyDeviceToHost, h.orderStream),
              "cudaMemcpyAsync wave rows to host");
        // inside a capture the record must stay a real event record for the host to wait on
        Check(capturing ? cudaEventRecordWithFlags(h.waveEvents[k], h.orderStream, cudaEventRecordExternal)
                        : cudaEventRecord(h.waveEvents[k], h.orderStream),
              "cudaEventRecord wave");
    }
    // the other transport streams' and the ordering stream's last work joins
    // the handle's stream
    for (std::uint32_t k{}; k + 1U < kWaveSlots; ++k) {
        Check(cudaEventRecord(h.joinEvents[k], h.waveStreams[k]), "cudaEventRecord");
        Check(cudaStreamWaitEvent(h.stream, h.joinEvents[k], 0), "cudaStreamWaitEvent");
    }
    Check(cudaEventRecord(h.orderJoinEvent, h.orderStream), "cudaEventRecord");
    Check(cudaStreamWaitEvent(h.stream, h.orderJoinEvent, 0), "cudaStreamWaitEvent");
    return launches;
}

// The generation-pass waves as a CUDA graph: captured from the handle's
// streams (transport, generation, ordering) on every run (the launch
// parameters and wave count follow the batch), applied to the previous
// executable graph when its shape still fits and instantiated afresh when it
// does not, then launched. Relaunches of a batch therefore replay one graph.
std::uint64_t LaunchBatchedWavesGraph(g4b_handle& h, const LaunchParams& base, unsigned grid, std::uint32_t block) {
    PrepareWaves(h);  // allocations stay outside the capture
    Check(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    cudaGraph_t graph{nullptr};
    std::uint64_t launches{0};
    try {
        launches = LaunchBatchedWaves(h, base, grid, block, true);
    } catch (...) {
        cudaStreamEndCapture(h.stream, &graph);
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        static_cast<void>(cudaGetLastError());
        throw;
    }
    Check(cudaStreamEndCapture(h.stream, &graph), "cudaStreamEndCapture");
    bool updated{false};
    if (h.wavesExec != nullptr) {
        cudaGraphExecUpdateResultInfo info{};
        if (cudaGraphExecUpdate(h.wavesExec, graph, &info) == cudaSuccess) {
            updated = true;
        } else {
            static_cast<void>(cudaGetLastError());  // a shape change is not an error: instantiate anew
            cudaGraphExecDestroy(h.wavesExec);
            h.wavesExec = nullptr;
        }
    }
    if (!updated) {
        const cudaError_t status{cudaGraphInstantiate(&h.wavesExec, graph, 0)};
        if (status != cudaSuccess) {
            h.wavesExec = nullptr;
        }
        cudaGraphDestroy(graph);
        Check(status, "cudaGraphInstantiate");
    } else {
        cudaGraphDestroy(graph);
    }
    Check(cudaGraphLaunch(h.wavesExec, h.stream), "cudaGraphLaunch");
    return launches;
}

// Hit rows reserved by default: a quarter of the photons (at least 2^20, at
// most all of them). Overflow is caught after the launch and the batch is
// rerun with an exact-size buffer, which gives identical results because
// every photon replays from its RNG counters.
std::uint64_t DefaultHitRows(std::uint64_t photons) {
    return std::min<std::uint64_t>(photons, std::max<std::uint64_t>(photons / 4U, 1U << 20U));
}

// Runs the staged batch once: counters zeroed, transport, metadata back.
void RunStaged(g4b_handle& h) {
    EnsureHitCapacity(h, h.config.hit_capacity != 0 ? h.config.hit_capacity : DefaultHitRows(h.photonCount));
    LaunchParams base{BaseParams(h)};
    Check(cudaEventRecord(h.kernelTimer.start, h.stream), "cudaEventRecord");
    if (Form(h) == g4b::kBatched) {
        const unsigned grid{BatchedGrid(h)};
        if (UsesGenerationPass(h)) {
            SizeWaves(h);
        }
        if (h.chunkAdaptive) {
            // at least eight queue grabs per warp, so that a small batch's
            // photons (and its tail) are shared out over every warp; never
            // more than the configured chunk
            const std::uint64_t warps{static_cast<std::uint64_t>(grid) * (h.blockSize / 32U)};
            const std::uint64_t photons{UsesGenerationPass(h) ? WavePhotons(h) : h.photonCount};
            const std::uint64_t perWarp{photons / (warps * 8U)};
            base.chunk = RoundChunk(static_cast<std::uint32_t>(std::clamp<std::uint64_t>(perWarp, 32U, h.chunk)));
        }
        h.pendingWaves = 0;
        if (UsesGenerationPass(h)) {
            h.launchCount += h.config.use_cuda_graph != 0 ? LaunchBatchedWavesGraph(h, base, grid, h.blockSize)
                                                           : LaunchBatchedWaves(h, base, grid, h.blockSize);
            h.pendingWaves = (h.photonCount + WavePhotons(h) - 1U) / WavePhotons(h);
        } else if (h.config.use_cuda_graph != 0) {
            LaunchBatchedGraph(h, base, grid);
            h.launchCount += 2;
        } else {
            Check(g4b::LaunchZeroCounters(base.events, base.eventCount, base.run, h.stream), "zero counters");
            Check(g4b::LaunchTransport(base, Precision(h), KernelOf(h, g4b::kBatched), grid, h.blockSize,
                                       SharedBytes(h, g4b::kBatched, h.blockSize), h.stream),
                  "transport launch");
            h.launchCount += 2;
        }
    } else {
        Check(g4b::LaunchZeroCounters(base.events, base.eventCount, base.run, h.stream), "zero counters");
        ++h.launchCount;
        for (const auto& event : h.plainEvents) {
            LaunchParams p{base};
            p.emissionBegin = event.emissionBegin;
            p.emissionEnd = event.emissionEnd;
            p.photonBegin = event.photonBegin;
            p.photonEnd = event.photonEnd;
            const std::uint32_t photons{event.photonEnd - event.photonBegin};
            const unsigned grid{(photons + h.blockSize - 1U) / h.blockSize};
            Check(g4b::LaunchTransport(p, Precision(h), KernelOf(h, g4b::kPlain), grid, h.blockSize,
                                       SharedBytes(h, g4b::kPlain, h.blockSize), h.stream),
                  "transport launch");
            ++h.launchCount;
        }
    }
    Check(cudaEventRecord(h.kernelTimer.stop, h.stream), "cudaEventRecord");
    Check(cudaEventRecord(h.metadataTimer.start, h.stream), "cudaEventRecord");
    Check(cudaMemcpyAsync(h.hEvents.pointer, h.dEvents.pointer, sizeof(EventCounters) * h.eventCount,
                          cudaMemcpyDeviceToHost, h.stream),
          "cudaMemcpyAsync event counters");
    Check(cudaMemcpyAsync(h.hRun.pointer, h.dRun.pointer, sizeof(RunCounters), cudaMemcpyDeviceToHost, h.stream),
          "cudaMemcpyAsync run counters");
    Check(cudaEventRecord(h.metadataTimer.stop, h.stream), "cudaEventRecord");
    Check(cudaEventRecord(h.metadataReadyEvent, h.stream), "cudaEventRecord");
    h.metadataReady = false;
    h.fatesValid = h.config.record_photon_fates != 0;
}

// Host threads for the staging loops of a batch: reading and copying the
// gensteps is memory bound on one thread (241 MB for 1.9e6 gensteps). At least
// 2^16 gensteps per thread, at most 16 threads, and, where each thread keeps
// its own per-event tallies, at most 2^24 tally entries in all.
unsigned StagingThreads(std::uint64_t items, std::uint64_t tallyEntries = 0) {
    std::uint64_t threads{std::min<std::uint64_t>(std::max(1U, std::thread::hardware_concurrency()), 16U)};
    threads = std::min(threads, std::max<std::uint64_t>(items >> 16U, 1U));
    if (tallyEntries != 0) {
        threads = std::min(threads, std::max<std::uint64_t>((1ULL << 24U) / tallyEntries, 1U));
    }
    return static_cast<unsigned>(threads);
}

// body(begin, end, t) over `threads` contiguous parts of [0, count); part 0 on
// the calling thread. The body must not throw. A thread that cannot be started
// leaves its part to the calling thread.
template<class Body>
void ParallelRanges(std::uint32_t count, unsigned threads, const Body& body) {
    const auto begin{[&](unsigned t) {
        return static_cast<std::uint32_t>(static_cast<std::uint64_t>(count) * t / threads);
    }};
    std::vector<std::thread> pool;
    unsigned started{1U};
    try {
        pool.reserve(threads - 1U);
        for (; started < threads; ++started) {
            pool.emplace_back(body, begin(started), begin(started + 1U), started);
        }
    } catch (...) {
        // fewer threads than asked for: the remaining parts run below
    }
    for (unsigned t{started}; t < threads; ++t) {
        body(begin(t), begin(t + 1U), t);
    }
    body(begin(0U), begin(1U), 0U);
    for (auto& thread : pool) {
        thread.join();
    }
}

void Stage(g4b_handle& h, const g4b_optical_emission* emissions, std::uint32_t emissionCount,
           const std::uint32_t* eventIDs, std::uint32_t eventCount, const std::uint32_t* emissionEventIndices) {
    if (!h.hasScene) {
        Throw(G4B_ERR_NO_SCENE, "no scene has been set");
    }
    if (h.busy) {
        Throw(G4B_ERR_LOGIC, "transport queue is full");
    }
    if ((emissionCount != 0 && (emissions == nullptr || emissionEventIndices == nullptr)) ||
        (eventCount != 0 && eventIDs == nullptr)) {
        Throw(G4B_ERR_INVALID_ARGUMENT, "batch pointer is null");
    }
    // EnqueueEmissions checks (OptiXTransportHost.cpp:574-596).
    std::unordered_map<std::uint32_t, std::uint32_t> eventIndex;
    eventIndex.reserve(eventCount);
    for (std::uint32_t i{}; i < eventCount; ++i) {
        if (!eventIndex.emplace(eventIDs[i], i).second) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "event batch contains duplicate event IDs");
        }
    }
    // per-event photon totals, in parallel parts with their own tallies; the
    // first mismatching emission of any part fails the batch
    const unsigned tallyThreads{StagingThreads(emissionCount, eventCount)};
    std::vector<std::vector<std::uint64_t>> capturedBy(tallyThreads);
    std::vector<std::vector<std::uint8_t>> hasEmissionBy(tallyThreads);
    std::vector<std::uint64_t> photonsBy(tallyThreads, 0);
    std::vector<std::uint8_t> mismatchBy(tallyThreads, 0);
    for (unsigned t{}; t < tallyThreads; ++t) {  // allocated here: the parts must not throw
        capturedBy[t].assign(eventCount, 0);
        hasEmissionBy[t].assign(eventCount, 0);
    }
    ParallelRanges(emissionCount, tallyThreads, [&](std::uint32_t begin, std::uint32_t end, unsigned t) {
        std::vector<std::uint64_t>& captured{capturedBy[t]};
        std::vector<std::uint8_t>& hasEmission{hasEmissionBy[t]};
        std::uint64_t photons{0};
        for (std::uint32_t i{begin}; i < end; ++i) {
            const auto index{emissionEventIndices[i]};
            if (index >= eventCount || emissions[i].event_id != eventIDs[index]) {
                mismatchBy[t] = 1;
                return;
            }
            captured[index] += emissions[i].photon_count;
            hasEmission[index] = 1;
            photons += emissions[i].photon_count;
        }
        photonsBy[t] = photons;
    });
    if (std::find(mismatchBy.begin(), mismatchBy.end(), 1) != mismatchBy.end()) {
        Throw(G4B_ERR_INVALID_ARGUMENT, "emission event index does not match event ID");
    }
    std::vector<std::uint64_t> captured{std::move(capturedBy[0])};
    std::vector<std::uint8_t> hasEmission{std::move(hasEmissionBy[0])};
    std::uint64_t photonCount{photonsBy[0]};
    for (unsigned t{1U}; t < tallyThreads; ++t) {
        for (std::uint32_t e{}; e < eventCount; ++e) {
            captured[e] += capturedBy[t][e];
            hasEmission[e] |= hasEmissionBy[t][e];
        }
        photonCount += photonsBy[t];
    }
    if (photonCount > 0xffffffffULL) {
        Throw(G4B_ERR_OVERFLOW, "emission batch exceeds the supported photon count");
    }

    h.hasStaged = false;
    h.pendingWaves = 0;
    h.emissionCount = emissionCount;
    h.eventCount = eventCount;
    h.photonCount = photonCount;
    h.eventIDs.assign(eventIDs, eventIDs + eventCount);
    h.captured = std::move(captured);
    h.eventHasEmission = std::move(hasEmission);
    h.plainEvents.clear();
    h.usesSlotBase = false;
    h.hostToDeviceBytes = 0;
    if (emissionCount == 0 || photonCount == 0) {
        h.hasStaged = true;
        return;
    }

    // Launch order: the batch order for the batched form; for the plain form
    // each event's emissions must be contiguous, so they are grouped by event
    // (stable) and every emission keeps its original flattened slot.
    std::vector<std::uint32_t> order;
    if (Form(h) == g4b::kPlain) {
        order.resize(emissionCount);
        for (std::uint32_t i{}; i < emissionCount; ++i) {
            order[i] = i;
        }
        std::stable_sort(order.begin(), order.end(), [&](std::uint32_t a, std::uint32_t b) {
            return emissionEventIndices[a] < emissionEventIndices[b];
        });
        for (std::uint32_t i{}; i < emissionCount; ++i) {
            if (order[i] != i) {
                h.usesSlotBase = true;
                break;
            }
        }
    }
    h.hEmissions.Ensure(sizeof(g4b_optical_emission) * emissionCount, "cudaMallocHost emissions");
    h.hOffsets.Ensure(sizeof(std::uint32_t) * (emissionCount + 1U), "cudaMallocHost offsets");
    h.hEventIndices.Ensure(sizeof(std::uint32_t) * emissionCount, "cudaMallocHost event indices");
    if (h.usesSlotBase) {
        h.hSlotBase.Ensure(sizeof(std::uint32_t) * emissionCount, "cudaMallocHost slot base");
    }
    std::vector<std::uint32_t> originalOffsets;
    if (h.usesSlotBase) {
        originalOffsets.resize(emissionCount);
        std::uint32_t running{0};
        for (std::uint32_t i{}; i < emissionCount; ++i) {
            originalOffsets[i] = running;
            running += emissions[i].photon_count;
        }
    }
    auto* stagedEmissions{h.hEmissions.As<g4b_optical_emission>()};
    auto* offsets{h.hOffsets.As<std::uint32_t>()};
    auto* indices{h.hEventIndices.As<std::uint32_t>()};
    auto* slotBase{h.usesSlotBase ? h.hSlotBase.As<std::uint32_t>() : nullptr};
    const std::uint32_t* launchOrder{order.empty() ? nullptr : order.data()};
    // Staged in parallel parts of the launch order: each part copies its
    // records into pinned memory, maps their volume IDs (keeping the last
    // lookup: consecutive gensteps mostly share a volume) and writes offsets
    // relative to its first emission; the parts' totals are added after.
    constexpr std::uint32_t kNoFailure{0xffffffffU};
    const unsigned stageThreads{StagingThreads(emissionCount)};
    std::vector<std::uint32_t> partPhotons(stageThreads, 0);
    std::vector<std::uint32_t> failedAt(stageThreads, kNoFailure);
    std::vector<std::uint8_t> unknownVolume(stageThreads, 0);
    ParallelRanges(emissionCount, stageThreads, [&](std::uint32_t begin, std::uint32_t end, unsigned t) {
        bool cached{false};
        std::uint32_t lastVolumeID{0};
        std::uint32_t lastVolume{0};
        std::uint32_t running{0};
        for (std::uint32_t k{begin}; k < end; ++k) {
            const std::uint32_t i{launchOrder != nullptr ? launchOrder[k] : k};
            g4b_optical_emission record{emissions[i]};
            if (!cached || record.volume_id != lastVolumeID) {
                const auto volume{h.volumeIndex.find(record.volume_id)};
                if (volume == h.volumeIndex.end()) {
                    failedAt[t] = k;
                    unknownVolume[t] = 1;
                    return;
                }
                cached = true;
                lastVolumeID = record.volume_id;
                lastVolume = volume->second;
            }
            if (record.material_id >= h.materialCount) {
                failedAt[t] = k;
                return;
            }
            record.volume_id = lastVolume;
            stagedEmissions[k] = record;
            indices[k] = emissionEventIndices[i];
            if (slotBase != nullptr) {
                slotBase[k] = originalOffsets[i];
            }
            running += record.photon_count;
            offsets[k + 1] = running;
        }
        partPhotons[t] = running;
    });
    // the first failing emission in launch order, as a sequential pass finds it
    for (unsigned t{}; t < stageThreads; ++t) {
        if (failedAt[t] != kNoFailure) {
            Throw(G4B_ERR_INVALID_ARGUMENT, unknownVolume[t] != 0 ? "emission references an unknown scene volume ID"
                                                                  : "emission references an unknown scene material ID");
        }
    }
    offsets[0] = 0;
    if (stageThreads > 1U) {
        std::vector<std::uint32_t> partBase(stageThreads, 0);
        for (unsigned t{1U}; t < stageThreads; ++t) {
            partBase[t] = partBase[t - 1U] + partPhotons[t - 1U];
        }
        ParallelRanges(emissionCount, stageThreads, [&](std::uint32_t begin, std::uint32_t end, unsigned t) {
            for (std::uint32_t k{begin}; k < end && partBase[t] != 0; ++k) {
                offsets[k + 1] += partBase[t];
            }
        });
    }
    if (Form(h) == g4b::kPlain) {
        std::uint32_t k{0};
        while (k < emissionCount) {
            std::uint32_t end{k};
            while (end < emissionCount && indices[end] == indices[k]) {
                ++end;
            }
            if (offsets[end] > offsets[k]) {
                h.plainEvents.push_back({k, end, offsets[k], offsets[end]});
            }
            k = end;
        }
    }

    h.dEmissions.Ensure(sizeof(g4b_optical_emission) * emissionCount, "cudaMalloc emissions");
    h.dOffsets.Ensure(sizeof(std::uint32_t) * (emissionCount + 1U), "cudaMalloc offsets");
    h.dEventIndices.Ensure(sizeof(std::uint32_t) * emissionCount, "cudaMalloc event indices");
    h.dEvents.Ensure(sizeof(EventCounters) * std::max<std::uint32_t>(eventCount, 1), "cudaMalloc event counters");
    h.dRun.Ensure(sizeof(RunCounters), "cudaMalloc run counters");
    h.hEvents.Ensure(sizeof(EventCounters) * std::max<std::uint32_t>(eventCount, 1), "cudaMallocHost event counters");
    h.hRun.Ensure(sizeof(RunCounters), "cudaMallocHost run counters");
    if (h.config.record_photon_fates != 0) {
        h.dFate.Ensure(sizeof(std::uint32_t) * photonCount, "cudaMalloc photon fates");
        h.dFateTime.Ensure(sizeof(double) * photonCount, "cudaMalloc photon times");
    }

    Check(cudaEventRecord(h.hostToDeviceTimer.start, h.stream), "cudaEventRecord");
    Check(cudaMemcpyAsync(h.dEmissions.pointer, h.hEmissions.pointer, sizeof(g4b_optical_emission) * emissionCount,
                          cudaMemcpyHostToDevice, h.stream),
          "cudaMemcpyAsync emissions");
    Check(cudaMemcpyAsync(h.dOffsets.pointer, h.hOffsets.pointer, sizeof(std::uint32_t) * (emissionCount + 1U),
                          cudaMemcpyHostToDevice, h.stream),
          "cudaMemcpyAsync emission offsets");
    Check(cudaMemcpyAsync(h.dEventIndices.pointer, h.hEventIndices.pointer, sizeof(std::uint32_t) * emissionCount,
                          cudaMemcpyHostToDevice, h.stream),
          "cudaMemcpyAsync emission event indices");
    h.hostToDeviceBytes = sizeof(g4b_optical_emission) * emissionCount + sizeof(std::uint32_t) * (2U * emissionCount + 1U);
    if (h.usesSlotBase) {
        h.dSlotBase.Ensure(sizeof(std::uint32_t) * emissionCount, "cudaMalloc slot base");
        Check(cudaMemcpyAsync(h.dSlotBase.pointer, h.hSlotBase.pointer, sizeof(std::uint32_t) * emissionCount,
                              cudaMemcpyHostToDevice, h.stream),
              "cudaMemcpyAsync slot base");
        h.hostToDeviceBytes += sizeof(std::uint32_t) * emissionCount;
    }
    Check(cudaEventRecord(h.hostToDeviceTimer.stop, h.stream), "cudaEventRecord");
    h.hasStaged = true;
}

// Waits for the pending batch's metadata; re-runs it with a larger hit buffer
// if the device buffer overflowed (the counter RNG makes the rerun identical).
void WaitMetadata(g4b_handle& h) {
    if (h.metadataReady) {
        return;
    }
    if (h.photonCount == 0) {
        h.metadataReady = true;
        return;
    }
    Check(cudaEventSynchronize(h.metadataReadyEvent), "cudaEventSynchronize metadata");
    const auto* run{h.hRun.As<RunCounters>()};
    if (h.pendingWaves != 0U) {
        // generation-pass waves: each wave has an equal region of the hit rows
        if (run->maxWaveHits > h.waveRegionRows) {
            const std::uint64_t region{run->maxWaveHits + run->maxWaveHits / 8U};
            EnsureHitCapacity(h, region * h.pendingWaves);
            RunStaged(h);
            Check(cudaEventSynchronize(h.metadataReadyEvent), "cudaEventSynchronize metadata");
        }
    } else if (run->hitCount > h.hitCapacity) {
        EnsureHitCapacity(h, run->hitCount + run->hitCount / 8U);
        RunStaged(h);
        Check(cudaEventSynchronize(h.metadataReadyEvent), "cudaEventSynchronize metadata");
    }
    h.metadataReady = true;
}

void FillStatistics(const g4b_handle& h, g4b_output& output) {
    // Per-event statistics with the valid-field bits of EnqueueEmissions /
    // CompleteOldestBatch (OptiXTransportHost.cpp:588-627,827-844).
    g4b_statistics batch{};
    const bool transported{h.emissionCount != 0 && h.photonCount != 0};
    const bool zeroPhotons{h.emissionCount != 0 && h.photonCount == 0};
    const auto* events{h.hEvents.As<EventCounters>()};
    for (std::uint32_t i{}; i < h.eventCount; ++i) {
        g4b_event_statistics record{};
        record.event_id = h.eventIDs[i];
        auto& s{record.statistics};
        if (h.eventHasEmission[i] != 0) {
            s.captured_count = h.captured[i];
            s.valid_fields |= FieldBit(G4B_FIELD_CAPTURED);
        }
        if (zeroPhotons) {
            s.valid_fields |= TerminalFields();
        }
        if (transported) {
            const auto& c{events[i]};
            s.detected_count = c.detected;
            s.absorbed_count = c.absorbed;
            s.escaped_count = c.escaped;
            s.truncated_count = c.truncated;
            s.max_bounce_count = c.maxBounce;
            s.invalid_state_count = c.invalid;
            s.zero_step_count = c.zeroStep;
            s.valid_fields |= TerminalFields();
            batch.detected_count += c.detected;
            batch.absorbed_count += c.absorbed;
            batch.escaped_count += c.escaped;
            batch.truncated_count += c.truncated;
            batch.max_bounce_count = std::max<std::uint64_t>(batch.max_bounce_count, c.maxBounce);
            batch.invalid_state_count += c.invalid;
            batch.zero_step_count += c.zeroStep;
        }
        output.event_statistics[i] = record;
    }
    if (transported) {
        batch.captured_count = h.photonCount;
        batch.valid_fields = FieldBit(G4B_FIELD_CAPTURED) | TerminalFields() | FieldBit(G4B_FIELD_TRANSPORT_TIME);
        batch.transport_time_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h.startedAt).count();
    }
    output.statistics = batch;
}

// Detections of a batch already ordered wave by wave during its transport
// (the generation-pass form): each wave's records are copied to a pinned
// caller buffer as soon as that wave has finished, on the copy stream, while
// the later waves still run; a pageable buffer gets them in one copy at the
// end. Returns false when they cannot come from there (a wave's region of the
// hit buffer overflowed and the batch was rerun, or the caller's buffer is too
// small): the caller's completion then copies the rerun's records or reports
// the capacity.
bool CompleteByWaves(g4b_handle& h, g4b_output& output) {
    if (h.pendingWaves == 0U || output.detections == nullptr || output.detection_capacity == 0U) {
        return false;
    }
    cudaPointerAttributes attributes{};
    const bool pinned{cudaPointerGetAttributes(&attributes, output.detections) == cudaSuccess &&
                      attributes.type == cudaMemoryTypeHost};
    static_cast<void>(cudaGetLastError());
    if (h.copyStream == nullptr) {
        Check(cudaStreamCreateWithFlags(&h.copyStream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
    }
    const auto* records{static_cast<const g4b_photon_detection*>(h.dDetections.pointer)};
    auto* target{static_cast<g4b_photon_detection*>(output.detections)};
    const auto* rows{h.hWaveRows.As<unsigned long long>()};
    std::uint64_t copied{0};
    Check(cudaEventRecord(h.hitsTimer.start, h.copyStream), "cudaEventRecord");
    for (std::uint64_t k{0}; k < h.pendingWaves; ++k) {
        Check(cudaEventSynchronize(h.waveEvents[k]), "cudaEventSynchronize wave");
        const std::uint64_t end{rows[k + 1U]};
        if (end > h.hitCapacity || end > output.detection_capacity) {
            Check(cudaStreamSynchronize(h.copyStream), "cudaStreamSynchronize");
            return false;
        }
        if (pinned && end > copied) {
            Check(cudaMemcpyAsync(target + copied, records + copied, sizeof(g4b_photon_detection) * (end - copied),
                                  cudaMemcpyDeviceToHost, h.copyStream),
                  "cudaMemcpyAsync detections");
            copied = end;
        }
    }
    if (!pinned) {
        copied = rows[h.pendingWaves];
        const std::size_t bytes{sizeof(g4b_photon_detection) * copied};
        h.hDetections.Ensure(bytes, "cudaMallocHost detections");
        Check(cudaMemcpyAsync(h.hDetections.pointer, records, bytes, cudaMemcpyDeviceToHost, h.copyStream),
              "cudaMemcpyAsync detections");
        Check(cudaStreamSynchronize(h.copyStream), "cudaStreamSynchronize");
        std::memcpy(target, h.hDetections.pointer, bytes);
    }
    Check(cudaEventRecord(h.hitsTimer.stop, h.copyStream), "cudaEventRecord");
    Check(cudaStreamSynchronize(h.copyStream), "cudaStreamSynchronize");
    // reruns the batch if a wave's region of the hit buffer overflowed; the
    // records copied above are then incomplete and the caller's completion
    // copies the rerun's instead
    WaitMetadata(h);
    return h.hRun.As<RunCounters>()->hitCount == copied;
}

void Complete(g4b_handle& h, g4b_output& output) {
    if (!h.busy) {
        Throw(G4B_ERR_LOGIC, "transport queue is empty");
    }
    const auto wavesStart{std::chrono::steady_clock::now()};
    const bool byWaves{CompleteByWaves(h, output)};
    WaitMetadata(h);
    const bool transported{h.emissionCount != 0 && h.photonCount != 0};
    const std::uint64_t hits{transported ? h.hRun.As<RunCounters>()->hitCount : 0};
    output.detection_count = hits;
    output.event_count = h.eventCount;
    // No detection buffer and zero capacity: counts and statistics only, the
    // hits stay on the device.
    const bool countsOnly{output.detections == nullptr && output.detection_capacity == 0};
    if (output.event_capacity < h.eventCount || (!countsOnly && hits != 0 && output.detection_capacity < hits) ||
        (h.eventCount != 0 && output.event_statistics == nullptr)) {
        Throw(G4B_ERR_CAPACITY, "output buffers are too small for the pending batch");
    }
    output.performance = g4b_performance{};
    if (byWaves) {
        output.performance.device_hits_to_host_ms = h.hitsTimer.Milliseconds();
        output.performance.device_hits_to_host_bytes = sizeof(g4b_photon_detection) * hits;
        output.performance.host_hit_compaction_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wavesStart).count();
    } else if (hits != 0 && !countsOnly) {
        const std::uint32_t words{static_cast<std::uint32_t>((h.photonCount + 31U) / 32U)};
        const bool ordered{h.config.ordered_detections != 0};
        if (ordered) {
            h.dBitmap.Ensure(sizeof(std::uint32_t) * words, "cudaMalloc slot bitmap");
            h.dPrefix.Ensure(sizeof(std::uint32_t) * words, "cudaMalloc slot prefix");
            h.dBlockSums.Ensure(sizeof(std::uint32_t) * ((words + 1023U) / 1024U + 1U), "cudaMalloc block sums");
        }
        const auto hostStart{std::chrono::steady_clock::now()};
        if (h.pendingWaves == 0U) {
            h.dDetections.Ensure(sizeof(g4b_photon_detection) * hits, "cudaMalloc detections");
            const LaunchParams p{BaseParams(h)};
            Check(g4b::LaunchOrderHits(p.hits, hits, static_cast<std::uint32_t>(h.photonCount),
                                       h.dBitmap.As<std::uint32_t>(), h.dPrefix.As<std::uint32_t>(),
                                       h.dBlockSums.As<std::uint32_t>(), h.dDetections.pointer, ordered, h.stream),
                  "hit ordering");
            h.launchCount += ordered ? 5 : 1;
        }
        // else: generation-pass waves, already ordered into dDetections by the
        // (re)run that WaitMetadata waited for; only the copy remains
        Check(cudaEventRecord(h.hitsTimer.start, h.stream), "cudaEventRecord");
        cudaPointerAttributes attributes{};
        const bool pinnedTarget{cudaPointerGetAttributes(&attributes, output.detections) == cudaSuccess &&
                                attributes.type == cudaMemoryTypeHost};
        cudaGetLastError();
        const std::size_t bytes{sizeof(g4b_photon_detection) * hits};
        if (pinnedTarget) {
            Check(cudaMemcpyAsync(output.detections, h.dDetections.pointer, bytes, cudaMemcpyDeviceToHost, h.stream),
                  "cudaMemcpyAsync detections");
            Check(cudaEventRecord(h.hitsTimer.stop, h.stream), "cudaEventRecord");
            Check(cudaStreamSynchronize(h.stream), "cudaStreamSynchronize");
        } else {
            h.hDetections.Ensure(bytes, "cudaMallocHost detections");
            Check(cudaMemcpyAsync(h.hDetections.pointer, h.dDetections.pointer, bytes, cudaMemcpyDeviceToHost, h.stream),
                  "cudaMemcpyAsync detections");
            Check(cudaEventRecord(h.hitsTimer.stop, h.stream), "cudaEventRecord");
            Check(cudaStreamSynchronize(h.stream), "cudaStreamSynchronize");
            std::memcpy(output.detections, h.hDetections.pointer, bytes);
        }
        output.performance.device_hits_to_host_ms = h.hitsTimer.Milliseconds();
        output.performance.device_hits_to_host_bytes = bytes;
        output.performance.host_hit_compaction_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - hostStart).count();
    }
    FillStatistics(h, output);
    if (transported) {
        const auto* run{h.hRun.As<RunCounters>()};
        auto& perf{output.performance};
        perf.host_to_device_ms = h.hostToDeviceBytes != 0 ? h.hostToDeviceTimer.Milliseconds() : 0.0;
        perf.host_to_device_bytes = h.hostToDeviceBytes;
        perf.kernel_ms = h.kernelTimer.Milliseconds();
        perf.device_metadata_to_host_ms = h.metadataTimer.Milliseconds();
        perf.device_metadata_to_host_bytes = sizeof(EventCounters) * h.eventCount + sizeof(RunCounters);
        perf.device_to_host_ms = perf.device_metadata_to_host_ms + perf.device_hits_to_host_ms;
        perf.total_bounce_count = run->totalBounces;
        perf.coincident_candidate_trace_count = run->coincidentTraces;
        perf.coincident_candidate_hit_count = run->coincidentHits;
    }
    output.performance.kernel_launch_count = h.launchCount - h.batchLaunches;
    h.busy = false;
}

template<class F>
int Guard(g4b_handle* h, F&& body) {
    try {
        body();
        return G4B_OK;
    } catch (const EngineError& error) {
        (h != nullptr ? h->error : gHandlelessError) = error.what();
        return error.code;
    } catch (const std::bad_alloc&) {
        (h != nullptr ? h->error : gHandlelessError) = "host allocation failed";
        return G4B_ERR_CUDA;
    } catch (const std::exception& error) {
        (h != nullptr ? h->error : gHandlelessError) = error.what();
        return G4B_ERR_CUDA;
    }
}

void SelectDevice(int device) {
    int count{0};
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        Throw(G4B_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    if (device >= 0) {
        if (device >= count) {
            Throw(G4B_ERR_NO_DEVICE, "CUDA device ordinal out of range");
        }
        Check(cudaSetDevice(device), "cudaSetDevice");
    }
    int current{0};
    Check(cudaGetDevice(&current), "cudaGetDevice");
    int major{0};
    Check(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, current), "cudaDeviceGetAttribute");
    if (major != 10) {
        Throw(G4B_ERR_NO_DEVICE, "this engine is built for sm_100a (B200); the visible device is not compute 10.x");
    }
}

// Copies host doubles to the device, runs `launch`, copies results back.
template<class In, class Out, class L>
void DeviceEval(int device, std::size_t inCount, const In* input, std::size_t outCount, Out* output, L&& launch) {
    SelectDevice(device);
    In* dIn{nullptr};
    Out* dOut{nullptr};
    Check(cudaMalloc(&dIn, std::max<std::size_t>(inCount, 1) * sizeof(In)), "cudaMalloc eval input");
    const auto cleanup{[&]() {
        if (dIn != nullptr) cudaFree(dIn);
        if (dOut != nullptr) cudaFree(dOut);
    }};
    try {
        Check(cudaMalloc(&dOut, std::max<std::size_t>(outCount, 1) * sizeof(Out)), "cudaMalloc eval output");
        Check(cudaMemcpy(dIn, input, inCount * sizeof(In), cudaMemcpyHostToDevice), "cudaMemcpy eval input");
        Check(launch(dIn, dOut), "eval kernel launch");
        Check(cudaDeviceSynchronize(), "eval kernel");
        Check(cudaMemcpy(output, dOut, outCount * sizeof(Out), cudaMemcpyDeviceToHost), "cudaMemcpy eval output");
    } catch (...) {
        cleanup();
        throw;
    }
    cleanup();
}

// --- ordering without allocation ------------------------------------------
//
// g4b_order_detections_static must not allocate, so it reports failures by
// status code with a message written into a buffer reserved on the thread's
// first call, and keeps the scratch address of each device in a fixed table.

static_assert(G4B_ORDER_STATIC_MAX_SLOTS == g4b::kStaticOrderMaxSlots,
              "the header's slot limit must match the kernels' scratch size");
constexpr std::size_t kStaticOrderMessageBytes{256};
constexpr int kStaticOrderDevices{64};
std::mutex gStaticOrderLock;
std::uint32_t* gStaticOrderScratch[kStaticOrderDevices]{};

int StaticOrderFailure(int code, const char* what, cudaError_t error = cudaSuccess) {
    // the message stays below the reserved capacity, so no allocation
    gHandlelessError.assign(what);
    if (error != cudaSuccess) {
        gHandlelessError.append(": ");
        gHandlelessError.append(cudaGetErrorName(error));
    }
    return code;
}

}  // namespace

extern "C" {

uint32_t g4b_abi_version(void) { return G4B_ABI_VERSION; }

const char* g4b_last_error(const g4b_handle* handle) {
    return handle != nullptr ? handle->error.c_str() : gHandlelessError.c_str();
}

int g4b_create(const g4b_config* config, g4b_handle** outHandle) {
    return Guard(nullptr, [&]() {
        if (config == nullptr || outHandle == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null config or handle pointer");
        }
        *outHandle = nullptr;
        if (config->abi_version != G4B_ABI_VERSION) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "g4b_config.abi_version does not match this library");
        }
        if (config->precision > G4B_PRECISION_FP64 || config->launch_form > G4B_FORM_PLAIN) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "unknown precision or launch form");
        }
        if (config->block_size != 0 && (config->block_size % 32 != 0 || config->block_size > 256)) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "block_size must be a multiple of 32 and at most 256");
        }
        if (config->generation_pass > 3U) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "generation_pass must be 0, 1, 2 or 3");
        }
        SelectDevice(config->device);
        auto handle{std::make_unique<g4b_handle>()};
        handle->config = *config;
        if (handle->config.max_bounces_per_photon == 0) {
            handle->config.max_bounces_per_photon = 4096;
        }
        if (!(handle->config.boundary_tolerance_mm > 0.0F)) {
            handle->config.boundary_tolerance_mm = 1.0e-4F;
        }
        Check(cudaGetDevice(&handle->device), "cudaGetDevice");
        Check(cudaDeviceGetAttribute(&handle->smCount, cudaDevAttrMultiProcessorCount, handle->device),
              "cudaDeviceGetAttribute");
        Check(cudaStreamCreateWithFlags(&handle->stream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
        handle->hostToDeviceTimer.Create();
        handle->memsetTimer.Create();
        handle->kernelTimer.Create();
        handle->metadataTimer.Create();
        handle->hitsTimer.Create();
        Check(cudaEventCreateWithFlags(&handle->metadataReadyEvent, cudaEventDisableTiming), "cudaEventCreate");
        handle->blockSize = config->block_size != 0 ? config->block_size : 256;
        handle->blocksPerSM = config->blocks_per_sm;
        handle->chunk = RoundChunk(config->chunk_photons != 0 ? config->chunk_photons : 512);
        handle->chunkAdaptive = config->chunk_photons == 0;
        *outHandle = handle.release();
    });
}

int g4b_destroy(g4b_handle* handle) {
    if (handle == nullptr) {
        return G4B_OK;
    }
    if (handle->stream != nullptr) {
        cudaStreamSynchronize(handle->stream);
    }
    if (handle->generationStream != nullptr) {
        cudaStreamSynchronize(handle->generationStream);
    }
    DestroyGraph(*handle);
    if (handle->wavesExec != nullptr) {
        cudaGraphExecDestroy(handle->wavesExec);
    }
    handle->hostToDeviceTimer.Destroy();
    handle->memsetTimer.Destroy();
    handle->kernelTimer.Destroy();
    handle->metadataTimer.Destroy();
    handle->hitsTimer.Destroy();
    if (handle->metadataReadyEvent != nullptr) {
        cudaEventDestroy(handle->metadataReadyEvent);
    }
    for (cudaStream_t stream : handle->waveStreams) {
        if (stream != nullptr) {
            cudaStreamSynchronize(stream);
        }
    }
    if (handle->orderStream != nullptr) {
        cudaStreamSynchronize(handle->orderStream);
    }
    std::vector<cudaEvent_t> events{handle->zeroedEvent, handle->orderJoinEvent};
    for (std::uint32_t k{}; k < kWaveSlots; ++k) {
        events.push_back(handle->generatedEvent[k]);
        events.push_back(handle->storeFreeEvent[k]);
        events.push_back(handle->parkedEvent[k]);
    }
    for (cudaEvent_t event : handle->joinEvents) {
        events.push_back(event);
    }
    for (cudaEvent_t event : events) {
        if (event != nullptr) {
            cudaEventDestroy(event);
        }
    }
    for (cudaEvent_t event : handle->waveEvents) {
        cudaEventDestroy(event);
    }
    if (handle->copyStream != nullptr) {
        cudaStreamSynchronize(handle->copyStream);
        cudaStreamDestroy(handle->copyStream);
    }
    for (cudaStream_t stream : handle->waveStreams) {
        if (stream != nullptr) {
            cudaStreamDestroy(stream);
        }
    }
    if (handle->generationStream != nullptr) {
        cudaStreamDestroy(handle->generationStream);
    }
    if (handle->orderStream != nullptr) {
        cudaStreamDestroy(handle->orderStream);
    }
    if (handle->stream != nullptr) {
        cudaStreamDestroy(handle->stream);
    }
    delete handle;
    return G4B_OK;
}

int g4b_set_scene(g4b_handle* h, const g4b_scene* scene) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (scene == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null scene");
        }
        if (h->busy) {
            Throw(G4B_ERR_LOGIC, "scene cannot be rebuilt with pending batches");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        BuildScene(*h, *scene);
    });
}

int g4b_enqueue(g4b_handle* h, const g4b_optical_emission* emissions, uint32_t emissionCount, const uint32_t* eventIDs,
                uint32_t eventCount, const uint32_t* emissionEventIndices) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        h->startedAt = std::chrono::steady_clock::now();
        h->batchLaunches = h->launchCount;
        Stage(*h, emissions, emissionCount, eventIDs, eventCount, emissionEventIndices);
        if (h->photonCount != 0) {
            RunStaged(*h);
        }
        h->metadataReady = h->photonCount == 0;
        h->busy = true;
    });
}

int g4b_relaunch(g4b_handle* h) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (h->busy) {
            Throw(G4B_ERR_LOGIC, "transport queue is full");
        }
        if (!h->hasStaged) {
            Throw(G4B_ERR_LOGIC, "no staged batch to relaunch");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        h->startedAt = std::chrono::steady_clock::now();
        h->batchLaunches = h->launchCount;
        h->hostToDeviceBytes = 0;
        if (h->photonCount != 0) {
            RunStaged(*h);
        }
        h->metadataReady = h->photonCount == 0;
        h->busy = true;
    });
}

int g4b_query_oldest(g4b_handle* h, uint64_t* detectionCount, uint32_t* eventCount) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (!h->busy) {
            Throw(G4B_ERR_LOGIC, "transport queue is empty");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        WaitMetadata(*h);
        const bool transported{h->emissionCount != 0 && h->photonCount != 0};
        if (detectionCount != nullptr) {
            *detectionCount = transported ? h->hRun.As<RunCounters>()->hitCount : 0;
        }
        if (eventCount != nullptr) {
            *eventCount = h->eventCount;
        }
    });
}

int g4b_poll_oldest(g4b_handle* h, int* ready) {
    if (h == nullptr || ready == nullptr) {
        gHandlelessError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (!h->busy) {
            Throw(G4B_ERR_LOGIC, "transport queue is empty");
        }
        if (h->metadataReady || h->photonCount == 0) {
            *ready = 1;
            return;
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        const cudaError_t status{cudaEventQuery(h->metadataReadyEvent)};
        if (status == cudaErrorNotReady) {
            // not an error: leave no trace of it for later launch checks
            static_cast<void>(cudaGetLastError());
            *ready = 0;
            return;
        }
        Check(status, "cudaEventQuery metadata");
        *ready = 1;
    });
}

int g4b_complete(g4b_handle* h, g4b_output* output) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (output == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null output");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        Complete(*h, *output);
    });
}

int g4b_get_stream(g4b_handle* h, void** stream) {
    if (h == nullptr || stream == nullptr) {
        gHandlelessError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    *stream = static_cast<void*>(h->stream);
    return G4B_OK;
}

int g4b_photon_fates(g4b_handle* h, uint32_t* fate, double* time, uint64_t capacity, uint64_t* count) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (!h->fatesValid || h->busy) {
            Throw(G4B_ERR_LOGIC, "no completed batch with photon fates (set record_photon_fates)");
        }
        if (count != nullptr) {
            *count = h->photonCount;
        }
        if (capacity < h->photonCount) {
            Throw(G4B_ERR_CAPACITY, "photon fate buffers are too small");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        if (fate != nullptr && h->photonCount != 0) {
            Check(cudaMemcpy(fate, h->dFate.pointer, sizeof(std::uint32_t) * h->photonCount, cudaMemcpyDeviceToHost),
                  "cudaMemcpy photon fates");
        }
        if (time != nullptr && h->photonCount != 0) {
            Check(cudaMemcpy(time, h->dFateTime.pointer, sizeof(double) * h->photonCount, cudaMemcpyDeviceToHost),
                  "cudaMemcpy photon times");
        }
    });
}

int g4b_autotune(g4b_handle* h, const uint32_t* blockSizes, uint32_t nBlockSizes, const uint32_t* chunkSizes,
                 uint32_t nChunkSizes, uint32_t repeats, g4b_tune_result* result) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (h->busy) {
            Throw(G4B_ERR_LOGIC, "autotune needs the pending batch completed first");
        }
        if (!h->hasStaged || h->photonCount == 0) {
            Throw(G4B_ERR_LOGIC, "autotune needs a staged batch with photons (enqueue and complete one first)");
        }
        if (Form(*h) != g4b::kBatched) {
            Throw(G4B_ERR_LOGIC, "autotune applies to the batched launch form");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        const std::vector<std::uint32_t> defaultBlocks{128, 256};
        const std::vector<std::uint32_t> defaultChunks{128, 512, 2048};
        std::vector<std::uint32_t> blocks(blockSizes, blockSizes + (blockSizes != nullptr ? nBlockSizes : 0));
        std::vector<std::uint32_t> chunks(chunkSizes, chunkSizes + (chunkSizes != nullptr ? nChunkSizes : 0));
        if (blocks.empty()) blocks = defaultBlocks;
        if (chunks.empty()) chunks = defaultChunks;
        repeats = std::max<uint32_t>(repeats, 1);
        g4b_tune_result best{};
        best.best_ms = std::numeric_limits<double>::infinity();
        best.worst_ms = 0.0;
        EnsureHitCapacity(*h, h->config.hit_capacity != 0 ? h->config.hit_capacity : DefaultHitRows(h->photonCount));
        for (const auto block : blocks) {
            if (block % 32 != 0 || block > 256 || block == 0) {
                Throw(G4B_ERR_INVALID_ARGUMENT, "autotune block sizes must be multiples of 32 up to 256");
            }
            int maxBlocks{0};
            Check(g4b::TransportOccupancy(Precision(*h), KernelOf(*h, g4b::kBatched), static_cast<int>(block),
                                          SharedBytes(*h, g4b::kBatched, block), &maxBlocks),
                  "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            maxBlocks = std::max(maxBlocks, 1);
            std::vector<std::uint32_t> perSM{static_cast<std::uint32_t>(maxBlocks)};
            if (maxBlocks > 1) {
                perSM.push_back(static_cast<std::uint32_t>(maxBlocks - 1));
            }
            for (const auto blocksPerSM : perSM) {
                for (const auto requested : chunks) {
                    if (requested == 0) {
                        continue;
                    }
                    const std::uint32_t chunk{RoundChunk(requested)};
                    h->blockSize = block;
                    h->blocksPerSM = blocksPerSM;
                    h->chunk = chunk;
                    LaunchParams p{BaseParams(*h)};
                    const unsigned grid{static_cast<unsigned>(h->smCount) * blocksPerSM};
                    double total{0.0};
                    for (std::uint32_t r{}; r < repeats + 1; ++r) {
                        if (UsesGenerationPass(*h)) {
                            Check(cudaEventRecord(h->kernelTimer.start, h->stream), "cudaEventRecord");
                            h->launchCount += LaunchBatchedWaves(*h, p, grid, block);
                        } else {
                            Check(g4b::LaunchZeroCounters(p.events, p.eventCount, p.run, h->stream),
                                  "zero counters");
                            Check(cudaEventRecord(h->kernelTimer.start, h->stream), "cudaEventRecord");
                            Check(g4b::LaunchTransport(p, Precision(*h), KernelOf(*h, g4b::kBatched), grid, block,
                                                       SharedBytes(*h, g4b::kBatched, block), h->stream),
                                  "transport launch");
                            h->launchCount += 2;
                        }
                        Check(cudaEventRecord(h->kernelTimer.stop, h->stream), "cudaEventRecord");
                        Check(cudaEventSynchronize(h->kernelTimer.stop), "cudaEventSynchronize");
                        if (r > 0) {
                            total += h->kernelTimer.Milliseconds();
                        }
                    }
                    const double ms{total / repeats};
                    ++best.candidates_tried;
                    best.worst_ms = std::max(best.worst_ms, ms);
                    if (ms < best.best_ms) {
                        best.best_ms = ms;
                        best.block_size = block;
                        best.blocks_per_sm = blocksPerSM;
                        best.chunk_photons = chunk;
                    }
                }
            }
        }
        h->blockSize = best.block_size;
        h->blocksPerSM = best.blocks_per_sm;
        h->chunk = best.chunk_photons;
        h->chunkAdaptive = false;
        if (result != nullptr) {
            *result = best;
        }
    });
}

int g4b_gradients(g4b_handle* h, const g4b_gradient_request* request, g4b_gradient_result* result) {
    if (h == nullptr) {
        gHandlelessError = "null handle";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Guard(h, [&]() {
        if (request == nullptr || result == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null argument");
        }
        if (h->busy) {
            Throw(G4B_ERR_LOGIC, "gradients need the pending batch completed first");
        }
        if (!h->hasStaged || h->photonCount == 0) {
            Throw(G4B_ERR_LOGIC, "gradients need a completed batch with photons");
        }
        if (h->usesSlotBase) {
            Throw(G4B_ERR_UNSUPPORTED, "gradients of a batch the plain form regrouped by event are not supported");
        }
        if (request->rindex_material_id != kInvalidID && request->rindex_material_id >= h->materialCount) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "gradient request names an unknown material");
        }
        if (request->abs_length_material_id != kInvalidID && request->abs_length_material_id >= h->materialCount) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "gradient request names an unknown material");
        }
        if (!std::isfinite(request->edge_band_mm) || !std::isfinite(request->edge_index_window)) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "gradient request's edge window is not finite");
        }
        Check(cudaSetDevice(h->device), "cudaSetDevice");
        const std::uint64_t hits{std::min<std::uint64_t>(h->hRun.As<RunCounters>()->hitCount, h->hitCapacity)};
        h->dGradient.Ensure(sizeof(g4b::GradientSums), "cudaMalloc gradient sums");
        Check(cudaMemsetAsync(h->dGradient.pointer, 0, sizeof(g4b::GradientSums), h->stream), "cudaMemsetAsync");
        const LaunchParams p{BaseParams(*h)};
        Check(cudaEventRecord(h->kernelTimer.start, h->stream), "cudaEventRecord");
        // a grid-stride replay: a few resident 128-thread blocks per SM
        const unsigned grid{static_cast<unsigned>(h->smCount) * 8U};
        const float band{request->edge_band_mm == 0.0F ? kDefaultEdgeBandMm
                                                        : (request->edge_band_mm > 0.0F ? request->edge_band_mm : 0.0F)};
        const float indexWindow{request->edge_index_window > 0.0F ? request->edge_index_window : 0.0F};
        Check(g4b::LaunchGradientReplay(p, Precision(*h), request->rindex_material_id, request->abs_length_material_id,
                                        request->reflectivity_surface_id, band, indexWindow, grid,
                                        SceneSharedBytes(*h),
                                        h->dGradient.As<g4b::GradientSums>(), h->stream),
              "gradient replay");
        Check(cudaEventRecord(h->kernelTimer.stop, h->stream), "cudaEventRecord");
        ++h->launchCount;
        g4b::GradientSums sums{};
        Check(cudaMemcpyAsync(&sums, h->dGradient.pointer, sizeof(sums), cudaMemcpyDeviceToHost, h->stream),
              "cudaMemcpyAsync gradient sums");
        Check(cudaStreamSynchronize(h->stream), "cudaStreamSynchronize");
        // N = sum f; mean t = sum f t / N; dN = sum dN_i; d(mean t) = (d(sum f t) - mean t * dN) / N.
        g4b_gradient_result out{};
        out.detected = static_cast<std::uint64_t>(sums.detected);
        out.replay_mismatches = out.detected > hits ? out.detected - hits : hits - out.detected;
        const double n{sums.detected};
        out.mean_time_ns = n > 0.0 ? sums.time / n : 0.0;
        for (int j{}; j < 4; ++j) {
            out.d_detected[j] = sums.score[j];
            out.d_mean_time_ns[j] = n > 0.0 ? (sums.timeScore[j] - out.mean_time_ns * sums.score[j]) / n : 0.0;
        }
        out.kernel_ms = h->kernelTimer.Milliseconds();
        *result = out;
    });
}

int g4b_host_alloc(size_t bytes, void** pointer) {
    return Guard(nullptr, [&]() {
        if (pointer == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null pointer");
        }
        Check(cudaMallocHost(pointer, std::max<std::size_t>(bytes, 1)), "cudaMallocHost");
    });
}

int g4b_host_free(void* pointer) {
    return Guard(nullptr, [&]() {
        if (pointer != nullptr) {
            Check(cudaFreeHost(pointer), "cudaFreeHost");
        }
    });
}

int g4b_order_detections_static(const g4b_photon_detection* unordered, const uint32_t* slots, uint64_t count,
                                uint32_t slot_limit, g4b_photon_detection* ordered, void* stream) {
    if (gHandlelessError.capacity() < kStaticOrderMessageBytes) {
        try {
            gHandlelessError.reserve(kStaticOrderMessageBytes);
        } catch (const std::bad_alloc&) {
            return G4B_ERR_CUDA;
        }
    }
    if (slot_limit > G4B_ORDER_STATIC_MAX_SLOTS) {
        return StaticOrderFailure(G4B_ERR_OVERFLOW,
                                  "slot_limit exceeds G4B_ORDER_STATIC_MAX_SLOTS (16777216), the static scratch size");
    }
    if (count == 0) {
        return G4B_OK;
    }
    if (count > slot_limit) {
        return StaticOrderFailure(G4B_ERR_INVALID_ARGUMENT, "count exceeds slot_limit: keys must be unique and below it");
    }
    if (unordered == nullptr || slots == nullptr || ordered == nullptr) {
        return StaticOrderFailure(G4B_ERR_INVALID_ARGUMENT, "null argument");
    }
    const auto in{reinterpret_cast<std::uintptr_t>(unordered)};
    const auto out{reinterpret_cast<std::uintptr_t>(ordered)};
    if (in % 16U != 0U || out % 16U != 0U || reinterpret_cast<std::uintptr_t>(slots) % 4U != 0U) {
        return StaticOrderFailure(G4B_ERR_INVALID_ARGUMENT,
                                  "records must be 16-byte aligned and slot keys 4-byte aligned");
    }
    const std::uintptr_t bytes{static_cast<std::uintptr_t>(count) * sizeof(g4b_photon_detection)};
    if (in < out + bytes && out < in + bytes) {
        return StaticOrderFailure(G4B_ERR_INVALID_ARGUMENT, "unordered and ordered records overlap");
    }
    int device{0};
    cudaError_t error{cudaGetDevice(&device)};
    if (error != cudaSuccess) {
        cudaGetLastError();
        return StaticOrderFailure(G4B_ERR_NO_DEVICE, "no current CUDA device", error);
    }
    if (device < 0 || device >= kStaticOrderDevices) {
        return StaticOrderFailure(G4B_ERR_NO_DEVICE, "device ordinal beyond the scratch address table (64 devices)");
    }
    std::uint32_t* scratch{nullptr};
    {
        const std::lock_guard<std::mutex> lock{gStaticOrderLock};
        if (gStaticOrderScratch[device] == nullptr) {
            error = g4b::StaticOrderScratch(&gStaticOrderScratch[device]);
            if (error != cudaSuccess) {
                gStaticOrderScratch[device] = nullptr;
                cudaGetLastError();
                const bool noImage{error == cudaErrorNoKernelImageForDevice || error == cudaErrorInvalidDeviceFunction};
                return StaticOrderFailure(noImage ? G4B_ERR_NO_DEVICE : G4B_ERR_CUDA,
                                          "cudaGetSymbolAddress of the static scratch", error);
            }
        }
        scratch = gStaticOrderScratch[device];
    }
    std::uint32_t rejected{0};
    error = g4b::LaunchOrderRecordsStatic(unordered, slots, count, slot_limit, scratch, ordered, &rejected,
                                          static_cast<cudaStream_t>(stream));
    if (error != cudaSuccess) {
        cudaGetLastError();
        return StaticOrderFailure(G4B_ERR_CUDA, "static ordering", error);
    }
    if (rejected != 0U) {
        return StaticOrderFailure(G4B_ERR_INVALID_ARGUMENT, "slot keys out of range or repeated");
    }
    return G4B_OK;
}

int g4b_eval_fresnel(int device, uint32_t precision, uint32_t n, const double* direction, const double* polarization,
                     const double* normal, const double* indexFrom, const double* indexTo, double* out) {
    return Guard(nullptr, [&]() {
        if (n == 0) {
            return;
        }
        if (direction == nullptr || polarization == nullptr || normal == nullptr || indexFrom == nullptr ||
            indexTo == nullptr || out == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null argument");
        }
        std::vector<double> rows(static_cast<std::size_t>(n) * 11U);
        for (std::uint32_t i{}; i < n; ++i) {
            double* row{rows.data() + static_cast<std::size_t>(i) * 11U};
            for (int k{}; k < 3; ++k) {
                row[k] = direction[3 * i + k];
                row[3 + k] = polarization[3 * i + k];
                row[6 + k] = normal[3 * i + k];
            }
            row[9] = indexFrom[i];
            row[10] = indexTo[i];
        }
        const int p{precision == G4B_PRECISION_FP64 ? g4b::kFP64 : g4b::kFP32};
        DeviceEval(device, rows.size(), rows.data(), static_cast<std::size_t>(n) * 14U, out,
                   [&](const double* in, double* o) { return g4b::LaunchEvalFresnel(p, n, in, o, nullptr); });
    });
}

int g4b_eval_lambertian(int device, uint32_t precision, uint32_t n, const double* normal, const double* radial,
                        const double* azimuth, double* out) {
    return Guard(nullptr, [&]() {
        if (n == 0) {
            return;
        }
        if (normal == nullptr || radial == nullptr || azimuth == nullptr || out == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null argument");
        }
        std::vector<double> rows(static_cast<std::size_t>(n) * 5U);
        for (std::uint32_t i{}; i < n; ++i) {
            rows[5 * i] = normal[3 * i];
            rows[5 * i + 1] = normal[3 * i + 1];
            rows[5 * i + 2] = normal[3 * i + 2];
            rows[5 * i + 3] = radial[i];
            rows[5 * i + 4] = azimuth[i];
        }
        const int p{precision == G4B_PRECISION_FP64 ? g4b::kFP64 : g4b::kFP32};
        DeviceEval(device, rows.size(), rows.data(), static_cast<std::size_t>(n) * 3U, out,
                   [&](const double* in, double* o) { return g4b::LaunchEvalLambertian(p, n, in, o, nullptr); });
    });
}

int g4b_eval_math(int device, uint32_t kind, uint32_t n, const float* x, float* out) {
    return Guard(nullptr, [&]() {
        if (n == 0) {
            return;
        }
        if (x == nullptr || out == nullptr || kind > 2) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "bad argument");
        }
        DeviceEval(device, n, x, static_cast<std::size_t>(n) * (kind == 2 ? 2U : 1U), out,
                   [&](const float* in, float* o) { return g4b::LaunchEvalMath(kind, n, in, o, nullptr); });
    });
}

int g4b_eval_uniform(int device, uint32_t n, uint64_t seed, const uint64_t* keys, const uint32_t* bounce,
                     const uint32_t* process, const uint32_t* draw, float* out) {
    return Guard(nullptr, [&]() {
        if (n == 0) {
            return;
        }
        if (keys == nullptr || bounce == nullptr || process == nullptr || draw == nullptr || out == nullptr) {
            Throw(G4B_ERR_INVALID_ARGUMENT, "null argument");
        }
        SelectDevice(device);
        unsigned long long* dKeys{nullptr};
        std::uint32_t* dCounters{nullptr};
        float* dOut{nullptr};
        std::vector<std::uint32_t> counters(static_cast<std::size_t>(n) * 3U);
        for (std::uint32_t i{}; i < n; ++i) {
            counters[3 * i] = bounce[i];
            counters[3 * i + 1] = process[i];
            counters[3 * i + 2] = draw[i];
        }
        const auto cleanup{[&]() {
            if (dKeys != nullptr) cudaFree(dKeys);
            if (dCounters != nullptr) cudaFree(dCounters);
            if (dOut != nullptr) cudaFree(dOut);
        }};
        try {
            Check(cudaMalloc(&dKeys, sizeof(unsigned long long) * n), "cudaMalloc");
            Check(cudaMalloc(&dCounters, sizeof(std::uint32_t) * 3U * n), "cudaMalloc");
            Check(cudaMalloc(&dOut, sizeof(float) * n), "cudaMalloc");
            Check(cudaMemcpy(dKeys, keys, sizeof(unsigned long long) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
            Check(cudaMemcpy(dCounters, counters.data(), sizeof(std::uint32_t) * 3U * n, cudaMemcpyHostToDevice),
                  "cudaMemcpy");
            Check(g4b::LaunchEvalUniform(n, seed, dKeys, dCounters, dOut, nullptr), "eval uniform");
            Check(cudaDeviceSynchronize(), "eval uniform");
            Check(cudaMemcpy(out, dOut, sizeof(float) * n, cudaMemcpyDeviceToHost), "cudaMemcpy");
        } catch (...) {
            cleanup();
            throw;
        }
        cleanup();
    });
}

}  // extern "C"
