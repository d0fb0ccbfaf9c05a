// g4b_transport_host.hpp - header-only C++ drop-in for OptiXTransportHost.
//
// Keeps the signatures of G4GO's OptiXTransportHost
// (include/g4go/optical/optix/OptiXTransportHost.hpp:10-26) on top of the C
// ABI in g4b.h and turns status codes back into the exception types the
// reference throws (src/optical/optix/OptiXTransportHost.cpp:47-52,515,524,
// 574-605,655-660,781), so OpticalBatchScheduler can call it unchanged:
//
//   G4B_ERR_INVALID_ARGUMENT -> std::invalid_argument
//   G4B_ERR_OVERFLOW         -> std::overflow_error
//   G4B_ERR_LOGIC/NO_SCENE   -> std::logic_error
//   anything else            -> std::runtime_error
//
// The batch type is generic: anything with `emissions`, `eventIDs` and
// `emissionEventIndices` spans whose element is the 128-byte OpticalEmission
// record (PhotonTransport.hpp:159-163) is passed through without copying.
// The scene is either a g4b_scene of boxes or the reference's exported Scene
// itself, converted by g4b::BoxScene (g4b_scene_adapter.hpp).
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "g4b.h"
#include "g4b_scene_adapter.hpp"

namespace g4b {

[[noreturn]] inline void ThrowStatus(int status, const char* message) {
    const std::string text{message != nullptr ? message : "g4b error"};
    switch (status) {
    case G4B_ERR_INVALID_ARGUMENT: throw std::invalid_argument(text);
    case G4B_ERR_OVERFLOW: throw std::overflow_error(text);
    case G4B_ERR_LOGIC:
    case G4B_ERR_NO_SCENE: throw std::logic_error(text);
    default: throw std::runtime_error(text);
    }
}

// PhotonTransportOutput (PhotonTransport.hpp:152-157) in the engine's record types.
struct TransportOutput {
    std::vector<g4b_photon_detection> detections;
    g4b_statistics statistics{};
    g4b_performance performance{};
    std::vector<g4b_event_statistics> eventStatistics;
};

class TransportHost final {
public:
    explicit TransportHost(const g4b_config& configuration) {
        g4b_config config{configuration};
        config.abi_version = G4B_ABI_VERSION;
        const int status{g4b_create(&config, &fHandle)};
        if (status != G4B_OK) {
            ThrowStatus(status, g4b_last_error(nullptr));
        }
    }
    ~TransportHost() { g4b_destroy(fHandle); }
    TransportHost(const TransportHost&) = delete;
    TransportHost& operator=(const TransportHost&) = delete;

    // PrepareScene: rebuilds when a scene at a different address is passed
    // (OptiXTransportHost.cpp:511-519).
    void PrepareScene(const g4b_scene& scene) {
        if (fSceneAddress == &scene) {
            return;
        }
        Check(g4b_set_scene(fHandle, &scene));
        fSceneAddress = &scene;
    }

    // The reference's own Scene (meshes + transforms): converted to boxes by
    // g4b::BoxScene, again only when a scene at a different address is passed.
    template<class Scene, class = decltype(std::declval<const Scene&>().Volumes())>
    void PrepareScene(const Scene& scene) {
        if (fSceneAddress == static_cast<const void*>(&scene)) {
            return;
        }
        auto boxes{std::make_unique<BoxScene>(scene)};
        Check(g4b_set_scene(fHandle, &boxes->Get()));
        fBoxScene = std::move(boxes);
        fSceneAddress = &scene;
    }

    template<class Scene, class Batch>
    void EnqueueEmissions(const Scene& scene, const Batch& batch) {
        static_assert(sizeof(*batch.emissions.data()) == sizeof(g4b_optical_emission),
                      "emission records must be the 128-byte OpticalEmission layout");
        PrepareScene(scene);
        if (batch.eventIDs.size() > 0xffffffffULL) {
            throw std::overflow_error("event batch exceeds the supported event count");
        }
        if (batch.emissions.size() > 0xffffffffULL) {
            throw std::overflow_error("emission batch exceeds the supported launch size");
        }
        if (batch.emissionEventIndices.size() != batch.emissions.size()) {
            throw std::invalid_argument("emission event-index count does not match emissions");
        }
        Check(g4b_enqueue(fHandle, reinterpret_cast<const g4b_optical_emission*>(batch.emissions.data()),
                          static_cast<std::uint32_t>(batch.emissions.size()), batch.eventIDs.data(),
                          static_cast<std::uint32_t>(batch.eventIDs.size()), batch.emissionEventIndices.data()));
        fPendingEvents = static_cast<std::uint32_t>(batch.eventIDs.size());
    }

    TransportOutput CompleteOldestBatch() {
        std::uint64_t detections{0};
        std::uint32_t events{0};
        Check(g4b_query_oldest(fHandle, &detections, &events));
        TransportOutput output;
        output.detections.resize(static_cast<std::size_t>(detections));
        output.eventStatistics.resize(events);
        g4b_output raw{};
        raw.detections = output.detections.data();
        raw.detection_capacity = detections;
        raw.event_statistics = output.eventStatistics.data();
        raw.event_capacity = events;
        Check(g4b_complete(fHandle, &raw));
        output.statistics = raw.statistics;
        output.performance = raw.performance;
        return output;
    }

    // CompleteOldestBatch into the caller's detection buffer, without asking
    // for the counts first. With a pinned buffer (g4b_host_alloc), a batch of
    // at least 2^24 photons has each wave's detections copied into it while
    // its later waves still run. The batch's records are the first
    // `detectionCount` of `detections`; `output.detections` stays empty.
    // Returns false, with the batch still pending, when `capacity` is below
    // the batch's detection count: CompleteOldestBatch() then completes it.
    // A null `detections` throws std::invalid_argument and leaves the batch
    // pending (g4b_complete would otherwise take it as a counts-only call and
    // leave the hits on the device).
    bool CompleteOldestBatchInto(g4b_photon_detection* detections, std::uint64_t capacity, TransportOutput& output,
                                 std::uint64_t& detectionCount) {
        if (detections == nullptr) {
            throw std::invalid_argument("CompleteOldestBatchInto needs a detection buffer");
        }
        output.detections.clear();
        output.eventStatistics.resize(std::max<std::uint32_t>(fPendingEvents, 1U));
        g4b_output raw{};
        raw.detections = detections;
        raw.detection_capacity = capacity;
        raw.event_statistics = output.eventStatistics.data();
        raw.event_capacity = fPendingEvents;
        const int status{g4b_complete(fHandle, &raw)};
        if (status == G4B_ERR_CAPACITY) {
            return false;
        }
        Check(status);
        output.eventStatistics.resize(raw.event_count);
        output.statistics = raw.statistics;
        output.performance = raw.performance;
        detectionCount = raw.detection_count;
        return true;
    }

    g4b_handle* Handle() const { return fHandle; }

private:
    void Check(int status) const {
        if (status != G4B_OK) {
            ThrowStatus(status, g4b_last_error(fHandle));
        }
    }

    g4b_handle* fHandle{nullptr};
    std::uint32_t fPendingEvents{0};  // events of the batch last enqueued
    const void* fSceneAddress{nullptr};
    std::unique_ptr<BoxScene> fBoxScene;
};

}  // namespace g4b
