// g4b_batch_scheduler.hpp - header-only C++ drop-in for OpticalBatchScheduler.
//
// Keeps the calls G4GO's Geant4 side makes on OpticalBatchScheduler
// (include/g4go/optical/geant4/OpticalBatchScheduler.hpp:32-93) on top of the
// C ABI in g4b_scheduler.h: BeginRun, Submit returning a shared future of
// the event's output (PhotonTransportFuture, PhotonTransport.hpp:173),
// EndRun, RunStatistics and BatchStatistics. Statuses come back as the
// reference's exception types (g4b::ThrowStatus in g4b_transport_host.hpp);
// a failed transport surfaces from the future's get(), as a promise's
// set_exception does in the reference (OpticalBatchScheduler.cpp:599-616).
#pragma once

#include <cstdint>
#include <future>
#include <memory>
#include <stdexcept>
#include <vector>

#include "g4b_scheduler.h"
#include "g4b_transport_host.hpp"

namespace g4b {

using TransportFuture = std::shared_future<TransportOutput>;

class BatchScheduler final {
public:
    // Scheduler over the engine: batches_in_flight (0: eight) handles made
    // from `engine` with `scene` set on each.
    BatchScheduler(const g4b_config& engine, const g4b_scene& scene, const g4b_scheduler_config& batching)
        : fEngine{engine}, fScene{&scene}, fBatching{batching} {
        fEngine.abi_version = G4B_ABI_VERSION;
        fBatching.abi_version = G4B_ABI_VERSION;
    }
    // Scheduler over caller-supplied transports (one to eight).
    BatchScheduler(const std::vector<g4b_transport_ops>& transports, const g4b_scheduler_config& batching)
        : fTransports{transports}, fBatching{batching} {
        fBatching.abi_version = G4B_ABI_VERSION;
    }
    ~BatchScheduler() { g4b_scheduler_destroy(fHandle); }
    BatchScheduler(const BatchScheduler&) = delete;
    BatchScheduler& operator=(const BatchScheduler&) = delete;

    void BeginRun() {
        if (fHandle != nullptr) {
            return;
        }
        const int status{fTransports.empty()
                             ? g4b_scheduler_create(&fEngine, fScene, &fBatching, &fHandle)
                             : g4b_scheduler_create_with_transport(fTransports.data(),
                                                                   static_cast<std::uint32_t>(fTransports.size()),
                                                                   &fBatching, &fHandle)};
        Check(status);
    }

    void EndRun() {
        if (fHandle != nullptr) {
            Check(g4b_scheduler_end_run(fHandle));
        }
    }

    // Submit: `emissions` is any contiguous range of 128-byte OpticalEmission
    // records (a std::vector<OpticalEmission> or a span of them).
    template<class Emissions>
    TransportFuture Submit(std::uint32_t eventID, const Emissions& emissions, std::uint64_t photonCount,
                           const g4b_statistics* sourceStatistics = nullptr) {
        static_assert(sizeof(*emissions.data()) == sizeof(g4b_optical_emission),
                      "emission records must be the 128-byte OpticalEmission layout");
        if (fHandle == nullptr) {
            throw std::runtime_error("optical submission queue is not ready");
        }
        if (emissions.size() > 0xffffffffULL) {
            throw std::overflow_error("optical submission exceeds the supported emission count");
        }
        std::uint64_t ticket{};
        Check(g4b_scheduler_submit(fHandle, eventID, reinterpret_cast<const g4b_optical_emission*>(emissions.data()),
                                   static_cast<std::uint32_t>(emissions.size()), photonCount, sourceStatistics,
                                   &ticket));
        g4b_scheduler* handle{fHandle};
        return std::async(std::launch::deferred, [handle, ticket]() { return Collect(handle, ticket); }).share();
    }

    g4b_statistics RunStatistics() const {
        g4b_statistics run{};
        Check(g4b_scheduler_statistics(fHandle, &run, nullptr));
        return run;
    }

    g4b_batch_statistics BatchStatistics() const {
        g4b_batch_statistics batch{};
        Check(g4b_scheduler_statistics(fHandle, nullptr, &batch));
        return batch;
    }

private:
    static TransportOutput Collect(g4b_scheduler* handle, std::uint64_t ticket) {
        TransportOutput output;
        output.eventStatistics.resize(1);
        output.detections.resize(1024);
        for (;;) {
            g4b_output raw{};
            raw.detections = output.detections.data();
            raw.detection_capacity = output.detections.size();
            raw.event_statistics = output.eventStatistics.data();
            raw.event_capacity = 1U;
            const int status{g4b_scheduler_wait(handle, ticket, -1, &raw)};
            if (status == G4B_ERR_CAPACITY) {
                output.detections.resize(static_cast<std::size_t>(raw.detection_count));
                continue;
            }
            if (status != G4B_OK) {
                ThrowStatus(status, g4b_scheduler_last_error());
            }
            output.detections.resize(static_cast<std::size_t>(raw.detection_count));
            output.statistics = raw.statistics;
            output.performance = raw.performance;
            return output;
        }
    }

    static void Check(int status) {
        if (status != G4B_OK) {
            ThrowStatus(status, g4b_scheduler_last_error());
        }
    }

    g4b_config fEngine{};
    const g4b_scene* fScene{nullptr};
    std::vector<g4b_transport_ops> fTransports;
    g4b_scheduler_config fBatching{};
    g4b_scheduler* fHandle{nullptr};
};

}  // namespace g4b
