// scheduler.cpp - streaming batch scheduler (include/g4b_scheduler.h).
//
// Host-side counterpart of OpticalBatchScheduler
// (src/optical/geant4/OpticalBatchScheduler.cpp): producers submit one event's
// gensteps at a time; one transport thread batches them, drives the transport
// and hands every event its detections and statistics. Plain C++17 threads;
// no CUDA call here (the engine's C ABI does those on the transport thread).

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "../../include/g4b.h"
#include "../../include/g4b_scheduler.h"

namespace {

using Clock = std::chrono::steady_clock;

thread_local std::string tLastError;

// A failure with the status it maps to at the C ABI.
struct Failure : std::runtime_error {
    int status;
    Failure(int code, const std::string& message) : std::runtime_error(message), status(code) {}
};

constexpr std::uint32_t Bit(int field) { return 1U << static_cast<unsigned>(field); }

// PhotonTransportStatisticField bits the transport fills
// (OpticalBatchScheduler.cpp:178-184, 233-239).
constexpr std::uint32_t kTerminalFields{Bit(G4B_FIELD_DETECTED) | Bit(G4B_FIELD_ABSORBED) |
                                        Bit(G4B_FIELD_ESCAPED) | Bit(G4B_FIELD_TRUNCATED) |
                                        Bit(G4B_FIELD_MAX_BOUNCE) | Bit(G4B_FIELD_INVALID_STATE) |
                                        Bit(G4B_FIELD_ZERO_STEP)};

double MillisecondsSince(Clock::time_point start) {
    return std::chrono::duration<double, std::milli>(Clock::now() - start).count();
}

void Accumulate(g4b_performance& total, const g4b_performance& p) {
    total.host_to_device_ms += p.host_to_device_ms;
    total.host_to_device_bytes += p.host_to_device_bytes;
    total.device_memset_ms += p.device_memset_ms;
    total.kernel_ms += p.kernel_ms;
    total.device_hit_compaction_ms += p.device_hit_compaction_ms;
    total.device_to_host_ms += p.device_to_host_ms;
    total.device_metadata_to_host_ms += p.device_metadata_to_host_ms;
    total.device_metadata_to_host_bytes += p.device_metadata_to_host_bytes;
    total.device_hits_to_host_ms += p.device_hits_to_host_ms;
    total.device_hits_to_host_bytes += p.device_hits_to_host_bytes;
    total.host_hit_compaction_ms += p.host_hit_compaction_ms;
    total.total_bounce_count += p.total_bounce_count;
    total.coincident_candidate_trace_count += p.coincident_candidate_trace_count;
    total.coincident_candidate_hit_count += p.coincident_candidate_hit_count;
    total.kernel_launch_count += p.kernel_launch_count;
}

struct Request {
    std::uint64_t ticket{};
    std::uint32_t eventID{};
    std::uint64_t photons{};
    std::vector<g4b_optical_emission> emissions;
    g4b_statistics source{};
    Clock::time_point queuedAt{};
};

using Detections = std::vector<g4b_photon_detection>;

// What g4b_scheduler_wait hands out for one ticket: the event's detections are
// [begin, begin + count) of its batch's detection array, shared by the
// batch's events (one run per event when the batch's detections come back in
// flattened-photon order), or of an array of its own.
struct Result {
    bool ready{false};
    int status{G4B_OK};
    std::string message;
    std::shared_ptr<const Detections> detections;
    std::size_t begin{0};
    std::size_t count{0};
    g4b_event_statistics event{};
};

struct Batch {
    std::vector<Request> requests;
    std::uint64_t photons{};
    std::vector<g4b_optical_emission> emissions;
    std::vector<std::uint32_t> eventIDs;
    std::vector<std::uint32_t> emissionEventIndices;
};

struct InFlight {
    Batch batch;
    std::size_t transport{};
};

struct Retired {
    Batch batch;
    Detections detections;
    std::vector<g4b_event_statistics> events;
    g4b_output output{};
};

// A transport behind g4b_transport_ops, with statuses turned into Failure.
class Transport {
public:
    explicit Transport(const g4b_transport_ops& ops) : ops_(ops) {}

    void Enqueue(const Batch& batch) {
        Check(ops_.enqueue(ops_.context, batch.emissions.data(), static_cast<std::uint32_t>(batch.emissions.size()),
                           batch.eventIDs.data(), static_cast<std::uint32_t>(batch.eventIDs.size()),
                           batch.emissionEventIndices.data()),
              "enqueue");
    }
    bool Ready() {
        int ready{0};
        Check(ops_.poll(ops_.context, &ready), "poll");
        return ready != 0;
    }
    void Complete(Retired& retired) {
        std::uint64_t detections{};
        std::uint32_t events{};
        Check(ops_.query(ops_.context, &detections, &events), "query");
        retired.detections.resize(detections);
        retired.events.resize(events);
        g4b_output& out{retired.output};
        out = {};
        out.detections = retired.detections.data();
        out.detection_capacity = detections;
        out.event_statistics = retired.events.data();
        out.event_capacity = events;
        Check(ops_.complete(ops_.context, &out), "complete");
        retired.detections.resize(out.detection_count);
        retired.events.resize(out.event_count);
    }

private:
    void Check(int status, const char* step) {
        if (status != G4B_OK) {
            const char* message{ops_.last_error != nullptr ? ops_.last_error(ops_.context) : nullptr};
            throw Failure(status, std::string{"transport "} + step + " failed: " +
                                      (message != nullptr ? message : "no message"));
        }
    }
    g4b_transport_ops ops_;
};

// The engine as a transport (one handle, one stream, its own pinned staging).
int EngineEnqueue(void* context, const g4b_optical_emission* emissions, uint32_t emissionCount,
                  const uint32_t* eventIDs, uint32_t eventCount, const uint32_t* emissionEventIndices) {
    return g4b_enqueue(static_cast<g4b_handle*>(context), emissions, emissionCount, eventIDs, eventCount,
                       emissionEventIndices);
}
int EnginePoll(void* context, int* ready) { return g4b_poll_oldest(static_cast<g4b_handle*>(context), ready); }
int EngineQuery(void* context, uint64_t* detections, uint32_t* events) {
    return g4b_query_oldest(static_cast<g4b_handle*>(context), detections, events);
}
int EngineComplete(void* context, g4b_output* output) {
    return g4b_complete(static_cast<g4b_handle*>(context), output);
}
const char* EngineLastError(void* context) { return g4b_last_error(static_cast<g4b_handle*>(context)); }

}  // namespace

struct g4b_scheduler {
    g4b_scheduler_config config{};
    // engine-owned transports: created and destroyed on the transport thread
    bool ownsEngine{false};
    g4b_config engineConfig{};
    const g4b_scene* scene{nullptr};  // only until the transport thread is ready
    std::vector<g4b_handle*> engines;
    std::vector<g4b_transport_ops> ops;

    std::mutex mutex;
    std::condition_variable condition;        // queue state, readiness, stop
    std::condition_variable resultCondition;  // results becoming ready
    std::deque<Request> pending;
    std::uint64_t queuedPhotons{0};
    std::uint64_t queuedSubmissions{0};
    std::unordered_map<std::uint64_t, Result> results;
    std::uint64_t nextTicket{1};
    std::thread thread;
    bool started{false};
    bool ready{false};
    bool stopRequested{false};
    bool failed{false};
    int failureStatus{G4B_OK};
    std::string failureMessage;

    g4b_statistics run{};
    g4b_batch_statistics batch{};

    void RunTransportThread();
    std::optional<Batch> Collect(bool busy, Transport& oldest);
    void Flatten(Batch& batch);
    void Deliver(Retired& retired);
    void Fail(int status, const std::string& message, std::vector<Batch*> batches);
};

namespace {

// Most batches on the GPU at once (engine handles of a pipelined scheduler).
// With the reference's closest-hit semantics a 1e6-photon batch ends in its
// longest histories, serial chains of thousands of steps, so batches in
// flight overlap one another's tails.
constexpr std::uint32_t kMaxBatchesInFlight{8U};

void ApplyDefaults(g4b_scheduler_config& c) {
    if (c.target_photons_per_batch == 0U) c.target_photons_per_batch = 1000000U;
    if (c.max_events_per_batch == 0U) c.max_events_per_batch = 10000U;
    if (c.max_queued_photons == 0U) c.max_queued_photons = 2000000U;
    if (c.max_queued_submissions == 0U) c.max_queued_submissions = 1024U;
    if (c.batch_collection_timeout_ms == 0U) c.batch_collection_timeout_ms = 10U;
    if (c.batches_in_flight == 0U) c.batches_in_flight = kMaxBatchesInFlight;
    c.batches_in_flight = std::min(c.batches_in_flight, kMaxBatchesInFlight);
}

template<class F>
int Api(F&& body) {
    try {
        body();
        return G4B_OK;
    } catch (const Failure& failure) {
        tLastError = failure.what();
        return failure.status;
    } catch (const std::exception& error) {
        tLastError = error.what();
        return G4B_ERR_LOGIC;
    }
}

// Starts the transport thread and waits until it is ready (BeginRun,
// OpticalBatchScheduler.cpp:45-120); on failure the scheduler is freed.
int Start(g4b_scheduler* s, g4b_scheduler** out) {
    {
        std::unique_lock lock{s->mutex};
        s->started = true;
        s->thread = std::thread([s]() { s->RunTransportThread(); });
        s->condition.wait(lock, [s]() { return s->ready; });
        s->scene = nullptr;
        if (s->failed) {
            const int status{s->failureStatus};
            tLastError = s->failureMessage;
            lock.unlock();
            s->thread.join();
            delete s;
            return status;
        }
    }
    *out = s;
    return G4B_OK;
}

}  // namespace

// The run loop of the transport thread (ProcessBatches,
// OpticalBatchScheduler.cpp:555-618), with up to ops.size() batches in flight.
void g4b_scheduler::RunTransportThread() {
    try {
        if (ownsEngine) {
            const std::size_t count{config.serial != 0U ? 1U : config.batches_in_flight};
            for (std::size_t i{}; i < count; ++i) {
                g4b_handle* handle{nullptr};
                int status{g4b_create(&engineConfig, &handle)};
                if (status != G4B_OK) {
                    throw Failure(status, std::string{"engine creation failed: "} + g4b_last_error(nullptr));
                }
                engines.push_back(handle);
                status = g4b_set_scene(handle, scene);
                if (status != G4B_OK) {
                    throw Failure(status, std::string{"engine scene failed: "} + g4b_last_error(handle));
                }
                ops.push_back({handle, EngineEnqueue, EnginePoll, EngineQuery, EngineComplete, EngineLastError});
            }
        }
    } catch (const Failure& failure) {
        for (g4b_handle* handle : engines) {
            g4b_destroy(handle);
        }
        engines.clear();
        std::scoped_lock lock{mutex};
        failed = true;
        failureStatus = failure.status;
        failureMessage = failure.what();
        ready = true;
        condition.notify_all();
        return;
    }
    std::vector<Transport> transports;
    for (const auto& o : ops) {
        transports.emplace_back(o);
    }
    const std::size_t depth{config.serial != 0U ? std::size_t{1} : transports.size()};
    {
        std::scoped_lock lock{mutex};
        ready = true;
    }
    condition.notify_all();

    std::deque<InFlight> inflight;
    std::optional<Batch> prepared;
    std::deque<Retired> retired;
    std::vector<bool> transportBusy(transports.size(), false);
    try {
        for (;;) {
            // 1. Launch a prepared batch on a free transport.
            if (prepared.has_value() && inflight.size() < depth) {
                std::size_t t{0};
                while (transportBusy[t]) {
                    ++t;
                }
                transports[t].Enqueue(*prepared);
                transportBusy[t] = true;
                if (!inflight.empty()) {
                    std::scoped_lock lock{mutex};
                    ++batch.overlapped_batch_count;
                }
                inflight.push_back({std::move(*prepared), t});
                prepared.reset();
                continue;
            }
            // 2. Hand out retired batches while the GPU works on the next ones.
            if (!retired.empty()) {
                Deliver(retired.front());
                retired.pop_front();
                continue;
            }
            // 3. Collect the next batch; with batches in flight, only until the
            //    oldest one finishes.
            if (!prepared.has_value() && (config.serial == 0U || inflight.empty())) {
                Transport* oldest{inflight.empty() ? nullptr : &transports[inflight.front().transport]};
                prepared = Collect(oldest != nullptr, oldest != nullptr ? *oldest : transports[0]);
                if (prepared.has_value()) {
                    Flatten(*prepared);
                    continue;
                }
            }
            if (inflight.empty()) {
                break;  // stop requested and the queue drained
            }
            // 4. Retire the oldest batch.
            const auto waitStart{Clock::now()};
            Retired r{};
            const std::size_t t{inflight.front().transport};
            transports[t].Complete(r);
            r.batch = std::move(inflight.front().batch);
            inflight.pop_front();
            transportBusy[t] = false;
            {
                std::scoped_lock lock{mutex};
                batch.scheduler_gpu_wait_ms += MillisecondsSince(waitStart);
            }
            retired.push_back(std::move(r));
        }
    } catch (const Failure& failure) {
        std::vector<Batch*> lost;
        for (auto& f : inflight) lost.push_back(&f.batch);
        for (auto& r : retired) lost.push_back(&r.batch);
        if (prepared.has_value()) lost.push_back(&*prepared);
        Fail(failure.status, failure.what(), lost);
    } catch (const std::exception& error) {
        std::vector<Batch*> lost;
        for (auto& f : inflight) lost.push_back(&f.batch);
        for (auto& r : retired) lost.push_back(&r.batch);
        if (prepared.has_value()) lost.push_back(&*prepared);
        Fail(G4B_ERR_LOGIC, error.what(), lost);
    }
    // A batch left in flight by a failure is abandoned with its handle.
    for (g4b_handle* handle : engines) {
        g4b_destroy(handle);
    }
    engines.clear();
}

// CollectRequests (OpticalBatchScheduler.cpp:462-509): takes queued
// submissions in order until the batch reaches the target photon count or
// the event cap, waiting for more until the collection deadline (measured
// from the first submission's queueing). With `busy` a batch is on the GPU:
// nothing to collect and `oldest` finished returns nothing (time to retire
// it), and a partial batch is closed as soon as `oldest` finishes.
std::optional<Batch> g4b_scheduler::Collect(bool busy, Transport& oldest) {
    constexpr auto kPollSlice{std::chrono::microseconds(100)};
    const bool diagnostics{config.enable_performance_diagnostics != 0U};
    std::unique_lock lock{mutex};
    const auto waitStart{Clock::now()};
    if (!busy) {
        condition.wait(lock, [this]() { return stopRequested || !pending.empty(); });
    } else {
        while (pending.empty() && !stopRequested) {
            lock.unlock();
            const bool done{oldest.Ready()};
            lock.lock();
            if (done && pending.empty()) {
                return std::nullopt;
            }
            condition.wait_for(lock, kPollSlice, [this]() { return stopRequested || !pending.empty(); });
        }
    }
    if (diagnostics) {
        batch.scheduler_input_wait_ms += MillisecondsSince(waitStart);
    }
    if (pending.empty()) {
        return std::nullopt;
    }
    Batch next;
    const auto deadline{pending.front().queuedAt + std::chrono::milliseconds(config.batch_collection_timeout_ms)};
    while (next.photons < config.target_photons_per_batch && next.requests.size() < config.max_events_per_batch) {
        if (pending.empty()) {
            if (stopRequested || next.photons == 0U) {
                break;
            }
            const auto sliceStart{Clock::now()};
            if (busy) {
                lock.unlock();
                const bool done{oldest.Ready()};
                lock.lock();
                if (done) {
                    break;  // the GPU is free: launch what there is
                }
                condition.wait_until(lock, std::min(deadline, Clock::now() + kPollSlice),
                                     [this]() { return stopRequested || !pending.empty(); });
            } else {
                condition.wait_until(lock, deadline, [this]() { return stopRequested || !pending.empty(); });
            }
            if (diagnostics) {
                batch.scheduler_input_wait_ms += MillisecondsSince(sliceStart);
            }
            if (pending.empty()) {
                if (stopRequested || Clock::now() >= deadline) {
                    break;
                }
                continue;
            }
        }
        Request request{std::move(pending.front())};
        pending.pop_front();
        next.photons += request.photons;
        queuedPhotons -= request.photons;
        --queuedSubmissions;
        if (diagnostics) {
            batch.scheduler_queue_wait_ms += MillisecondsSince(request.queuedAt);
            ++batch.total_queue_wait_count;
        }
        next.requests.push_back(std::move(request));
    }
    lock.unlock();
    condition.notify_all();  // room in the queue for blocked producers
    return next;
}

// EnqueueRequests (OpticalBatchScheduler.cpp:511-551): one flat genstep
// array with the batch's event IDs and each genstep's event index.
void g4b_scheduler::Flatten(Batch& next) {
    const auto start{Clock::now()};
    std::size_t emissions{0};
    for (const auto& request : next.requests) {
        emissions += request.emissions.size();
    }
    next.emissions.clear();
    next.emissions.reserve(emissions);
    next.eventIDs.clear();
    next.eventIDs.reserve(next.requests.size());
    next.emissionEventIndices.clear();
    next.emissionEventIndices.reserve(emissions);
    std::unordered_set<std::uint32_t> seen;
    seen.reserve(next.requests.size());
    for (const auto& request : next.requests) {
        const auto eventIndex{static_cast<std::uint32_t>(next.eventIDs.size())};
        if (!seen.insert(request.eventID).second) {
            throw Failure(G4B_ERR_INVALID_ARGUMENT, "optical batch contains duplicate event IDs");
        }
        next.eventIDs.push_back(request.eventID);
        next.emissions.insert(next.emissions.end(), request.emissions.begin(), request.emissions.end());
        next.emissionEventIndices.insert(next.emissionEventIndices.end(), request.emissions.size(), eventIndex);
    }
    if (config.enable_performance_diagnostics != 0U) {
        std::scoped_lock lock{mutex};
        batch.scheduler_batch_flatten_ms += MillisecondsSince(start);
        batch.scheduler_batch_flatten_bytes += emissions * sizeof(g4b_optical_emission);
    }
}

// CompleteBatch (OpticalBatchScheduler.cpp:230-446): splits the batch output
// per event after checking that the transport's per-event statistics, batch
// statistics and detections agree, then publishes every event's result and
// adds the batch to the run and batch statistics.
void g4b_scheduler::Deliver(Retired& retired) {
    auto& requests{retired.batch.requests};
    const std::size_t n{requests.size()};
    std::vector<Result> outputs(n);
    std::unordered_map<std::uint32_t, std::size_t> eventToRequest;
    eventToRequest.reserve(n);
    for (std::size_t i{}; i < n; ++i) {
        outputs[i].event.event_id = requests[i].eventID;
        outputs[i].event.statistics = requests[i].source;
        eventToRequest.emplace(requests[i].eventID, i);
    }
    if (retired.events.size() != n) {
        throw Failure(G4B_ERR_LOGIC, "transport output event statistics count does not match the batch");
    }
    std::vector<bool> seen(n, false);
    std::vector<std::uint64_t> detectionCounts(n, 0);
    std::uint64_t captured{}, detected{}, absorbed{}, escaped{}, truncated{}, invalid{}, zeroStep{}, maxBounce{};
    std::uint32_t commonFields{std::numeric_limits<std::uint32_t>::max()};
    for (const auto& record : retired.events) {
        const auto found{eventToRequest.find(record.event_id)};
        if (found == eventToRequest.end()) {
            throw Failure(G4B_ERR_LOGIC, "transport output contains an unknown event ID");
        }
        const std::size_t i{found->second};
        if (seen[i]) {
            throw Failure(G4B_ERR_LOGIC, "transport output contains duplicate event statistics");
        }
        seen[i] = true;
        const g4b_statistics& s{record.statistics};
        const std::uint32_t fields{s.valid_fields};
        commonFields &= fields;
        if ((fields & Bit(G4B_FIELD_TRANSPORT_TIME)) != 0U) {
            throw Failure(G4B_ERR_LOGIC, "transport event transport time is unavailable per event");
        }
        if ((fields & Bit(G4B_FIELD_CAPTURED)) != 0U) captured += s.captured_count;
        if ((fields & Bit(G4B_FIELD_DETECTED)) != 0U) detected += s.detected_count;
        if ((fields & Bit(G4B_FIELD_ABSORBED)) != 0U) absorbed += s.absorbed_count;
        if ((fields & Bit(G4B_FIELD_ESCAPED)) != 0U) escaped += s.escaped_count;
        if ((fields & Bit(G4B_FIELD_TRUNCATED)) != 0U) truncated += s.truncated_count;
        if ((fields & Bit(G4B_FIELD_INVALID_STATE)) != 0U) invalid += s.invalid_state_count;
        if ((fields & Bit(G4B_FIELD_ZERO_STEP)) != 0U) zeroStep += s.zero_step_count;
        if ((fields & Bit(G4B_FIELD_MAX_BOUNCE)) != 0U) maxBounce = std::max(maxBounce, s.max_bounce_count);
        g4b_statistics& destination{outputs[i].event.statistics};
        const std::uint32_t sourceFields{destination.valid_fields};
        if ((fields & Bit(G4B_FIELD_DETECTED)) != 0U) destination.detected_count = s.detected_count;
        if ((fields & Bit(G4B_FIELD_ABSORBED)) != 0U) destination.absorbed_count = s.absorbed_count;
        if ((fields & Bit(G4B_FIELD_ESCAPED)) != 0U) destination.escaped_count = s.escaped_count;
        if ((fields & Bit(G4B_FIELD_TRUNCATED)) != 0U) destination.truncated_count = s.truncated_count;
        if ((fields & Bit(G4B_FIELD_MAX_BOUNCE)) != 0U) destination.max_bounce_count = s.max_bounce_count;
        if ((fields & Bit(G4B_FIELD_INVALID_STATE)) != 0U) destination.invalid_state_count = s.invalid_state_count;
        if ((fields & Bit(G4B_FIELD_ZERO_STEP)) != 0U) destination.zero_step_count = s.zero_step_count;
        destination.valid_fields = ((sourceFields & ~kTerminalFields) | (fields & kTerminalFields)) &
                                   ~Bit(G4B_FIELD_TRANSPORT_TIME);
    }
    const g4b_statistics& total{retired.output.statistics};
    struct Field {
        int field;
        std::uint64_t events;
        std::uint64_t batch;
        const char* name;
    };
    const Field fields[]{{G4B_FIELD_CAPTURED, captured, total.captured_count, "captured count"},
                         {G4B_FIELD_DETECTED, detected, total.detected_count, "detected count"},
                         {G4B_FIELD_ABSORBED, absorbed, total.absorbed_count, "absorbed count"},
                         {G4B_FIELD_ESCAPED, escaped, total.escaped_count, "escaped count"},
                         {G4B_FIELD_TRUNCATED, truncated, total.truncated_count, "truncated count"},
                         {G4B_FIELD_INVALID_STATE, invalid, total.invalid_state_count, "invalid-state count"},
                         {G4B_FIELD_ZERO_STEP, zeroStep, total.zero_step_count, "zero-step count"},
                         {G4B_FIELD_MAX_BOUNCE, maxBounce, total.max_bounce_count, "maximum-bounce count"}};
    for (const Field& f : fields) {
        if ((total.valid_fields & Bit(f.field)) != 0U && (commonFields & Bit(f.field)) == 0U) {
            throw Failure(G4B_ERR_LOGIC, std::string{"transport batch statistics field is missing from event "} +
                                             f.name);
        }
    }
    for (const Field& f : fields) {
        if ((total.valid_fields & Bit(f.field)) != 0U && f.events != f.batch) {
            throw Failure(G4B_ERR_LOGIC, std::string{"transport batch/event statistics mismatch in "} + f.name);
        }
    }
    // Route the detections: one run of equal event IDs per event shares the
    // batch's array; an event whose detections are not contiguous gets a copy.
    auto shared{std::make_shared<const Detections>(std::move(retired.detections))};
    const Detections& all{*shared};
    std::vector<std::size_t> runs(n, 0);
    bool contiguous{true};
    for (std::size_t k{0}; k < all.size();) {
        const std::uint32_t eventID{all[k].event_id};
        std::size_t end{k + 1};
        while (end < all.size() && all[end].event_id == eventID) {
            ++end;
        }
        const auto found{eventToRequest.find(eventID)};
        if (found == eventToRequest.end()) {
            throw Failure(G4B_ERR_LOGIC, "transport output contains a detection for an unknown event ID");
        }
        const std::size_t i{found->second};
        if (runs[i]++ == 0U) {
            outputs[i].begin = k;
        }
        detectionCounts[i] += end - k;
        k = end;
    }
    for (std::size_t i{}; i < n; ++i) {
        contiguous = contiguous && runs[i] <= 1U;
        outputs[i].count = detectionCounts[i];
        outputs[i].detections = shared;
    }
    if (!contiguous) {
        std::vector<Detections> own(n);
        for (std::size_t i{}; i < n; ++i) {
            own[i].reserve(detectionCounts[i]);
        }
        for (const auto& detection : all) {
            own[eventToRequest.at(detection.event_id)].push_back(detection);
        }
        for (std::size_t i{}; i < n; ++i) {
            outputs[i].detections = std::make_shared<const Detections>(std::move(own[i]));
            outputs[i].begin = 0;
        }
    }
    for (std::size_t i{}; i < n; ++i) {
        if (!seen[i]) {
            throw Failure(G4B_ERR_LOGIC, "transport output is missing event statistics");
        }
        const g4b_statistics& s{outputs[i].event.statistics};
        if ((s.valid_fields & Bit(G4B_FIELD_DETECTED)) != 0U && s.detected_count != detectionCounts[i]) {
            throw Failure(G4B_ERR_LOGIC, "transport event detected count does not match compacted hits");
        }
    }
    {
        std::scoped_lock lock{mutex};
        for (std::size_t i{}; i < n; ++i) {
            Result& slot{results[requests[i].ticket]};
            slot = std::move(outputs[i]);
            slot.ready = true;
        }
        run.detected_count += total.detected_count;
        run.absorbed_count += total.absorbed_count;
        run.escaped_count += total.escaped_count;
        run.truncated_count += total.truncated_count;
        run.max_bounce_count = std::max(run.max_bounce_count, total.max_bounce_count);
        run.invalid_state_count += total.invalid_state_count;
        run.zero_step_count += total.zero_step_count;
        run.valid_fields |= total.valid_fields;
        if ((total.valid_fields & Bit(G4B_FIELD_TRANSPORT_TIME)) != 0U) {
            run.transport_time_ms += total.transport_time_ms;
        }
        Accumulate(batch.performance, retired.output.performance);
        ++batch.batch_count;
        batch.event_count += n;
        batch.photon_count += retired.batch.photons;
        batch.max_batch_event_count = std::max<std::uint64_t>(batch.max_batch_event_count, n);
        batch.max_batch_photon_count = std::max(batch.max_batch_photon_count, retired.batch.photons);
        batch.min_batch_photon_count = batch.batch_count == 1U
                                           ? retired.batch.photons
                                           : std::min(batch.min_batch_photon_count, retired.batch.photons);
    }
    resultCondition.notify_all();
}

// The failure path of ProcessBatches and FailPendingRequests
// (OpticalBatchScheduler.cpp:595-634): every request not yet handed out, and
// every later submission, fails with the error.
void g4b_scheduler::Fail(int status, const std::string& message, std::vector<Batch*> batches) {
    {
        std::scoped_lock lock{mutex};
        const auto failTicket{[&](std::uint64_t ticket) {
            Result& slot{results[ticket]};
            slot = Result{};
            slot.ready = true;
            slot.status = status;
            slot.message = message;
        }};
        for (Batch* b : batches) {
            for (const auto& request : b->requests) {
                failTicket(request.ticket);
            }
        }
        for (const auto& request : pending) {
            failTicket(request.ticket);
        }
        pending.clear();
        queuedPhotons = 0;
        queuedSubmissions = 0;
        failed = true;
        failureStatus = status;
        failureMessage = message;
        stopRequested = true;
    }
    condition.notify_all();
    resultCondition.notify_all();
}

extern "C" {

int g4b_scheduler_create(const g4b_config* engineConfig, const g4b_scene* scene, const g4b_scheduler_config* config,
                         g4b_scheduler** out) {
    if (engineConfig == nullptr || scene == nullptr || config == nullptr || out == nullptr) {
        tLastError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    if (config->abi_version != G4B_ABI_VERSION || engineConfig->abi_version != G4B_ABI_VERSION) {
        tLastError = "ABI version mismatch";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    auto* s{new g4b_scheduler{}};
    s->config = *config;
    ApplyDefaults(s->config);
    s->ownsEngine = true;
    s->engineConfig = *engineConfig;
    s->scene = scene;
    return Start(s, out);
}

int g4b_scheduler_create_with_transport(const g4b_transport_ops* ops, uint32_t opsCount,
                                        const g4b_scheduler_config* config, g4b_scheduler** out) {
    if (ops == nullptr || config == nullptr || out == nullptr) {
        tLastError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    if (config->abi_version != G4B_ABI_VERSION) {
        tLastError = "ABI version mismatch";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    if (opsCount < 1U || opsCount > kMaxBatchesInFlight) {
        tLastError = "a scheduler takes one to eight transports";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    for (uint32_t i{}; i < opsCount; ++i) {
        if (ops[i].enqueue == nullptr || ops[i].poll == nullptr || ops[i].query == nullptr ||
            ops[i].complete == nullptr) {
            tLastError = "transport operation missing";
            return G4B_ERR_INVALID_ARGUMENT;
        }
    }
    auto* s{new g4b_scheduler{}};
    s->config = *config;
    ApplyDefaults(s->config);
    s->ops.assign(ops, ops + opsCount);
    return Start(s, out);
}

int g4b_scheduler_submit(g4b_scheduler* s, uint32_t eventID, const g4b_optical_emission* emissions,
                         uint32_t emissionCount, uint64_t photonCount, const g4b_statistics* sourceStatistics,
                         uint64_t* ticket) {
    if (s == nullptr || ticket == nullptr || (emissionCount != 0U && emissions == nullptr)) {
        tLastError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Api([&]() {
        // Submit's checks (OpticalBatchScheduler.cpp:152-164); the event IDs of
        // the gensteps, which the reference checks when it flattens a batch
        // (:523-527) and then fails the whole run, are checked here instead.
        std::uint64_t counted{0};
        for (uint32_t i{}; i < emissionCount; ++i) {
            counted += emissions[i].photon_count;
            if (emissions[i].event_id != eventID) {
                throw Failure(G4B_ERR_INVALID_ARGUMENT, "optical emission event ID does not match its submission");
            }
        }
        if (counted != photonCount) {
            throw Failure(G4B_ERR_INVALID_ARGUMENT, "optical submission photon count does not match its emissions");
        }
        if (photonCount == 0U && emissionCount != 0U) {
            throw Failure(G4B_ERR_INVALID_ARGUMENT, "empty optical submissions cannot contain emissions");
        }
        if (photonCount != 0U && emissionCount == 0U) {
            throw Failure(G4B_ERR_INVALID_ARGUMENT, "non-empty optical submissions require emissions");
        }
        Request request;
        request.eventID = eventID;
        request.photons = photonCount;
        if (sourceStatistics != nullptr) {
            request.source = *sourceStatistics;
        }
        request.emissions.assign(emissions, emissions + emissionCount);

        std::unique_lock lock{s->mutex};
        if (!s->started || !s->ready) {
            throw Failure(G4B_ERR_LOGIC, "optical submission queue is not ready");
        }
        if (s->failed) {
            throw Failure(s->failureStatus, s->failureMessage);
        }
        if (s->stopRequested) {
            throw Failure(G4B_ERR_LOGIC, "photon submission queue is stopping");
        }
        const std::uint64_t maxPhotons{s->config.max_queued_photons};
        const std::uint64_t maxSubmissions{s->config.max_queued_submissions};
        if (photonCount == 0U) {
            // (:169-193) nothing to transport: complete at once
            s->run.generated_count += request.source.generated_count;
            s->run.captured_count += request.source.captured_count;
            s->run.valid_fields |= request.source.valid_fields | kTerminalFields;
            const std::uint64_t id{s->nextTicket++};
            Result& slot{s->results[id]};
            slot.ready = true;
            slot.event.event_id = eventID;
            slot.event.statistics = request.source;
            slot.event.statistics.valid_fields |= kTerminalFields;
            *ticket = id;
            lock.unlock();
            s->resultCondition.notify_all();
            return;
        }
        s->condition.wait(lock, [&]() {
            return s->failed || s->stopRequested ||
                   (s->queuedSubmissions < maxSubmissions && s->queuedPhotons + photonCount <= maxPhotons) ||
                   (s->queuedSubmissions == 0U && photonCount > maxPhotons);
        });
        if (s->failed) {
            throw Failure(s->failureStatus, s->failureMessage);
        }
        if (s->stopRequested) {
            throw Failure(G4B_ERR_LOGIC, "photon submission queue is stopping");
        }
        s->run.generated_count += request.source.generated_count;
        s->run.captured_count += request.source.captured_count;
        s->run.valid_fields |= request.source.valid_fields;
        s->queuedPhotons += photonCount;
        ++s->queuedSubmissions;
        s->batch.queue_high_water_mark = std::max(s->batch.queue_high_water_mark, s->queuedPhotons);
        request.ticket = s->nextTicket++;
        request.queuedAt = Clock::now();
        s->results[request.ticket] = Result{};
        *ticket = request.ticket;
        s->pending.push_back(std::move(request));
        lock.unlock();
        s->condition.notify_all();
    });
}

int g4b_scheduler_wait(g4b_scheduler* s, uint64_t ticket, int64_t timeoutMs, g4b_output* output) {
    if (s == nullptr || output == nullptr) {
        tLastError = "null argument";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Api([&]() {
        std::unique_lock lock{s->mutex};
        auto found{s->results.find(ticket)};
        if (found == s->results.end()) {
            throw Failure(G4B_ERR_INVALID_ARGUMENT, "unknown or released ticket");
        }
        const auto isReady{[&]() { return s->results.at(ticket).ready; }};
        if (timeoutMs < 0) {
            s->resultCondition.wait(lock, isReady);
        } else if (!s->resultCondition.wait_for(lock, std::chrono::milliseconds(timeoutMs), isReady)) {
            throw Failure(G4B_ERR_TIMEOUT, "ticket not ready");
        }
        Result& slot{s->results.at(ticket)};
        if (slot.status != G4B_OK) {
            const Failure failure{slot.status, slot.message};
            s->results.erase(ticket);
            throw failure;
        }
        output->detection_count = slot.count;
        output->event_count = 1U;
        if (output->detection_capacity < slot.count || output->event_capacity < 1U ||
            (slot.count != 0U && output->detections == nullptr) || output->event_statistics == nullptr) {
            throw Failure(G4B_ERR_CAPACITY, "output buffers too small for the event");
        }
        // the detections are immutable once published: copy them out unlocked
        const Result result{std::move(slot)};
        s->results.erase(ticket);
        lock.unlock();
        if (result.count != 0U) {
            std::memcpy(output->detections, result.detections->data() + result.begin,
                        result.count * sizeof(g4b_photon_detection));
        }
        output->event_statistics[0] = result.event;
        output->statistics = result.event.statistics;
        output->performance = g4b_performance{};
    });
}

int g4b_scheduler_end_run(g4b_scheduler* s) {
    if (s == nullptr) {
        tLastError = "null scheduler";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    return Api([&]() {
        {
            std::scoped_lock lock{s->mutex};
            if (!s->started) {
                return;
            }
            s->stopRequested = true;
        }
        s->condition.notify_all();
        if (s->thread.joinable()) {
            s->thread.join();
        }
        std::scoped_lock lock{s->mutex};
        s->started = false;
    });
}

int g4b_scheduler_statistics(g4b_scheduler* s, g4b_statistics* run, g4b_batch_statistics* batch) {
    if (s == nullptr) {
        tLastError = "null scheduler";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    std::scoped_lock lock{s->mutex};
    if (run != nullptr) {
        *run = s->run;
    }
    if (batch != nullptr) {
        *batch = s->batch;
    }
    return G4B_OK;
}

int g4b_scheduler_replay(g4b_scheduler* s, const g4b_optical_emission* emissions, const uint64_t* offsets,
                         const uint32_t* eventIDs, uint32_t eventCount, uint32_t producers, uint32_t window,
                         uint64_t* detections, double* seconds) {
    if (s == nullptr || (eventCount != 0U && (offsets == nullptr || eventIDs == nullptr)) || producers == 0U ||
        window == 0U) {
        tLastError = "invalid replay arguments";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    if (eventCount != 0U && offsets[eventCount] != 0U && emissions == nullptr) {
        tLastError = "null gensteps";
        return G4B_ERR_INVALID_ARGUMENT;
    }
    std::mutex errorMutex;
    int firstStatus{G4B_OK};
    std::string firstMessage;
    std::uint64_t total{0};
    const auto record{[&](int status, std::uint64_t found) {
        std::scoped_lock lock{errorMutex};
        total += found;
        if (status != G4B_OK && firstStatus == G4B_OK) {
            firstStatus = status;
            firstMessage = tLastError;
        }
    }};
    const auto produce{[&](std::uint32_t k) {
        std::deque<std::uint64_t> outstanding;
        std::vector<g4b_photon_detection> buffer(4096);
        g4b_event_statistics event{};
        std::uint64_t found{0};
        int status{G4B_OK};
        const auto collect{[&](std::uint64_t ticket) {
            for (;;) {
                g4b_output out{};
                out.detections = buffer.data();
                out.detection_capacity = buffer.size();
                out.event_statistics = &event;
                out.event_capacity = 1U;
                const int result{g4b_scheduler_wait(s, ticket, -1, &out)};
                if (result == G4B_ERR_CAPACITY) {
                    buffer.resize(out.detection_count);
                    continue;
                }
                if (result == G4B_OK) {
                    found += out.detection_count;
                }
                return result;
            }
        }};
        for (std::uint32_t i{k}; i < eventCount && status == G4B_OK; i += producers) {
            const std::uint64_t begin{offsets[i]};
            const std::uint64_t count{offsets[i + 1U] - begin};
            std::uint64_t photons{0};
            for (std::uint64_t j{}; j < count; ++j) {
                photons += emissions[begin + j].photon_count;
            }
            std::uint64_t ticket{};
            status = g4b_scheduler_submit(s, eventIDs[i], count != 0U ? emissions + begin : nullptr,
                                          static_cast<std::uint32_t>(count), photons, nullptr, &ticket);
            if (status != G4B_OK) {
                break;
            }
            outstanding.push_back(ticket);
            if (outstanding.size() > window) {
                status = collect(outstanding.front());
                outstanding.pop_front();
            }
        }
        while (!outstanding.empty()) {
            const int result{collect(outstanding.front())};
            outstanding.pop_front();
            if (status == G4B_OK) {
                status = result;
            }
        }
        record(status, found);
    }};
    const auto start{Clock::now()};
    std::vector<std::thread> threads;
    threads.reserve(producers);
    for (std::uint32_t k{}; k < producers; ++k) {
        threads.emplace_back(produce, k);
    }
    for (auto& t : threads) {
        t.join();
    }
    if (seconds != nullptr) {
        *seconds = std::chrono::duration<double>(Clock::now() - start).count();
    }
    if (detections != nullptr) {
        *detections = total;
    }
    if (firstStatus != G4B_OK) {
        tLastError = firstMessage;
    }
    return firstStatus;
}

int g4b_scheduler_destroy(g4b_scheduler* s) {
    if (s == nullptr) {
        return G4B_OK;
    }
    const int status{g4b_scheduler_end_run(s)};
    delete s;
    return status;
}

const char* g4b_scheduler_last_error(void) { return tLastError.c_str(); }

}  // extern "C"
