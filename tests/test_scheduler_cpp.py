"""The C++ drop-in for OpticalBatchScheduler (include/g4b_batch_scheduler.hpp),
compiled with g++ against libg4b.so and run on the CPU over a C++ stand-in
transport: Submit returns a shared future per event, the reference's
exception types come back, and every event gets its own detections."""
import subprocess

from g4go_b200 import build

PROGRAM = r"""
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

#include "g4b_batch_scheduler.hpp"

// One pending batch; emission j yields photon_count / 10 detections.
struct Fake {
    std::vector<g4b_optical_emission> emissions;
    std::vector<uint32_t> ids, indices;
    bool pending{false};
    std::string error{"none"};
};

static int Enqueue(void* c, const g4b_optical_emission* e, uint32_t n, const uint32_t* ids, uint32_t events,
                   const uint32_t* idx) {
    auto* f = static_cast<Fake*>(c);
    if (f->pending) { f->error = "transport queue is full"; return G4B_ERR_LOGIC; }
    f->emissions.assign(e, e + n);
    f->ids.assign(ids, ids + events);
    f->indices.assign(idx, idx + n);
    f->pending = true;
    return G4B_OK;
}
static int Poll(void*, int* ready) { *ready = 1; return G4B_OK; }
static int Query(void* c, uint64_t* d, uint32_t* events) {
    auto* f = static_cast<Fake*>(c);
    uint64_t total = 0;
    for (const auto& e : f->emissions) total += e.photon_count / 10;
    *d = total;
    *events = static_cast<uint32_t>(f->ids.size());
    return G4B_OK;
}
static int Complete(void* c, g4b_output* out) {
    auto* f = static_cast<Fake*>(c);
    const uint32_t terminal = (1u << G4B_FIELD_DETECTED) | (1u << G4B_FIELD_ABSORBED);
    g4b_statistics batch{};
    batch.valid_fields = terminal;
    uint64_t row = 0;
    for (uint32_t i = 0; i < f->ids.size(); ++i) {
        g4b_event_statistics& record = out->event_statistics[i];
        record = g4b_event_statistics{};
        record.event_id = f->ids[i];
        record.statistics.valid_fields = terminal;
    }
    for (size_t j = 0; j < f->emissions.size(); ++j) {
        const auto& e = f->emissions[j];
        auto& s = out->event_statistics[f->indices[j]].statistics;
        for (uint32_t k = 0; k < e.photon_count / 10; ++k) {
            g4b_photon_detection d{};
            d.event_id = e.event_id;
            d.photon_id = e.first_photon_id + k;
            out->detections[row++] = d;
        }
        s.detected_count += e.photon_count / 10;
        s.absorbed_count += e.photon_count - e.photon_count / 10;
        batch.detected_count += e.photon_count / 10;
        batch.absorbed_count += e.photon_count - e.photon_count / 10;
    }
    out->detection_count = row;
    out->event_count = static_cast<uint32_t>(f->ids.size());
    out->statistics = batch;
    f->pending = false;
    return G4B_OK;
}
static const char* LastError(void* c) { return static_cast<Fake*>(c)->error.c_str(); }

static std::vector<g4b_optical_emission> Event(uint32_t id) {
    std::vector<g4b_optical_emission> e(3);
    for (uint32_t j = 0; j < 3; ++j) {
        e[j] = g4b_optical_emission{};
        e[j].event_id = id;
        e[j].photon_count = 20 + 10 * j + id;
        e[j].first_photon_id = 1000 * j;
    }
    return e;
}

int main() {
    Fake a, b;
    std::vector<g4b_transport_ops> ops{{&a, Enqueue, Poll, Query, Complete, LastError},
                                       {&b, Enqueue, Poll, Query, Complete, LastError}};
    g4b_scheduler_config batching{};
    batching.target_photons_per_batch = 500;
    batching.batch_collection_timeout_ms = 1;
    g4b::BatchScheduler scheduler{ops, batching};
    scheduler.BeginRun();
    std::atomic<int> good{0}, bad{0};
    std::vector<std::thread> threads;
    for (uint32_t t = 0; t < 3; ++t) {
        threads.emplace_back([&, t]() {
            std::vector<std::pair<uint32_t, g4b::TransportFuture>> futures;
            for (uint32_t id = t; id < 60; id += 3) {
                auto e = Event(id);
                uint64_t photons = 0;
                for (const auto& x : e) photons += x.photon_count;
                futures.emplace_back(id, scheduler.Submit(id, e, photons));
            }
            for (auto& [id, future] : futures) {
                const auto& out = future.get();
                uint64_t want = 0;
                for (const auto& x : Event(id)) want += x.photon_count / 10;
                bool ok = out.detections.size() == want && out.statistics.detected_count == want;
                for (const auto& d : out.detections) ok = ok && d.event_id == id;
                (ok ? good : bad)++;
            }
        });
    }
    for (auto& t : threads) t.join();
    bool threw = false;
    try {
        auto e = Event(99);
        scheduler.Submit(99, e, 1);  // photon count does not match the emissions
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    scheduler.EndRun();
    const auto stats = scheduler.BatchStatistics();
    std::printf("%d %d %d %llu\n", good.load(), bad.load(), threw ? 1 : 0,
                static_cast<unsigned long long>(stats.event_count));
    return 0;
}
"""


def test_cpp_batch_scheduler_shim_runs_over_a_stand_in_transport(tmp_path):
    library = build.build()
    source = tmp_path / "scheduler_shim.cpp"
    source.write_text(PROGRAM)
    exe = tmp_path / "scheduler_shim"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-pthread",
                    "-I", str(build.PACKAGE.parent / "include"), str(source), "-o", str(exe),
                    str(library), f"-Wl,-rpath,{library.parent}"], check=True)
    result = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120)
    good, bad, threw, events = map(int, result.stdout.split())
    assert (good, bad, threw, events) == (60, 0, 1, 60)
