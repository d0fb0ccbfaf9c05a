"""The header-only C++ drop-in (include/g4b_transport_host.hpp) over stand-in
C-ABI functions: its completion paths on the CPU, without a GPU.

The program defines the seven g4b_* functions the header calls. The stand-in
engine stages a batch of four events and 12 detections, and its g4b_complete
behaves as the engine's does: G4B_ERR_CAPACITY with the batch still pending when
the detection buffer is too small, otherwise detections, counts and per-event
records. The program checks CompleteOldestBatchInto (refused for a null and
for a small buffer, then filled into the caller's buffer without a count query) and
CompleteOldestBatch (query first, then a vector of the exact size).
"""
import subprocess

from g4go_b200 import build

PROGRAM = r"""
#include <cstdio>
#include <cstring>
#include <vector>

#include "g4b_transport_host.hpp"

struct g4b_handle { int pending{0}; std::uint32_t events{0}; int queries{0}; };
static g4b_handle gHandle;
constexpr std::uint64_t kDetections{12};

extern "C" {
int g4b_create(const g4b_config*, g4b_handle** out) { *out = &gHandle; return G4B_OK; }
int g4b_destroy(g4b_handle*) { return G4B_OK; }
const char* g4b_last_error(const g4b_handle*) { return "stand-in"; }
int g4b_set_scene(g4b_handle*, const g4b_scene*) { return G4B_OK; }
int g4b_enqueue(g4b_handle* h, const g4b_optical_emission*, uint32_t, const uint32_t*, uint32_t events,
                const uint32_t*) {
    h->pending = 1;
    h->events = events;
    return G4B_OK;
}
int g4b_query_oldest(g4b_handle* h, uint64_t* detections, uint32_t* events) {
    ++h->queries;
    *detections = kDetections;
    *events = h->events;
    return h->pending != 0 ? G4B_OK : G4B_ERR_LOGIC;
}
int g4b_complete(g4b_handle* h, g4b_output* out) {
    if (h->pending == 0) return G4B_ERR_LOGIC;
    if (out->event_capacity < h->events || (out->detections != nullptr && out->detection_capacity < kDetections)) {
        out->detection_count = kDetections;
        out->event_count = h->events;
        return G4B_ERR_CAPACITY;  // the batch stays pending
    }
    for (std::uint64_t i{}; i < kDetections; ++i) {
        out->detections[i] = g4b_photon_detection{};
        out->detections[i].photon_id = static_cast<uint32_t>(100 + i);
    }
    for (std::uint32_t e{}; e < h->events; ++e) {
        out->event_statistics[e] = g4b_event_statistics{};
        out->event_statistics[e].event_id = 7 * e;
        out->event_statistics[e].statistics.detected_count = 3;
    }
    out->detection_count = kDetections;
    out->event_count = h->events;
    out->statistics.detected_count = kDetections;
    h->pending = 0;
    return G4B_OK;
}
}

struct Batch {
    std::vector<g4b_optical_emission> emissions;
    std::vector<std::uint32_t> eventIDs;
    std::vector<std::uint32_t> emissionEventIndices;
};

int main() {
    g4b_config config{};
    g4b::TransportHost host{config};
    g4b_scene scene{};
    Batch batch{std::vector<g4b_optical_emission>(4), {0, 7, 14, 21}, {0, 1, 2, 3}};
    host.EnqueueEmissions(scene, batch);
    std::vector<g4b_photon_detection> buffer(16);
    g4b::TransportOutput output;
    std::uint64_t count{0};
    int nullRefused{0};
    try { host.CompleteOldestBatchInto(nullptr, 0, output, count); } catch (const std::invalid_argument&) { ++nullRefused; }
    const bool small{host.CompleteOldestBatchInto(buffer.data(), 8, output, count)};
    const bool filled{host.CompleteOldestBatchInto(buffer.data(), buffer.size(), output, count)};
    std::printf("into %d %d %d %llu %zu %zu %u %u %llu queries %d\n", nullRefused, small, filled,
                static_cast<unsigned long long>(count), output.detections.size(), output.eventStatistics.size(),
                buffer[11].photon_id, output.eventStatistics[3].event_id,
                static_cast<unsigned long long>(output.statistics.detected_count), gHandle.queries);
    int refused{0};
    try { host.CompleteOldestBatchInto(buffer.data(), buffer.size(), output, count); } catch (const std::logic_error&) { ++refused; }
    host.EnqueueEmissions(scene, batch);
    const g4b::TransportOutput whole{host.CompleteOldestBatch()};
    std::printf("whole %zu %zu %u queries %d refused %d\n", whole.detections.size(), whole.eventStatistics.size(),
                whole.detections[0].photon_id, gHandle.queries, refused);
    return 0;
}
"""


def test_completion_paths_of_the_cpp_drop_in(tmp_path):
    source = tmp_path / "host.cpp"
    source.write_text(PROGRAM)
    exe = tmp_path / "host"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-Wno-missing-field-initializers",
                    "-I", str(build.PACKAGE.parent / "include"), str(source), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    # a null buffer refused with the batch still pending, refused at capacity 8, then 12 records
    # in the caller's buffer, 4 events, no count query
    assert lines[0] == "into 1 0 1 12 0 4 111 21 12 queries 0"
    # nothing pending: a logic error; CompleteOldestBatch queries once and sizes its vector
    assert lines[1] == "whole 12 4 100 queries 1 refused 1"
