// g4b_ntuple.hpp - the reference's CrystalHit and SensorHit ntuple rows from
// the engine's output records, header-only, without ROOT.
//
// Columns as src/simulation/RunAction.cpp:30-43 declares them:
//   CrystalHit: eventID (int), moduleID (int), Edep (double), nOptPho (int), nGenOptPho (int)
//   SensorHit:  eventID (int), sensorID (vector<int>), timeOfFlight (vector<float>)
// filled as Analysis::WriteEvent does (src/simulation/Analysis.cpp:46-83):
//   - one CrystalHit row per module with a positive energy deposit, modules
//     in the order given (EventAction.cpp:41-47); nOptPho = the event's
//     detected count, nGenOptPho = its generated photon count (the captured
//     count of the engine's per-event statistics stands in when the caller
//     has no separate count: the GPU path generates every captured photon);
//   - one SensorHit row per event with at least one detection, its sensor IDs
//     and times in the output's order.
// A caller writes the rows with whatever it has (ROOT where it exists,
// CSV or numpy otherwise); g4go_b200/ntuple.py is the same in Python.
#pragma once

#include <cstddef>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "g4b.h"

namespace g4b {

struct EnergyDeposit {
    int eventID;
    int moduleID;
    float energyDeposit;  // the reference keeps it as float (Analysis.hpp:11-16)
};

struct CrystalHitRow {
    int eventID;
    int moduleID;
    double Edep;
    int nOptPho;
    int nGenOptPho;
};

struct SensorHitRow {
    int eventID;
    std::vector<int> sensorID;
    std::vector<float> timeOfFlight;
};

// Rows for the events of `statistics` (a completed batch's per-event
// records), event by event in that order. `deposits` lists the modules with
// a deposit per event, in module order; rows are written for deposits above
// zero.
inline std::vector<CrystalHitRow> CrystalHitRows(const g4b_event_statistics* statistics, std::size_t eventCount,
                                                 const std::vector<EnergyDeposit>& deposits) {
    std::unordered_map<int, std::vector<const EnergyDeposit*>> byEvent;
    for (const auto& deposit : deposits) {
        byEvent[deposit.eventID].push_back(&deposit);
    }
    std::vector<CrystalHitRow> rows;
    for (std::size_t e{}; e < eventCount; ++e) {
        const int eventID{static_cast<int>(statistics[e].event_id)};
        const auto found{byEvent.find(eventID)};
        if (found == byEvent.end()) {
            continue;
        }
        for (const EnergyDeposit* deposit : found->second) {
            if (deposit->energyDeposit > 0.0F) {
                rows.push_back({eventID, deposit->moduleID, static_cast<double>(deposit->energyDeposit),
                                static_cast<int>(statistics[e].statistics.detected_count),
                                static_cast<int>(statistics[e].statistics.captured_count)});
            }
        }
    }
    return rows;
}

// One row per event with detections, in the order the events first appear.
inline std::vector<SensorHitRow> SensorHitRows(const g4b_photon_detection* detections, std::size_t count) {
    std::vector<SensorHitRow> rows;
    std::unordered_map<std::uint32_t, std::size_t> rowOf;
    for (std::size_t i{}; i < count; ++i) {
        const auto [entry, added]{rowOf.emplace(detections[i].event_id, rows.size())};
        if (added) {
            rows.push_back({static_cast<int>(detections[i].event_id), {}, {}});
        }
        auto& row{rows[entry->second]};
        row.sensorID.push_back(static_cast<int>(detections[i].sensor_id));
        row.timeOfFlight.push_back(detections[i].time_ns);
    }
    return rows;
}

}  // namespace g4b
