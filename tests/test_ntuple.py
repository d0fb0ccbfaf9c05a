"""CrystalHit / SensorHit rows (g4go_b200/ntuple.py and include/g4b_ntuple.hpp)
as the reference's Analysis::WriteEvent fills them
(src/simulation/Analysis.cpp:46-83, columns src/simulation/RunAction.cpp:30-43),
from a transport output's per-event statistics and detections, on the CPU."""
import subprocess

import numpy as np

from g4go_b200 import DETECTION_DTYPE, PhotonTransportConfig, build, ntuple, scenes


def handmade_output():
    detections = np.zeros(5, dtype=DETECTION_DTYPE)
    detections["event_id"] = [10, 10, 12, 12, 12]
    detections["sensor_id"] = [0, 3, 1, 1, 2]
    detections["time_ns"] = [1.25, 2.5, 3.0, 40.125, 7.0]
    statistics = [(10, {"detected_count": 2, "captured_count": 1000}),
                  (11, {"detected_count": 0, "captured_count": 50}),
                  (12, {"detected_count": 3, "captured_count": 2000})]
    deposits = [(10, 0, 0.5), (10, 1, 0.0), (11, 0, 0.25), (12, 0, 1.5), (12, 2, 0.1)]
    return detections, statistics, deposits


def test_rows_follow_the_reference_filling_rules():
    detections, statistics, deposits = handmade_output()
    crystal = ntuple.crystal_hit_rows(statistics, deposits)
    # a zero deposit writes no row; nOptPho is the event's detected count, nGenOptPho its generated count
    assert crystal.tolist() == [(10, 0, 0.5, 2, 1000), (11, 0, 0.25, 0, 50), (12, 0, 1.5, 3, 2000),
                                (12, 2, float(np.float32(0.1)), 3, 2000)]
    sensor = ntuple.sensor_hit_rows(detections)
    # no row for the event without detections; vectors in the output's order
    assert len(sensor) == 2
    event, sensors, times = sensor.row(1)
    assert event == 12 and sensors.tolist() == [1, 1, 2] and times.tolist() == [3.0, 40.125, 7.0]
    assert sensor.timeOfFlight.dtype == np.float32 and sensor.sensorID.dtype == np.int32
    generated = ntuple.crystal_hit_rows(statistics, deposits, generated_counts={10: 7, 11: 8, 12: 9})
    assert generated["nGenOptPho"].tolist() == [7, 8, 9, 9]


def test_rows_of_a_transport_output_round_trip_through_npz_and_csv(oracle, tmp_path):
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("plain_cpu", event_count=25, seed=4)
    out = oracle.transport(scene, batch, PhotonTransportConfig(seed=3, precision="fp32"))
    deposits = [(int(e), 0, 1.0) for e in batch.event_ids]
    crystal = ntuple.crystal_hit_rows(out.event_statistics, deposits)
    sensor = ntuple.sensor_hit_rows(out.detections)
    assert crystal.shape[0] == 25
    assert int(crystal["nOptPho"].sum()) == out.detections.shape[0] == sensor.sensorID.shape[0]
    assert int(crystal["nGenOptPho"].sum()) == batch.photon_count
    assert np.array_equal(sensor.timeOfFlight, out.detections["time_ns"])  # flattened order is event order
    assert set(sensor.eventID.tolist()) == {e for e, s in out.event_statistics if s["detected_count"] > 0}
    ntuple.write_npz(tmp_path / "rows.npz", crystal, sensor)
    crystal2, sensor2 = ntuple.read_npz(tmp_path / "rows.npz")
    assert np.array_equal(crystal2, crystal)
    assert all(np.array_equal(getattr(sensor2, k), getattr(sensor, k))
               for k in ("eventID", "offsets", "sensorID", "timeOfFlight"))
    crystal_csv, sensor_csv = ntuple.write_csv(tmp_path, crystal, sensor)
    lines = sensor_csv.read_text().splitlines()
    assert lines[0] == "eventID,sensorID,timeOfFlight" and len(lines) == len(sensor) + 1
    event, sensors, times = lines[1].split(",")
    assert np.array_equal(np.array(times.split(), np.float32), sensor.row(0)[2])
    assert crystal_csv.read_text().splitlines()[0] == "eventID,moduleID,Edep,nOptPho,nGenOptPho"


PROGRAM = r"""
#include <cstdio>
#include <vector>

#include "g4b_ntuple.hpp"

int main() {
    std::vector<g4b_photon_detection> detections(5);
    const unsigned events[5]{10, 10, 12, 12, 12}, sensors[5]{0, 3, 1, 1, 2};
    const float times[5]{1.25F, 2.5F, 3.0F, 40.125F, 7.0F};
    for (int i = 0; i < 5; ++i) {
        detections[i].event_id = events[i];
        detections[i].sensor_id = sensors[i];
        detections[i].time_ns = times[i];
    }
    std::vector<g4b_event_statistics> stats(3);
    const unsigned ids[3]{10, 11, 12};
    const unsigned long long detected[3]{2, 0, 3}, captured[3]{1000, 50, 2000};
    for (int i = 0; i < 3; ++i) {
        stats[i].event_id = ids[i];
        stats[i].statistics.detected_count = detected[i];
        stats[i].statistics.captured_count = captured[i];
    }
    const std::vector<g4b::EnergyDeposit> deposits{{10, 0, 0.5F}, {10, 1, 0.0F}, {11, 0, 0.25F}, {12, 0, 1.5F},
                                                   {12, 2, 0.1F}};
    for (const auto& row : g4b::CrystalHitRows(stats.data(), stats.size(), deposits)) {
        std::printf("crystal %d %d %.9g %d %d\n", row.eventID, row.moduleID, row.Edep, row.nOptPho, row.nGenOptPho);
    }
    for (const auto& row : g4b::SensorHitRows(detections.data(), detections.size())) {
        std::printf("sensor %d", row.eventID);
        for (std::size_t k = 0; k < row.sensorID.size(); ++k) {
            std::printf(" %d:%g", row.sensorID[k], row.timeOfFlight[k]);
        }
        std::printf("\n");
    }
    return 0;
}
"""


def test_cpp_rows_match_the_python_rows(tmp_path):
    source = tmp_path / "rows.cpp"
    source.write_text(PROGRAM)
    exe = tmp_path / "rows"
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I",
                    str(build.PACKAGE.parent / "include"), str(source), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    assert lines == ["crystal 10 0 0.5 2 1000", "crystal 11 0 0.25 0 50", "crystal 12 0 1.5 3 2000",
                     "crystal 12 2 0.100000001 3 2000", "sensor 10 0:1.25 3:2.5", "sensor 12 1:3 1:40.125 2:7"]
