"""Regression-compatible output rows: the reference's CrystalHit and SensorHit
ntuples, as columns, without ROOT.

The reference writes two ntuples per run (src/simulation/RunAction.cpp:30-43):

    CrystalHit: eventID (I), moduleID (I), Edep (D), nOptPho (I), nGenOptPho (I)
    SensorHit:  eventID (I), sensorID (I vector), timeOfFlight (F vector)

and fills them per event as Analysis::WriteEvent does
(src/simulation/Analysis.cpp:46-83) with the event's transport output:

- one CrystalHit row per module with a positive energy deposit, in module
  order (EventAction.cpp:41-47); nOptPho is the event's detected count from
  the transport statistics (Analysis.cpp:48-50), nGenOptPho the event's
  generated photon count (EventAction.cpp:39), Edep the deposit as the float
  the reference keeps (Analysis.hpp:11-16) widened to double;
- one SensorHit row per event with at least one detection
  (Analysis.cpp:63-66): the event's detections in the transport's order, each
  giving its sensor ID and its time as float (Analysis.cpp:80-81).

Energy deposits come from Geant4's scintillator hits in a real run; they are
an input here. The columns go to .npz (numpy) or CSV (vectors as
space-separated values) for the reference's regression gates
(test/TestOpticalTransport.cxx:319-333) to read.
"""
from __future__ import annotations

import csv
from dataclasses import dataclass
from pathlib import Path
from typing import Iterable, Sequence

import numpy as np

CRYSTAL_HIT_DTYPE = np.dtype([("eventID", np.int32), ("moduleID", np.int32), ("Edep", np.float64),
                              ("nOptPho", np.int32), ("nGenOptPho", np.int32)])
DEPOSIT_DTYPE = np.dtype([("eventID", np.int32), ("moduleID", np.int32), ("Edep", np.float32)])


@dataclass
class SensorHitRows:
    """SensorHit as jagged columns: row i is eventID[i] with the vectors
    sensorID[offsets[i]:offsets[i+1]] and timeOfFlight[offsets[i]:offsets[i+1]]."""

    eventID: np.ndarray
    offsets: np.ndarray
    sensorID: np.ndarray
    timeOfFlight: np.ndarray

    def __len__(self) -> int:
        return int(self.eventID.shape[0])

    def row(self, i: int) -> tuple[int, np.ndarray, np.ndarray]:
        begin, end = int(self.offsets[i]), int(self.offsets[i + 1])
        return int(self.eventID[i]), self.sensorID[begin:end], self.timeOfFlight[begin:end]


def crystal_hit_rows(event_statistics: Iterable, deposits: np.ndarray | Sequence,
                     generated_counts: dict | None = None) -> np.ndarray:
    """CrystalHit rows of the events in `event_statistics` ([(event_id,
    statistics dict)], a transport output's), event by event in that order.

    deposits: (eventID, moduleID, Edep) records (DEPOSIT_DTYPE or tuples), one
    per module that saw a deposit, in module order within an event; rows are
    written for Edep > 0. generated_counts: event ID -> generated photon count;
    without it the event's captured count (the photons its gensteps carry,
    which the GPU path generates) stands in."""
    records = np.asarray(deposits, dtype=DEPOSIT_DTYPE) if not isinstance(deposits, np.ndarray) or \
        deposits.dtype != DEPOSIT_DTYPE else deposits
    rows = []
    for event_id, statistics in event_statistics:
        mine = records[records["eventID"] == np.int32(event_id)]
        generated = (generated_counts[event_id] if generated_counts is not None
                     else statistics["captured_count"])
        for deposit in mine:
            if deposit["Edep"] > 0:
                rows.append((event_id, int(deposit["moduleID"]), float(deposit["Edep"]),
                             int(statistics["detected_count"]), int(generated)))
    return np.array(rows, dtype=CRYSTAL_HIT_DTYPE)


def sensor_hit_rows(detections: np.ndarray) -> SensorHitRows:
    """SensorHit rows of a transport output's detections: one row per event
    with detections, in the order the events first appear, each with its
    detections' sensor IDs and times in the output's order."""
    event_ids = detections["event_id"]
    if event_ids.shape[0] == 0:
        empty = np.zeros(0, np.int32)
        return SensorHitRows(empty, np.zeros(1, np.int64), empty.copy(), np.zeros(0, np.float32))
    events, first, inverse = np.unique(event_ids, return_index=True, return_inverse=True)
    appearance = np.argsort(first, kind="stable")  # unique events in the order they first appear
    rank = np.empty_like(appearance)
    rank[appearance] = np.arange(appearance.shape[0])
    key = rank[inverse.reshape(-1)]
    order = np.argsort(key, kind="stable")  # stable: each event's detections keep the output's order
    counts = np.bincount(key, minlength=appearance.shape[0]).astype(np.int64)
    return SensorHitRows(
        eventID=events[appearance].astype(np.int32),
        offsets=np.concatenate([[0], np.cumsum(counts)]).astype(np.int64),
        sensorID=detections["sensor_id"][order].astype(np.int32),
        timeOfFlight=detections["time_ns"][order].astype(np.float32),
    )


def write_npz(path: str | Path, crystal: np.ndarray, sensor: SensorHitRows) -> None:
    """Both ntuples in one .npz: CrystalHit's columns by name, SensorHit's as
    SensorHit_eventID, SensorHit_offsets, SensorHit_sensorID and
    SensorHit_timeOfFlight."""
    np.savez(path, **{f"CrystalHit_{name}": crystal[name] for name in CRYSTAL_HIT_DTYPE.names},
             SensorHit_eventID=sensor.eventID, SensorHit_offsets=sensor.offsets,
             SensorHit_sensorID=sensor.sensorID, SensorHit_timeOfFlight=sensor.timeOfFlight)


def read_npz(path: str | Path) -> tuple[np.ndarray, SensorHitRows]:
    data = np.load(path)
    crystal = np.zeros(data["CrystalHit_eventID"].shape[0], dtype=CRYSTAL_HIT_DTYPE)
    for name in CRYSTAL_HIT_DTYPE.names:
        crystal[name] = data[f"CrystalHit_{name}"]
    sensor = SensorHitRows(data["SensorHit_eventID"], data["SensorHit_offsets"], data["SensorHit_sensorID"],
                           data["SensorHit_timeOfFlight"])
    return crystal, sensor


def write_csv(directory: str | Path, crystal: np.ndarray, sensor: SensorHitRows) -> tuple[Path, Path]:
    """CrystalHit.csv and SensorHit.csv in `directory`; SensorHit's vectors
    are space-separated within their cell; floats are written exactly
    (shortest round-tripping text)."""
    directory = Path(directory)
    directory.mkdir(parents=True, exist_ok=True)
    crystal_path = directory / "CrystalHit.csv"
    sensor_path = directory / "SensorHit.csv"
    with crystal_path.open("w", newline="") as f:
        writer = csv.writer(f)
        writer.writerow(CRYSTAL_HIT_DTYPE.names)
        for row in crystal:
            writer.writerow([int(row["eventID"]), int(row["moduleID"]), repr(float(row["Edep"])),
                             int(row["nOptPho"]), int(row["nGenOptPho"])])
    with sensor_path.open("w", newline="") as f:
        writer = csv.writer(f)
        writer.writerow(["eventID", "sensorID", "timeOfFlight"])
        for i in range(len(sensor)):
            event_id, sensors, times = sensor.row(i)
            writer.writerow([event_id, " ".join(map(str, sensors.tolist())),
                             " ".join(repr(float(t)) for t in times.tolist())])
    return crystal_path, sensor_path
