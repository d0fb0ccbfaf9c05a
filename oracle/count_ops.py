"""Algorithmic operations per photon-step of the benchmark workload.

Runs the oracle's FP32 photon step instantiated with a counting number type
(oracle/count_ops.cpp, built by oracle/Makefile into _build/libopcount.so) on
photon slices spread over the 50,000-event uneven workload, and writes the
per-step counts with the lane-operation weights below to
profiles/ops_per_step.json, which bench.py reads for its issue roofline.
MEASUREMENT INFRASTRUCTURE: nothing in the engine uses it.

Weights (lane operations of a minimal GPU implementation of each counted
operation): FP32 add/multiply/compare/min-max/abs/conversion 1; FP32 divide and
square root 4 (a special-function reciprocal or reciprocal root plus Newton
refinement); FP64 operation 1; log and exp 4 (one special-function
instruction plus range handling); sin+cos of an angle 6; a uniform draw 22
(one Philox-4x32-10 block - ten rounds of two 32x32->64 multiplies, two
three-way XORs and two key additions, 80 operations, plus the conversion of
its four words to floats, 8 - per four draws, the generator's minimal use).
Integer indexing, table searches and control flow are not counted.

    python oracle/count_ops.py
"""
from __future__ import annotations

import ctypes as C
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

NAMES = ("add", "mul", "div", "fma", "sqrt", "cmp", "minmax", "cvt", "fp64", "log", "exp", "sincos", "uniform")
WEIGHTS = {"add": 1, "mul": 1, "div": 4, "fma": 1, "sqrt": 4, "cmp": 1, "minmax": 1, "cvt": 1, "fp64": 1,
           "log": 4, "exp": 4, "sincos": 6, "uniform": 22}
OUT = ROOT / "profiles" / "ops_per_step.json"


def count(events: int = 50000, slices: int = 32, photons_per_slice: int = 20000) -> dict:
    from g4go_b200 import PhotonTransportConfig, _abi, scenes

    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "_build/libopcount.so"], check=True)
    lib = C.CDLL(str(ROOT / "oracle" / "_build" / "libopcount.so"))
    lib.oracle_count_ops.restype = C.c_int
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=events, seed=1)
    c_scene = scene.to_c()
    config = PhotonTransportConfig(seed=7, precision="fp32").to_c()
    totals = [0] * len(NAMES)
    steps_total = 0
    counts = (C.c_uint64 * len(NAMES))()
    steps = C.c_uint64()
    for k in range(slices):
        begin = batch.photon_count * k // slices
        status = lib.oracle_count_ops(C.byref(c_scene.struct), C.byref(config),
                                      batch.emissions.ctypes.data_as(C.c_void_p), batch.emissions.shape[0],
                                      _abi.as_ptr(batch.emission_event_indices, C.c_uint32),
                                      batch.event_ids.shape[0], C.c_uint64(begin),
                                      C.c_uint64(begin + photons_per_slice), counts, C.byref(steps))
        if status != 0:
            raise RuntimeError(f"operation count failed ({status})")
        totals = [t + int(c) for t, c in zip(totals, counts)]
        steps_total += int(steps.value)
    per_step = {name: total / steps_total for name, total in zip(NAMES, totals)}
    ops = sum(per_step[name] * WEIGHTS[name] for name in NAMES)
    return {
        "lane_ops_per_step": round(ops, 1),
        "per_step": {name: round(value, 3) for name, value in per_step.items()},
        "weights": WEIGHTS,
        "sample": f"{slices} slices of {photons_per_slice} photons spread over the {events}-event uneven workload "
                  f"(seed 1), {steps_total} photon-steps",
        "source": "oracle/count_ops.py: the oracle's FP32 step with a counting number type",
    }


def main() -> None:
    result = count()
    OUT.write_text(json.dumps(result, indent=1) + "\n")
    print(json.dumps(result, indent=1))


if __name__ == "__main__":
    main()
