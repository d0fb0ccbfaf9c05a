#!/usr/bin/env python
"""Optical photons traced per second on B200: the batched FP32 engine on the
uneven-event workload, next to the plain one-event-per-launch FP64 form and
the CPU port of the reference algorithm.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (launched by torchrun for N > 1); every rank transports
its own seeded copy of the workload (weak scaling: events are independent, no
data-path collective). A step is one pass of the transport over the batch.
`value` times the device path with the gensteps already in HBM
(g4b_relaunch); `e2e` times the public API with host buffers (g4b_enqueue
with the host-to-device copy of the gensteps, g4b_complete with the ordered
detections copied back to pinned host memory). Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Optical photons traced/s on 1 B200: batched FP32 vs plain form, same accuracy"
UNIT = "photons/s"
WORKLOAD_TEXT = ("50,000 e- events, energy log-uniform 0.1-20 MeV, entry uniform on the 3x3 mm face, incidence "
                 "uniform to 30 deg, 10,000 ph/MeV scintillation (40 ns, 420+-20 nm) + Cerenkov (n=1.82); "
                 "3x3x10 mm crystal, 0.95 specular wrapper, 0.1 mm n=1.41 grease, SiPM PDE 0.3")


def parse_args():
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=["ours", "reference"], default="ours")
    parser.add_argument("--events", type=int, default=50000, help="events per rank (the workload has 50,000)")
    parser.add_argument("--plain-events", type=int, default=1000,
                        help="events of the same workload timed in the plain FP64 form")
    parser.add_argument("--plain-repeats", type=int, default=5,
                        help="relaunches of the plain FP64 form; the median is reported")
    parser.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample length")
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-plain", action="store_true")
    parser.add_argument("--no-e2e", action="store_true")
    parser.add_argument("--no-autotune", action="store_true")
    parser.add_argument("--no-scheduler", action="store_true")
    parser.add_argument("--scheduler-events", type=int, default=5000,
                        help="events of the same workload streamed through the batch scheduler")
    return parser.parse_args()


def scheduler_leg(scene, events: int, local: int, producers: int = 8, window: int = 64) -> dict:
    """Events streamed one at a time through the batch scheduler
    (include/g4b_scheduler.h) by `producers` native threads
    (g4b_scheduler_replay), each keeping at most `window` results
    outstanding (the reference's maxPendingEvents per worker,
    PhotonTransportConfig.hpp:36): pipelined (eight batches in flight) and in the reference's
    serial order, both at the reference's batch target. Host wall clock from the first submission to the last result:
    the median of three passes after one warm-up pass, with the spread."""
    from g4go_b200 import PhotonTransportConfig, scenes
    from g4go_b200.scheduler import BatchSchedulerConfig, OpticalBatchScheduler, OpticalSubmission

    batch = scenes.workload("batched", event_count=events, seed=5)
    indices = batch.emission_event_indices
    if np.any(np.diff(indices.astype(np.int64)) < 0):
        order = np.argsort(indices, kind="stable")
        emissions, indices = batch.emissions[order], indices[order]
    else:
        emissions = batch.emissions
    bounds = np.searchsorted(indices, np.arange(len(batch.event_ids) + 1))
    submissions = [OpticalSubmission(int(event_id), emissions[bounds[i]:bounds[i + 1]])
                   for i, event_id in enumerate(batch.event_ids)]
    photons = int(sum(sub.photon_count for sub in submissions))
    out = {"unit": UNIT, "events": len(submissions), "photons": photons, "producers": producers,
           "window": window,
           "timing": "host wall clock, first submission to last result; median of three passes after a warm-up pass"}
    runs = (("pipelined", BatchSchedulerConfig(enable_performance_diagnostics=True)),
            ("serial", BatchSchedulerConfig(serial=True, enable_performance_diagnostics=True)))
    for name, batching in runs:
        config = PhotonTransportConfig(seed=7, device=local)
        with OpticalBatchScheduler(config, scene, batching) as scheduler:
            scheduler.replay(submissions, producers, window)  # warm-up: engine handles, graphs, staging
            passes = []
            for _ in range(3):
                before = scheduler.batch_statistics()
                detections, seconds = scheduler.replay(submissions, producers, window)
                after = scheduler.batch_statistics()
                passes.append((seconds, detections, before, after))
            passes.sort(key=lambda run: run[0])
            seconds, detections, before, after = passes[1]  # the median pass
        out[name] = {"value": photons / seconds, "seconds": seconds, "detections": detections,
                     "pass_seconds": [run[0] for run in passes],
                     "target_photons_per_batch": batching.target_photons_per_batch,
                     "batches": after["batch_count"] - before["batch_count"],
                     "overlapped_batches": after["overlapped_batch_count"] - before["overlapped_batch_count"],
                     "kernel_ms": after["performance"]["kernel_ms"] - before["performance"]["kernel_ms"],
                     "transport_thread_ms": {key: after[f"scheduler_{key}_ms"] - before[f"scheduler_{key}_ms"]
                                             for key in ("input_wait", "gpu_wait", "batch_flatten")}}
    out["value"] = out["pipelined"]["value"]
    return out


def distributed():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.device_index = device_index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None
        self._thread = None

    def start(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._proc = None
            return
        self._thread = threading.Thread(target=self._read, daemon=True)
        self._thread.start()

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        mhz = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        max_mhz = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {
            "sm_mhz": statistics.median(mhz) if mhz else None,
            "sm_max_mhz": max(max_mhz) if max_mhz else None,
            "reasons": reasons,
            "samples": len(self.samples),
        }


def measured_peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return data, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def profile_inputs():
    """Per-photon-step instruction count and DRAM traffic per photon from the
    committed ncu summary of the batched FP32 kernel, and the algorithmic
    operations per photon-step counted by oracle/count_ops.py (profiles/)."""
    data = {}
    path = ROOT / "profiles" / "roofline_inputs.json"
    if path.exists():
        data.update(json.loads(path.read_text()))
    ops = ROOT / "profiles" / "ops_per_step.json"
    if ops.exists():
        counted = json.loads(ops.read_text())
        data["algorithmic_ops_per_step"] = counted["lane_ops_per_step"]
        data["algorithmic_source"] = counted["source"]
    return data


def run_oracle_sample(batch, scene, seconds: float, seed: int, slices: int = 16):
    """The CPU port (FP64, all host threads, one transport per slice) on
    `slices` photon slices spread evenly over the whole batch, grown until
    about `seconds` of work, so the sample has the workload's mix of event
    sizes and energies. Returns (photons, seconds, threads)."""
    from g4go_b200 import PhotonTransportConfig
    from oracle import binding

    config = PhotonTransportConfig(seed=seed, precision="fp64")
    threads = os.cpu_count() or 1
    ends = np.cumsum(batch.emissions["photon_count"], dtype=np.int64)
    total = int(ends[-1]) if ends.size else 0

    def transport_slice(begin, end):
        # the slice's own gensteps: its photons take the same histories as in
        # the whole batch, without the whole batch's per-call checks
        part, inside = batch.photon_slice(begin, end, ends)
        binding.transport(scene, part, config, threads=threads, photon_range=inside)

    starts = [total * k // slices for k in range(slices)]
    per_slice = 12_500
    photons = 0
    elapsed = 0.0
    offset = [0] * slices
    while elapsed < seconds:
        grew = False
        for k, start in enumerate(starts):
            limit = (starts[k + 1] if k + 1 < slices else total)
            begin = start + offset[k]
            end = min(begin + per_slice, limit)
            if end <= begin:
                continue
            t0 = time.perf_counter()
            transport_slice(begin, end)
            elapsed += time.perf_counter() - t0
            photons += end - begin
            offset[k] += end - begin
            grew = True
        if not grew:
            break
        if elapsed < seconds / 8:
            per_slice *= 2
    return photons, elapsed, threads


def bench_reference(args, world, rank):
    """Reference arm: the CPU port of the reference's algorithm on the host
    cores, on the same workload as our arm (the full batch of args.events
    events), each step a bounded sample of photon slices spread over it."""
    if rank != 0:
        return
    from g4go_b200 import scenes

    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=args.events, seed=1)
    step_seconds = max(2.0, min(10.0, 60.0 / max(args.steps + args.warmup, 1)))
    for _ in range(args.warmup):
        run_oracle_sample(batch, scene, step_seconds / 4, seed=7)
    photons = 0
    elapsed = 0.0
    threads = os.cpu_count() or 1
    per_step = []
    for _ in range(args.steps):
        p, e, threads = run_oracle_sample(batch, scene, step_seconds, seed=7)
        photons += p
        elapsed += e
        per_step.append(p / e)
    value = photons / elapsed
    sample = (f"{photons / args.steps:.3g} photons per step in 16 slices spread evenly over the "
              f"{batch.event_ids.shape[0]}-event, {batch.photon_count:.3g}-photon batch "
              f"(FP64 CPU port, one transport of each slice's gensteps, {threads} threads)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD_TEXT, "events_per_gpu": int(batch.event_ids.shape[0]),
                   "photons_per_gpu": int(batch.photon_count),
                   "impl": "oracle port (the reference's CPU path is Geant4, not installed here)"},
        "step_values": {"median": statistics.median(per_step), "min": min(per_step), "max": max(per_step)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def bench_ours(args, world, rank, local):
    import torch

    from g4go_b200 import DETECTION_DTYPE, PhotonTransportConfig, TransportHost, scenes
    from g4go_b200 import _abi
    from g4go_b200.multigpu import max_over_ranks

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    scene = scenes.crystal_sipm_scene()
    t0 = time.perf_counter()
    batch = scenes.workload("batched", event_count=args.events, seed=1 + rank, first_event_id=rank * args.events)
    synth_seconds = time.perf_counter() - t0
    photons = batch.photon_count
    emissions = batch.emissions.shape[0]
    events = batch.event_ids.shape[0]

    # Autotune the launch shape on a sample of the workload (block size x blocks/SM x queue chunk).
    tuned = {}
    if not args.no_autotune:
        sample = scenes.workload("batched", event_count=min(2000, args.events), seed=1 + rank)
        with TransportHost(PhotonTransportConfig(seed=7, device=local)) as tuner:
            tuner.enqueue_emissions(scene, sample)
            tuner.complete_oldest_batch(counts_only=True)
            tuned = tuner.autotune(repeats=2)
    config = PhotonTransportConfig(
        seed=7, device=local, precision="fp32", launch_form="batched", use_cuda_graph=True,
        block_size=tuned.get("block_size", 0), blocks_per_sm=tuned.get("blocks_per_sm", 0),
        chunk_photons=tuned.get("chunk_photons", 0),
    )
    host = TransportHost(config)
    stream = torch.cuda.ExternalStream(host.stream, device=torch.device("cuda", local))

    # Stage the batch (host -> device once) and warm up.
    host.enqueue_emissions(scene, batch)
    first = host.complete_oldest_batch(counts_only=True)
    hits_per_step = first.statistics["detected_count"]
    bounces = first.performance["total_bounce_count"]
    for _ in range(max(args.warmup - 1, 0)):
        host.relaunch()
        host.complete_oldest_batch(counts_only=True)

    # Timed device path: K relaunches on the resident gensteps.
    sampler = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    launches = 0
    start.record(stream)
    for _ in range(args.steps):
        host.relaunch()
        out = host.complete_oldest_batch(counts_only=True)
        kernel_ms.append(out.performance["kernel_ms"])
        launches += out.performance["kernel_launch_count"]
        if out.statistics["detected_count"] != hits_per_step:
            raise RuntimeError("relaunch is not deterministic")
    stop.record(stream)
    torch.cuda.synchronize()
    sampler.stop()
    elapsed_ms = start.elapsed_time(stop)
    if world > 1:
        elapsed_ms = max_over_ranks(elapsed_ms)
    ms_per_step = elapsed_ms / args.steps
    value = photons * world / (ms_per_step / 1000.0)

    # End to end through the public API: host gensteps in, ordered detections back to pinned memory.
    e2e = None
    if not args.no_e2e:
        pinned = C_pinned(_abi, max(hits_per_step, 1) * DETECTION_DTYPE.itemsize)
        detections = np.frombuffer(pinned.buffer, dtype=DETECTION_DTYPE)
        host_emissions = C_pinned(_abi, emissions * 128)
        staged = np.frombuffer(host_emissions.buffer, dtype=_abi.EMISSION_DTYPE)
        staged[:] = batch.emissions
        from g4go_b200 import PhotonTransportBatch

        pinned_batch = PhotonTransportBatch(staged, batch.event_ids, batch.emission_event_indices)
        host.enqueue_emissions(scene, pinned_batch)
        host.complete_oldest_batch(detections_out=detections)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e2e_start = torch.cuda.Event(enable_timing=True)
        e2e_stop = torch.cuda.Event(enable_timing=True)
        e2e_steps = max(1, min(args.steps, 3))
        e2e_start.record(stream)
        h2d = d2h = 0
        for _ in range(e2e_steps):
            host.enqueue_emissions(scene, pinned_batch)
            out = host.complete_oldest_batch(detections_out=detections)
            h2d = out.performance["host_to_device_bytes"]
            d2h = out.performance["device_hits_to_host_bytes"] + out.performance["device_metadata_to_host_bytes"]
        e2e_stop.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e2e_start.elapsed_time(e2e_stop) / e2e_steps
        if world > 1:
            e2e_ms = max_over_ranks(e2e_ms)
        e2e = {"value": photons * world / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms}
        del detections, staged, pinned_batch
        pinned.free()
        host_emissions.free()

    # The plain form: one event per launch, one thread per photon, FP64, on the first events of the workload.
    plain = None
    if not args.no_plain and rank == 0:
        plain_batch = scenes.workload("batched", event_count=min(args.plain_events, args.events), seed=1 + rank)
        plain_runs = []
        with TransportHost(PhotonTransportConfig(seed=7, device=local, precision="fp64", launch_form="plain")) as ph:
            ph.enqueue_emissions(scene, plain_batch)
            ph.complete_oldest_batch(counts_only=True)
            pstream = torch.cuda.ExternalStream(ph.stream, device=torch.device("cuda", local))
            for _ in range(args.plain_repeats):
                ps = torch.cuda.Event(enable_timing=True)
                pe = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                ps.record(pstream)
                ph.relaunch()
                pout = ph.complete_oldest_batch(counts_only=True)
                pe.record(pstream)
                torch.cuda.synchronize()
                plain_runs.append(ps.elapsed_time(pe))
        plain_ms = statistics.median(plain_runs)
        plain = {"value": plain_batch.photon_count / (plain_ms / 1000.0), "unit": UNIT,
                 "events": int(plain_batch.event_ids.shape[0]), "photons": int(plain_batch.photon_count),
                 "ms": plain_ms, "ms_runs": plain_runs, "timing": f"median of {len(plain_runs)} relaunches",
                 "launches": int(pout.performance["kernel_launch_count"])}

    clocks = sampler.summary()
    host.close()

    streamed = None
    if not args.no_scheduler and rank == 0 and world == 1:
        streamed = scheduler_leg(scene, min(args.scheduler_events, args.events), local)

    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        cpu_photons, cpu_seconds, cores = run_oracle_sample(batch, scene, args.cpu_seconds, seed=7)
        cpu = {"value": cpu_photons / cpu_seconds, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{cpu_photons} photons in 16 slices spread evenly over the workload's batch, FP64 CPU "
                         f"port of the reference algorithm, one transport of each slice's gensteps, {cores} threads, "
                         f"{cpu_seconds:.1f} s"}

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    peaks, peak_kind = measured_peaks()
    kernel_mean_ms = sum(kernel_ms) / len(kernel_ms)
    # the path's own bytes: every genstep with its offset and event index, one
    # 48-B detection per hit, one counter record per event, the run counters;
    # the generation pass's photon stores are this engine's choice, not the
    # algorithm's, and show up in `traffic` only
    algorithmic_bytes = emissions * (128 + 4 + 4) + 4 + hits_per_step * 48 + events * 64 + 64
    achieved_gbs = algorithmic_bytes / (kernel_mean_ms / 1000.0) / 1e9
    prof = profile_inputs()
    traffic = None
    if "dram_bytes_per_photon" in prof:
        traffic = prof["dram_bytes_per_photon"] * photons
    roofline = {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved_gbs / peaks["hbm_gbs"], "traffic": traffic,
                "peak_kind": f"{peak_kind} (STREAM copy)",
                "note": "the transport is instruction-issue bound; see issue_roofline"}
    steps_per_s = bounces / (kernel_mean_ms / 1000.0)
    issue = None
    clock_mhz = clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
    if "algorithmic_ops_per_step" in prof:
        # the binding roofline: the algorithm's own operations per photon-step
        # (oracle/count_ops.py) at the photon-steps/s achieved, against every
        # lane of every scheduler issuing one operation per clock
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        peak_ops = sms * 4 * 32 * clock_mhz * 1e6
        achieved_ops = steps_per_s * prof["algorithmic_ops_per_step"]
        issue = {"achieved": achieved_ops, "peak": peak_ops, "unit": "lane-operations/s",
                 "frac": achieved_ops / peak_ops, "ops_per_step": prof["algorithmic_ops_per_step"],
                 "basis": "algorithmic operations per photon-step", "sm_mhz": clock_mhz,
                 "source": prof.get("algorithmic_source")}
        if "lane_ops_per_step" in prof:
            executed = steps_per_s * prof["lane_ops_per_step"]
            issue["executed"] = {"lane_instructions_per_step": prof["lane_ops_per_step"],
                                 "frac": executed / peak_ops, "source": prof.get("source"),
                                 "note": "issue utilisation from the executed lane-instructions of an ncu capture"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {
            "workload": WORKLOAD_TEXT, "events_per_gpu": events, "gensteps_per_gpu": emissions,
            "photons_per_gpu": photons, "form": "batched persistent kernel, device work queue, CUDA graph",
            "precision": "fp32 transport, fp64 global time and TIR test",
            "launch": {"block_size": host.config.block_size or tuned.get("block_size"),
                       "blocks_per_sm": tuned.get("blocks_per_sm"), "chunk_photons": tuned.get("chunk_photons"),
                       "autotune_best_ms_on_sample": tuned.get("best_ms")},
            "l2": "inputs larger than L2: %.0f MB of gensteps per step" % (emissions * 128 / 1e6),
            "synthesis_seconds": synth_seconds,
        },
        "e2e": e2e,
        "roofline": roofline,
        "issue_roofline": issue,
        "photon_steps_per_s": steps_per_s * world,
        "mean_steps_per_photon": bounces / photons,
        "detected_fraction": hits_per_step / photons,
        "kernel_ms": kernel_mean_ms,
        "kernel_ms_steps": {"median": statistics.median(kernel_ms), "min": min(kernel_ms), "max": max(kernel_ms)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "plain_fp64": plain,
        "batched_over_plain": (value / world / plain["value"]) if plain else None,
        "cpu_baseline": cpu,
        "scheduler": streamed,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


class C_pinned:
    """Page-locked host buffer from the engine (g4b_host_alloc)."""

    def __init__(self, abi, nbytes: int):
        import ctypes as C

        self._abi = abi
        self._lib = abi.load()
        self.pointer = C.c_void_p()
        status = self._lib.g4b_host_alloc(nbytes, C.byref(self.pointer))
        if status != 0:
            raise RuntimeError("g4b_host_alloc failed")
        self.buffer = (C.c_ubyte * nbytes).from_address(self.pointer.value)

    def free(self):
        if self.pointer:
            self.buffer = None
            self._lib.g4b_host_free(self.pointer)
            self.pointer = None


def main():
    args = parse_args()
    world, rank, local = distributed()
    if args.impl == "reference":
        bench_reference(args, world, rank)
        return
    bench_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
