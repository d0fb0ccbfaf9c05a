"""Event sharding across GPUs (one process per GPU).

Photons and events are independent given their gensteps and RNG keys, so a
batch splits across ranks with no exchange on the data path: each rank takes
a contiguous range of events balanced by photon count, transports it on its
own GPU, and the per-rank statistics are combined at the end (counters
summed, maximum bounce count maxed). torch.distributed carries only those few
counters and the max-over-ranks timing.
"""
from __future__ import annotations

import numpy as np

from .transport import PhotonTransportBatch

COUNTERS = ("captured_count", "detected_count", "absorbed_count", "escaped_count", "truncated_count",
            "invalid_state_count", "zero_step_count")


def shard_bounds(batch: PhotonTransportBatch, world: int) -> list[tuple[int, int]]:
    """Event-index ranges [begin, end) per rank with near-equal photon counts."""
    events = batch.event_ids.shape[0]
    per_event = np.bincount(batch.emission_event_indices, weights=batch.emissions["photon_count"].astype(np.float64),
                            minlength=events)
    cumulative = np.concatenate([[0.0], np.cumsum(per_event)])
    total = cumulative[-1]
    bounds = []
    begin = 0
    for rank in range(world):
        target = total * (rank + 1) / world
        end = events if rank == world - 1 else int(np.searchsorted(cumulative, target, side="left"))
        end = max(begin, min(end, events))
        bounds.append((begin, end))
        begin = end
    return bounds


def shard_batch(batch: PhotonTransportBatch, rank: int, world: int) -> PhotonTransportBatch:
    """The rank's events and their gensteps, in batch order, re-indexed from 0."""
    begin, end = shard_bounds(batch, world)[rank]
    keep = (batch.emission_event_indices >= begin) & (batch.emission_event_indices < end)
    return PhotonTransportBatch(batch.emissions[keep], batch.event_ids[begin:end],
                                batch.emission_event_indices[keep] - begin)


def allreduce_statistics(statistics: dict, group=None) -> dict:
    """Batch statistics summed over ranks (maximum bounce count maxed)."""
    import torch
    import torch.distributed as dist

    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    sums = torch.tensor([float(statistics[k]) for k in COUNTERS], dtype=torch.float64, device=device)
    peak = torch.tensor([float(statistics["max_bounce_count"])], dtype=torch.float64, device=device)
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(peak, op=dist.ReduceOp.MAX, group=group)
    out = dict(statistics)
    for k, v in zip(COUNTERS, sums.tolist()):
        out[k] = int(v)
    out["max_bounce_count"] = int(peak.item())
    return out


def max_over_ranks(value: float, group=None) -> float:
    """The largest of a per-rank measurement (timings are taken as the slowest rank)."""
    import torch
    import torch.distributed as dist

    device = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
