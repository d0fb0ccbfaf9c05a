"""Event sharding over two gloo ranks on the CPU: the shards' combined
results equal the whole batch's, exactly (every photon is keyed by its event
and photon IDs, so where it runs does not matter)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from g4go_b200 import PhotonTransportConfig, scenes
from g4go_b200.multigpu import shard_batch, shard_bounds


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, queue):
    import torch.distributed as dist

    from g4go_b200.multigpu import allreduce_statistics, max_over_ranks
    from oracle import binding

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        scene = scenes.crystal_sipm_scene()
        batch = scenes.workload("batched", event_count=120, seed=3)
        shard = shard_batch(batch, rank, world)
        out = binding.transport(scene, shard, PhotonTransportConfig(seed=11), threads=2)
        stats = dict(out.statistics)
        total = allreduce_statistics(stats)
        slowest = max_over_ranks(float(rank + 1))
        queue.put((rank, total, slowest, out.detections.tobytes()))
    finally:
        dist.destroy_process_group()


def test_shard_bounds_balance_photons():
    batch = scenes.workload("batched", event_count=400, seed=2)
    bounds = shard_bounds(batch, 4)
    assert bounds[0][0] == 0 and bounds[-1][1] == 400
    assert all(b[1] == c[0] for b, c in zip(bounds, bounds[1:]))
    photons = [shard_batch(batch, r, 4).photon_count for r in range(4)]
    assert sum(photons) == batch.photon_count
    assert max(photons) < 1.6 * batch.photon_count / 4


def test_two_gloo_ranks_reproduce_the_whole_batch(oracle):
    world = 2
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, queue)) for r in range(world)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    scene = scenes.crystal_sipm_scene()
    batch = scenes.workload("batched", event_count=120, seed=3)
    whole = oracle.transport(scene, batch, PhotonTransportConfig(seed=11), threads=2)
    for _, total, slowest, _ in results:
        assert slowest == 2.0
        for key in ("captured_count", "detected_count", "absorbed_count", "escaped_count", "truncated_count",
                    "invalid_state_count", "max_bounce_count"):
            assert total[key] == whole.statistics[key], key
    joined = b"".join(r[3] for r in results)
    assert joined == whole.detections.tobytes()
