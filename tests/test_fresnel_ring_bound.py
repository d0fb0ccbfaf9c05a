"""The Fresnel ring of the batched transport kernel cannot overflow at 64 entries.

The form of `TransportBatched` that reads the photon store has no full-ring
fallback: it relies on a warp never holding more than 63 ring entries at the
moment its lanes park (g4go_b200/csrc/transport_kernels.cu, the parking site).
This test explores every reachable state of that bookkeeping, as the kernel
runs it per warp iteration:

1. lanes without a photon take ready entries first: `min(need, ready)` of them,
   where `need` = lanes not alive (an entry truncated by its Fresnel step leaves
   its lane without a photon);
2. lanes still without one may take fresh photons from the store, any number;
3. the step: any `k` of the alive lanes park (entries needed: ready + pending + k),
   any others finish;
4. once 32 or more are pending, 32 are completed and become ready; when no lane
   holds a photon and no fresh work is left, the pending ones are completed
   even if fewer than 32 (the draining case).

States are (alive lanes, ready, pending) at the top of the loop; the adversary
picks the choices. The largest occupancy must fit the ring size declared in
engine_layout.h, and the 40-entry ring of the other forms must be reachable
beyond 40 (which is why they keep the fallback).
"""
import re

import numpy as np

from g4go_b200 import build

LANES = 32
MAX_READY = 4 * LANES  # far above any reachable value; asserted below


def reachable_occupancy():
    reach = np.zeros((LANES + 1, MAX_READY + 1, LANES), dtype=bool)  # [alive, ready, pending]
    reach[0, 0, 0] = True
    alive = np.arange(LANES + 1)[:, None, None]
    ready = np.arange(MAX_READY + 1)[None, :, None]
    pending = np.arange(LANES)[None, None, :]
    # ready entries left after the take, per state
    left = np.maximum(ready - (LANES - alive), 0) + 0 * pending
    worst = 0
    while True:
        states = np.argwhere(reach)
        if states.size == 0:
            break
        before = reach.copy()
        a, r, p = states[:, 0], states[:, 1], states[:, 2]
        r1 = left[a, r, p]
        # fresh photons can fill every lane, so any k parkers and any number of
        # survivors up to 32 - k are possible whatever the alive count was
        for k in range(LANES + 1):
            worst = max(worst, int((r1 + p + k).max()))
            total = p + k
            completed = total >= LANES
            next_pending = np.where(completed, total - LANES, total)
            next_ready = r1 + np.where(completed, LANES, 0)
            assert next_ready.max() <= MAX_READY
            reach[: LANES - k + 1, next_ready, next_pending] = True
        # draining: nothing alive after the take (the entries taken, if any,
        # were truncated ones and the store is empty), so nobody parks and every
        # pending entry is completed
        drained = r1 + p
        assert drained.max() <= MAX_READY
        reach[0, drained, 0] = True
        if np.array_equal(before, reach):
            break
    return worst


def ring_entries(name):
    text = (build.PACKAGE / "csrc" / "engine_layout.h").read_text()
    return int(re.search(rf"constexpr std::uint32_t {name} = (\d+);", text).group(1))


def test_sixty_four_entries_hold_every_parking_step():
    worst = reachable_occupancy()
    assert worst == 2 * LANES - 1  # 31 ready or pending, plus 32 parking
    assert ring_entries("kFresnelRingEntriesPass") >= worst
    # the forms with generation in the loop can fill their ring: they keep the fallback
    assert ring_entries("kFresnelRingEntries") < worst
