"""Request routing of the multi-GPU serving pool, on the CPU with a fake
device list (no GPU: zkmsm_route_pick is pure host logic in the library).

A pool holds one commitment server per GPU, each over its own resident
tables; a request goes whole to one replica.  The rule: replicas without a
table for the curve, with a table shorter than the request or with a budget
that can never hold it are skipped; one with free budget for the request now
beats one without; then the shallowest queue (points submitted and not
finished, divided by the replica's relative speed); among replicas that all
lack room, then the most free budget; then the first replica in cyclic order
from a rotating start (so full ties spread over the replicas).
"""
import random

import pytest

from zkmetal_b200 import route_pick

GB = 1 << 30


def rep(queued=0, budget=64 * GB, in_use=0, table=1 << 22, has=1, speed=1.0):
    return {"has_table": has, "table_points": table, "queued_points": queued, "budget_bytes": budget,
            "in_use_bytes": in_use, "relative_speed": speed}


def test_shallowest_queue_wins_and_ties_rotate():
    assert route_pick([rep(), rep()], 1000, GB) == 0
    assert route_pick([rep(), rep()], 1000, GB, first=1) == 1
    assert route_pick([rep(), rep(), rep()], 1000, GB, first=5) == 2
    assert route_pick([rep(queued=5000), rep(queued=10)], 1000, GB) == 1
    assert route_pick([rep(queued=7), rep(queued=7), rep(queued=3)], 1, 1) == 2
    assert route_pick([rep(queued=3), rep(queued=7), rep(queued=3)], 1, 1, first=1) == 2


def test_replicas_that_cannot_take_the_request_are_skipped():
    assert route_pick([rep(has=0), rep(queued=1 << 30)], 100, GB) == 1
    assert route_pick([rep(table=1000), rep(queued=1 << 30)], 1001, GB) == 1
    assert route_pick([rep(budget=GB), rep(queued=1 << 30, budget=8 * GB)], 100, 2 * GB) == 1
    assert route_pick([rep(has=0), rep(table=10), rep(budget=1)], 100, 2) == -1
    assert route_pick([], 1, 1) == -1


def test_free_memory_now_beats_a_shallower_queue():
    full = rep(queued=0, budget=8 * GB, in_use=7 * GB)
    busy = rep(queued=1 << 24, budget=8 * GB, in_use=0)
    assert route_pick([full, busy], 1 << 20, 2 * GB) == 1
    # neither has room now: the shallower queue waits for memory
    assert route_pick([rep(queued=9, budget=8 * GB, in_use=7 * GB), rep(queued=5, budget=8 * GB, in_use=7 * GB)],
                      10, 2 * GB) == 1
    # equal depth, neither with room: more free budget
    assert route_pick([rep(budget=8 * GB, in_use=7 * GB), rep(budget=8 * GB, in_use=int(6.5 * GB))], 10,
                      2 * GB) == 1
    # equal depth, both with room: the rotation decides, not the free budget
    assert route_pick([rep(in_use=3 * GB), rep(in_use=GB)], 10, GB) == 0
    assert route_pick([rep(in_use=3 * GB), rep(in_use=GB)], 10, GB, first=1) == 1


def test_relative_speed_scales_the_queue():
    assert route_pick([rep(queued=1000, speed=2.0), rep(queued=600, speed=1.0)], 100, 1) == 0


@pytest.mark.parametrize("n_gpus", [2, 4, 8])
def test_simulated_stream_balances_replicas(n_gpus):
    """A Poisson-like stream of mixed sizes over identical fake replicas that
    drain their queues at the same rate: routed work stays balanced and no
    request is refused."""
    rng = random.Random(n_gpus)
    reps = [rep(budget=100 * GB) for _ in range(n_gpus)]
    routed = [0] * n_gpus
    for k in range(4000):
        n = int(2 ** rng.uniform(10, 22))
        i = route_pick(reps, n, n * 200 + (64 << 20), first=k)
        assert i >= 0
        reps[i]["queued_points"] += n
        routed[i] += n
        for r in reps:  # every replica retires work at the same speed
            r["queued_points"] = max(0, r["queued_points"] - (1 << 19))
    assert max(routed) / min(routed) < 1.2, routed
