"""Host side of the batching form across GPUs: which systems each GPU takes.

Independent periodic systems shard across GPUs with no exchange on the data path: each rank (one process per GPU) takes
a disjoint subset of the systems, balanced by atom count, and evaluates its subset as one batch in its own engine
context. Results are gathered on the host only when the caller wants them in one place (bench.py and the tests).
"""
import numpy as np


def shard_systems(sizes, world, rank):
    """Indices of the systems rank `rank` of `world` evaluates.

    Longest-processing-time greedy on atom counts: systems in decreasing size (ties by index) go to the rank with the
    fewest atoms so far (ties by rank). Deterministic, so every rank computes the same partition without communicating.
    Every system lands on exactly one rank; indices come back in increasing order.
    """
    if world < 1 or not (0 <= rank < world):
        raise ValueError("need world >= 1 and 0 <= rank < world")
    sizes = np.asarray(sizes, dtype=np.int64)
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k))
    load = [0] * world
    owner = np.empty(len(sizes), dtype=np.int64)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += int(sizes[k])
    return [k for k in range(len(sizes)) if owner[k] == rank]


def shard_loads(sizes, world):
    """Atoms per rank under shard_systems."""
    return [int(sum(int(sizes[k]) for k in shard_systems(sizes, world, r))) for r in range(world)]
