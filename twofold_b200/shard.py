"""One set of independent worlds split over ranks, one process per GPU.

Worlds share nothing inside a step, so a shard is a list of whole worlds and the ranks exchange nothing while
they step. The split balances the work: the step's cost grows with a world's bodies, so worlds go to ranks by
greedy longest-processing-time on body counts (the heaviest world first, each to the rank with the fewest
bodies so far; ties to the lower world number and the lower rank), which keeps every rank within one world's
bodies of the others.
"""
import heapq

import numpy as np


def lpt_partition(weights, n_ranks):
    """Lists of world numbers, one per rank, each in ascending order. Deterministic for given weights."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be at least 1")
    w = np.asarray(weights, np.int64)
    order = sorted(range(len(w)), key=lambda i: (-int(w[i]), i))
    heap = [(0, r) for r in range(n_ranks)]
    shards = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(w[i]), r))
    return [sorted(s) for s in shards]


def shard_loads(weights, shards):
    w = np.asarray(weights, np.int64)
    return [int(w[s].sum()) if len(s) else 0 for s in shards]
