"""Sharding independent worlds across GPUs (one process per GPU).

Batched worlds never interact, so a batch shards with no exchange on the data path: each rank
builds and steps only its share. The cost of a world's step grows with its body count, so the
shares are balanced by the sum of body counts, N_w: longest-processing-time greedy packing
(worlds by decreasing N_w, each to the rank with the smallest load so far, ties to the lower
rank), which keeps the largest share within 4/3 of the optimum. The partition depends only on
the sizes and the rank count, so every rank computes the same one without communicating.
The reference has no counterpart (it steps one world per process, up to MAX_WORLDS 128,
base/constants.rs:27).
"""
import heapq


def partition_worlds(sizes, ranks):
    """Split world indices 0..len(sizes)-1 into ``ranks`` shares balanced by the sum of sizes.
    Returns a list of ``ranks`` index lists, each in ascending order."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(ranks)]
    shares = [[] for _ in range(ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(s) for s in shares]


def share_loads(sizes, shares):
    """Sum of sizes of each share."""
    return [sum(int(sizes[i]) for i in s) for s in shares]
