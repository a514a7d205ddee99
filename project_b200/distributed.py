"""Multi-GPU plumbing: one process per GPU with torch.distributed.

The propagator has no data-parallel exchange step: independent 1D instances
(a batched parameter sweep) are partitioned across ranks and each rank runs its
share in its own persistent launch; only per-instance diagnostics are gathered
afterwards.  A single 3+1D propagation does not shard (an all-to-all transpose
per 3D FFT would dominate); several ranks run independent replicas.
"""
import heapq

import torch.distributed as dist


def partition_instances(costs, world):
    """Longest-processing-time assignment of instances to ranks.

    Returns a list of index lists, one per rank; deterministic for equal inputs.
    """
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def instance_cost(Nt, L, h_est=1e-3):
    """Relative cost estimate of a 1D instance: Nt log2 Nt per attempt x attempts."""
    import math
    return Nt * math.log2(Nt) * max(L / h_est, 1.0)


def gather_results(local, group=None):
    """All-gather per-rank lists of (instance index, diagnostics dict) -> one dict."""
    world = dist.get_world_size(group)
    out = [None] * world
    dist.all_gather_object(out, local, group=group)
    merged = {}
    for part in out:
        for idx, diag in part:
            merged[idx] = diag
    return merged
