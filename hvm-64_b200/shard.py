"""Sharding a batch of independent nets over ranks (one process per GPU).

Nets never share nodes, so a batch splits into per-rank sub-batches with no
communication while they reduce.  Each rank gets a size-balanced share
(longest-processing-time greedy on the predicted interaction count), reduces
it on its own GPU, and rank 0 collects the per-net results; the step time is
the slowest rank's.
"""
import heapq


def lpt_partition(costs, parts):
    """Indices of `costs` split into `parts` lists with nearly equal sums:
    largest first, each to the currently lightest part.  Deterministic, so
    every rank computes the same split without talking."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    heap = [(0.0, p) for p in range(parts)]
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, p = heapq.heappop(heap)
        out[p].append(i)
        heapq.heappush(heap, (load + costs[i], p))
    for o in out:
        o.sort()
    return out


def rank_share(entries, cost, rank, world):
    """This rank's entries of a global batch."""
    parts = lpt_partition([cost(e) for e in entries], world)
    return [entries[i] for i in parts[rank]]


def max_over_ranks(value, dist, device):
    """The largest `value` over all ranks (the job's step time)."""
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist, device):
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t)
    return float(t.item())


def gather_to_root(obj, dist, rank, world):
    """Every rank's `obj`, in rank order, on rank 0 (None elsewhere)."""
    out = [None] * world if rank == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
