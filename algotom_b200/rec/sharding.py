"""Sharding slices across GPUs (one process per GPU).

Slices of a stack share only the angles and the centre, so the path shards
without any exchange on the data path: rank r reconstructs its own slab of
slices.  For stacks the slabs are contiguous (``slab_bounds``); for batches
of uneven sinograms the items are dealt out by longest-processing-time
(``lpt_assign``: cost = width^2 x angles, the number of pixel-angle
updates).  The only collective is the optional gather of results to one
rank (``gather_to_root``), through whichever ``torch.distributed`` backend
the process group uses (NCCL between GPUs, gloo in CPU tests).
"""
import heapq

import numpy as np


def slab_bounds(nslice, world, rank):
    """[start, stop) of rank's contiguous slab; sizes differ by at most 1."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank %d of %d" % (rank, world))
    base, extra = divmod(int(nslice), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def lpt_assign(costs, world):
    """Greedy longest-processing-time assignment of items to ranks.

    Returns a list (one per rank) of item indices; items sorted by cost,
    largest first, each to the currently least-loaded rank (ties to the
    lowest rank).  Deterministic, so every rank computes the same plan.
    """
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return out


def item_costs(shapes):
    """Pixel-angle updates of each (nrow, ncol) single-slice item."""
    return [float(r) * float(c) * float(c) for r, c in shapes]


def reconstruct_slab(sinogram, center, world, rank, fn, **kw):
    """Run ``fn`` (e.g. ``fbp_reconstruction``) on this rank's slab of a
    [nrow, nslice, ncol] stack; returns (start, stop, result)."""
    start, stop = slab_bounds(sinogram.shape[1], world, rank)
    return start, stop, fn(sinogram[:, start:stop, :], center, **kw)


def gather_to_root(obj, group=None, root=0):
    """Collect one picklable object per rank on ``root`` (others get None)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    objs = [None] * world if dist.get_rank(group) == root else None
    dist.gather_object(obj, objs, dst=root, group=group)
    return objs
