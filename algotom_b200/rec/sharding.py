"""Sharding slices across GPUs (one process per GPU).

Slices of a stack share only the angles and the centre, so the path shards
without any exchange on the data path: rank r reconstructs its own slab of
slices.  For stacks the slabs are contiguous (``slab_bounds``); for batches
of uneven sinograms the items are dealt out by longest-processing-time
(``lpt_assign``: cost = width^2 x angles, the number of pixel-angle
updates).  The only collective is the optional gather of results to one
rank (``gather_to_root``), through whichever ``torch.distributed`` backend
the process group uses (NCCL between GPUs, gloo in CPU tests).

One slice too large for one GPU's time budget can instead have its angles
split (``fbp_angle_split``): every rank filters and back-projects its
contiguous share of the sinogram's rows, and one in-place ``all_reduce``
sums the partial images -- the only exchange, after all the compute.
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


def _device_partial(rows, angles, center, mask_r2, scale, ramp_win,
                    filter_name, pad, pad_mode, apply_log, ncol):
    """A rank's partial image for ``fbp_angle_split``: the device ramp
    filter of its rows and their back-projection with the full
    reconstruction's mask and scale; float32 [ncol, ncol] on the device."""
    import torch
    from . import reconstruction as R
    if len(rows) == 0:
        return torch.zeros((ncol, ncol), dtype=torch.float32,
                           device=R._device())
    if apply_log:
        R._check_log_input(rows)
    t, _ = R._to_device(rows)
    f = R.filter_sinograms(R._as3(t), pad, pad_mode, apply_log, ramp_win,
                           filter_name)
    rec = R.backproject(f, angles, center, edge_pad=False, mask_r2=mask_r2,
                        scale=scale)
    return rec[:, 0, :].contiguous()


def fbp_angle_split(sinogram, center, angles=None, ratio=1.0, ramp_win=None,
                    filter_name="hann", pad=None, pad_mode="edge",
                    apply_log=True, group=None, partial=None):
    """FBP of one [nrow, ncol] sinogram with its angles split across the
    ranks of ``group``; the arguments are ``fbp_reconstruction``'s
    (``reconstruction.py:362-493``).

    Rank r takes the rows ``slab_bounds(nrow, world, r)`` (with their angles
    and, for a 2-D ``ramp_win`` of nrow rows, its rows), filters them and
    back-projects them with the whole reconstruction's circle mask and
    scale pi/(nrow-1) -- both linear, so they commute with the sum -- and
    one in-place ``all_reduce`` (sum) over the group adds the partial
    images.  Ranks without rows (more ranks than angles) add zeros.  Every
    rank returns the float32 [ncol, ncol] image on its device.
    ``partial(rows, angles, center, mask_r2, scale, ramp_win, filter_name,
    pad, pad_mode, apply_log, ncol)`` makes a rank's partial image as a
    tensor the group's backend can reduce; the default is the device filter
    and back-projection.
    """
    import torch.distributed as dist
    from . import reconstruction as R
    if len(getattr(sinogram, "shape", ())) != 2:
        raise ValueError("fbp_angle_split takes one 2-D [nrow, ncol] "
                         "sinogram")
    nrow, _, ncol, angles = R._validate(sinogram, center, angles)
    if pad is None:
        pad = min(int(0.15 * ncol), 150)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    start, stop = slab_bounds(nrow, world, rank)
    win = ramp_win
    if win is not None and np.ndim(win) == 2 and np.shape(win)[0] == nrow:
        win = win[start:stop]
    fn = _device_partial if partial is None else partial
    part = fn(sinogram[start:stop], angles[start:stop], center,
              R._mask_r2(ratio, center, ncol), R._scale(nrow), win,
              filter_name, pad, pad_mode, apply_log, ncol)
    dist.all_reduce(part, group=group)
    return part
