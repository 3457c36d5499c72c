"""Slice sharding across ranks, checked with 2 gloo processes on the CPU.

The reconstruction itself needs a GPU; in the gloo test each rank runs the
FP64 oracle on its slab (a stand-in with the same slab semantics), and rank
0 gathers and reassembles the stack, which must equal the unsharded result.
The GPU test runs the product's ``fbp_reconstruction`` on each of three
ranks' slabs in turn on one device and gathers them through a one-rank NCCL
group.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from algotom_b200.rec import sharding as SH


def test_slab_bounds_cover_exactly():
    for nslice in (1, 7, 256, 257):
        for world in (1, 2, 3, 8):
            spans = [SH.slab_bounds(nslice, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nslice
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        SH.slab_bounds(10, 2, 2)


def test_lpt_assign_balances_and_is_deterministic():
    rng = np.random.default_rng(0)
    shapes = [(int(rng.integers(361, 3602)), int(rng.integers(512, 4097)))
              for _ in range(64)]
    costs = SH.item_costs(shapes)
    a = SH.lpt_assign(costs, 8)
    assert a == SH.lpt_assign(costs, 8)
    assert sorted(i for part in a for i in part) == list(range(64))
    loads = [sum(costs[i] for i in part) for part in a]
    # LPT bound: max load <= 4/3 of the optimum (>= mean)
    assert max(loads) <= 4.0 / 3.0 * max(np.mean(loads), max(costs)) + 1e-6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_path):
    import torch.distributed as dist
    from algotom_b200 import phantom
    from oracle import fbp_oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nrow, nslice, ncol = 24, 5, 32
        stack = np.stack([phantom.ellipse_sinogram(40 + k, nrow, ncol,
                                                   15.5)[0]
                          for k in range(nslice)], axis=1)
        ang = np.linspace(0, np.pi, nrow, endpoint=False)
        start, stop, part = SH.reconstruct_slab(
            stack, 15.5, world, rank, O.fbp_reconstruction, angles=ang,
            apply_log=False)
        got = SH.gather_to_root((start, stop, part))
        if rank == 0:
            full = np.concatenate([p for _, _, p in sorted(
                got, key=lambda t: t[0])], axis=1)
            ref = O.fbp_reconstruction(stack, 15.5, angles=ang,
                                       apply_log=False)
            np.save(result_path, np.array([full.shape == ref.shape,
                                           np.array_equal(full, ref)]))
    finally:
        dist.destroy_process_group()


def test_two_rank_slab_sharding_gloo(tmp_path):
    result = str(tmp_path / "ok.npy")
    mp.start_processes(_worker, args=(2, _free_port(), result), nprocs=2,
                       join=True, start_method="spawn")
    ok = np.load(result)
    assert ok.all()


@pytest.mark.gpu
def test_device_slabs_match_whole_stack(cuda):
    """reconstruct_slab + the device fbp_reconstruction on the slabs of 3
    ranks (3, 2 and 2 of 7 slices: the 4-, 2- and 1-slice back-projection
    kernels in different mixes), gathered with gather_to_root over NCCL,
    against the whole stack in one call and against the FP64 oracle."""
    import torch.distributed as dist
    from algotom_b200 import phantom
    from algotom_b200.rec import reconstruction as REC
    from oracle import fbp_oracle as O
    nrow, nslice, ncol, cen = 181, 7, 256, 127.3
    stack = np.stack([phantom.ellipse_sinogram(70 + k, nrow, ncol, cen)[0]
                      for k in range(nslice)], axis=1).astype(np.float32)
    ang = np.linspace(0, np.pi, nrow, endpoint=False)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1,
                            device_id=cuda)
    try:
        parts = [SH.reconstruct_slab(stack, cen, 3, r, REC.fbp_reconstruction,
                                     angles=ang, apply_log=False)
                 for r in range(3)]
        got = SH.gather_to_root(parts)[0]
    finally:
        dist.destroy_process_group()
    assert [(a, b) for a, b, _ in got] == [(0, 3), (3, 5), (5, 7)]
    sharded = np.concatenate([p for _, _, p in got], axis=1)
    whole = REC.fbp_reconstruction(stack, cen, angles=ang, apply_log=False)
    ref = O.fbp_reconstruction(stack, cen, angles=ang, apply_log=False)
    assert sharded.shape == whole.shape == ref.shape
    assert O.rel_l2(sharded, whole) < 1e-6
    assert O.rel_l2(sharded, ref) < 1e-5
